"""ffbf_scan_static, the scan that allocates nothing, against the regular ffbf_scan and the oracle.

ffbf_scan_static is for callers that may not let the library call cudaMalloc (their allocator owns all
device memory, or allocation is forbidden where they call us). It runs the scan with its scratch in a fixed
device array of the library, so it must give exactly what ffbf_scan gives on the same inputs: the same hit
windows, the same lines and the same feed-forward bits. Two calls in a row on different inputs also check
that the shared scratch left over from one call does not leak into the next. The other cases: a text of
more than 4096 16-KiB tiles with a line spanning hundreds of them, against the oracle; more hit windows
than the fixed array holds (FFBF_ENOMEM_DEVICE with the full count and a subset of the hits); and the
device's free memory, unchanged across a call.

This file is collected last, so a run that stops at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

import oracle
from cases import build_inputs
from ffbf_b200 import Filter, load_library
from ffbf_b200 import datagen as dg

pytestmark = pytest.mark.gpu

MAX_HITS = 1 << 16
FFBF_ENOMEM_DEVICE = 2


def regular_scan(prm, pats, text):
    with Filter(prm) as f:
        f.add_patterns(pats)
        r = f.process(text)
        main, ff = f.get_filters()
    return main, ff, r


class Static:
    """Device buffers for ffbf_scan_static's outputs, and the call through the C ABI."""

    def __init__(self):
        import torch
        assert torch.cuda.is_available()
        self.torch = torch
        self.lib = load_library()
        self.dev = torch.device("cuda", 0)
        self.offs = torch.empty(MAX_HITS, dtype=torch.int64, device=self.dev)
        self.ls = torch.empty(MAX_HITS, dtype=torch.int64, device=self.dev)
        self.le = torch.empty(MAX_HITS, dtype=torch.int64, device=self.dev)

    def upload(self, main, text):
        t = self.torch
        d_main = t.from_numpy(main.view(np.int32).copy()).to(self.dev)
        d_text = t.empty(text.size + 64, dtype=t.uint8, device=self.dev)
        d_text[:text.size].copy_(t.from_numpy(text))
        return d_main, t.zeros_like(d_main), d_text

    def call(self, prm, d_main, d_ff, d_text, n):
        cnt = ctypes.c_uint32(12345)
        stream = self.torch.cuda.current_stream(self.dev)
        st = self.lib.ffbf_scan_static(ctypes.byref(prm), ctypes.c_void_p(d_main.data_ptr()),
                                       ctypes.c_void_p(d_ff.data_ptr()), ctypes.c_void_p(d_text.data_ptr()), n,
                                       ctypes.c_void_p(self.offs.data_ptr()), ctypes.c_void_p(self.ls.data_ptr()),
                                       ctypes.c_void_p(self.le.data_ptr()), ctypes.byref(cnt),
                                       ctypes.c_void_p(stream.cuda_stream))
        return st, cnt.value

    def results(self, k):
        """(offsets, line starts, line ends) of the first k records, sorted by offset."""
        k = min(k, MAX_HITS)
        o = self.offs[:k].cpu().numpy().astype(np.uint64)
        s = self.ls[:k].cpu().numpy().astype(np.uint64)
        e = self.le[:k].cpu().numpy().astype(np.uint64)
        order = np.argsort(o, kind="stable")
        return o[order], s[order], e[order]


def check_lines(s, e, line_start, line_end):
    """One line per distinct start, in text order, equal to the expected flagged lines."""
    starts, first = np.unique(s, return_index=True)
    np.testing.assert_array_equal(starts, line_start)
    np.testing.assert_array_equal(e[first], line_end)


def test_static_scan_matches_regular_scan_on_two_calls():
    sc = Static()
    for name in ("scale_small", "edge_chunks"):
        prm, pats, text = build_inputs(name)
        main, ff_ref, ref = regular_scan(prm, pats, text)
        d_main, d_ff, d_text = sc.upload(main, text)
        st, k = sc.call(prm, d_main, d_ff, d_text, text.size)
        assert st == 0, f"ffbf_scan_static returned {st}"
        assert k == ref.hit_offsets.size
        o, s, e = sc.results(k)
        np.testing.assert_array_equal(o, ref.hit_offsets)
        check_lines(s, e, ref.line_start, ref.line_end)
        np.testing.assert_array_equal(d_ff.cpu().numpy().view(np.uint8), ff_ref)


def test_static_scan_of_many_tiles_matches_oracle():
    """100 MiB + 13 bytes (6401 tiles; the length is not a multiple of 16): a 3 MiB line across ~190 tiles
    with hits in it, a hit in the unterminated last line, against the oracle's processFile."""
    wl = dg.plain(text_bytes=(100 << 20) + 13, n_patterns=5000)
    prm = wl.params
    pats = wl.patterns(31)
    text = wl.text(31, pats)
    plist = pats.tobytes().split(b"\n")
    lo, hi = 40 << 20, 43 << 20
    seg = text[lo:hi]
    seg[seg == 10] = 32  # one long line
    for i, pos in enumerate(range(lo + 1000, hi - 1000, 400_000)):
        p = np.frombuffer(plist[i], dtype=np.uint8)
        text[pos:pos + p.size] = p
    tail = np.frombuffer(plist[7], dtype=np.uint8)
    text[-60:] = 32
    text[-50:-50 + tail.size] = tail
    o_ = oracle.Oracle.from_params(prm)
    o_.build(pats)
    s_ = o_.scan(text)
    sc = Static()
    d_main, d_ff, d_text = sc.upload(o_.main, text)
    st, k = sc.call(prm, d_main, d_ff, d_text, text.size)
    assert st == 0, f"ffbf_scan_static returned {st}"
    assert k == s_["hits"].size <= MAX_HITS
    o, s, e = sc.results(k)
    np.testing.assert_array_equal(o, s_["hits"])
    check_lines(s, e, s_["line_start"], s_["line_end"])
    assert (s_["line_end"] - s_["line_start"] > (3 << 20) - 4096).any(), "the long line should be flagged"
    assert s_["line_end"][-1] == text.size, "the unterminated last line should be flagged"
    np.testing.assert_array_equal(d_ff.cpu().numpy().view(np.uint8), o_.ff)


def test_static_scan_overflow_reports_full_count():
    """More hit windows than FFBF_STATIC_MAX_HITS: FFBF_ENOMEM_DEVICE, *n_hits = the full count, the arrays a
    subset of the hits with their lines, and every feed-forward bit set (the scan itself is not cut)."""
    prm, pats, text = build_inputs("hit_flood")
    text = np.concatenate([text] * 2)  # ~600k windows, most of them hits
    main, ff_ref, ref = regular_scan(prm, pats, text)
    assert ref.hit_offsets.size > MAX_HITS
    sc = Static()
    d_main, d_ff, d_text = sc.upload(main, text)
    st, k = sc.call(prm, d_main, d_ff, d_text, text.size)
    assert st == FFBF_ENOMEM_DEVICE
    assert k == ref.hit_offsets.size
    o, s, e = sc.results(MAX_HITS)
    assert np.unique(o).size == MAX_HITS
    idx = np.searchsorted(ref.hit_offsets, o)
    np.testing.assert_array_equal(ref.hit_offsets[idx], o)
    # each returned hit's line is the regular scan's line holding that window
    li = np.searchsorted(ref.line_start, o, side="right") - 1
    np.testing.assert_array_equal(s, ref.line_start[li])
    np.testing.assert_array_equal(e, ref.line_end[li])
    np.testing.assert_array_equal(d_ff.cpu().numpy().view(np.uint8), ff_ref)


def test_static_scan_allocates_no_device_memory():
    """After one call (which loads the library's kernels and the array's module), another call leaves the
    device's free memory exactly where it was."""
    sc = Static()
    torch = sc.torch
    prm, pats, text = build_inputs("plain_small")
    main, ff_ref, ref = regular_scan(prm, pats, text)
    d_main, d_ff, d_text = sc.upload(main, text)
    assert sc.call(prm, d_main, d_ff, d_text, text.size) == (0, ref.hit_offsets.size)
    torch.cuda.synchronize()
    d_ff.zero_()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(sc.dev)
    st, k = sc.call(prm, d_main, d_ff, d_text, text.size)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(sc.dev)
    assert (st, k) == (0, ref.hit_offsets.size)
    assert free1 == free0, f"free device memory moved by {free0 - free1} bytes during the call"
    np.testing.assert_array_equal(d_ff.cpu().numpy().view(np.uint8), ff_ref)


def test_static_scan_rejects_oversized_text():
    lib = load_library()
    prm, _, _ = build_inputs("plain_small")
    n = ctypes.c_uint32()
    dummy = ctypes.c_void_p(256)
    st = lib.ffbf_scan_static(ctypes.byref(prm), dummy, dummy, dummy, (1 << 30) + 1, dummy, dummy, dummy,
                              ctypes.byref(n), None)
    assert st == 1
