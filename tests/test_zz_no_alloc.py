"""ffbf_scan_static, the scan that allocates nothing, against the regular ffbf_scan.

ffbf_scan_static is for callers that may not let the library call cudaMalloc (their allocator owns all
device memory, or allocation is forbidden where they call us). It runs the scan with its scratch in a fixed
device array of the library, so it must give exactly what ffbf_scan gives on the same inputs: the same hit
windows, the same lines and the same feed-forward bits. Two calls in a row on different inputs also check
that the shared scratch left over from one call does not leak into the next.
"""
import ctypes

import numpy as np
import pytest

from cases import build_inputs
from ffbf_b200 import Filter, load_library

pytestmark = pytest.mark.gpu

MAX_HITS = 1 << 16


def regular_scan(name):
    prm, pats, text = build_inputs(name)
    with Filter(prm) as f:
        f.add_patterns(pats)
        r = f.process(text)
        main, ff = f.get_filters()
    return prm, text, main, ff, r


def test_static_scan_matches_regular_scan_on_two_calls():
    import torch

    assert torch.cuda.is_available()
    lib = load_library()
    dev = torch.device("cuda", 0)
    offs = torch.empty(MAX_HITS, dtype=torch.int64, device=dev)
    ls = torch.empty(MAX_HITS, dtype=torch.int64, device=dev)
    le = torch.empty(MAX_HITS, dtype=torch.int64, device=dev)
    for name in ("scale_small", "edge_chunks"):
        prm, text, main, ff_ref, ref = regular_scan(name)
        d_main = torch.from_numpy(main.view(np.int32).copy()).to(dev)
        d_ff = torch.zeros_like(d_main)
        d_text = torch.from_numpy(text).to(dev)
        n = ctypes.c_uint32(12345)
        stream = torch.cuda.current_stream(dev)
        st = lib.ffbf_scan_static(ctypes.byref(prm), ctypes.c_void_p(d_main.data_ptr()),
                                  ctypes.c_void_p(d_ff.data_ptr()), ctypes.c_void_p(d_text.data_ptr()), text.size,
                                  ctypes.c_void_p(offs.data_ptr()), ctypes.c_void_p(ls.data_ptr()),
                                  ctypes.c_void_p(le.data_ptr()), ctypes.byref(n), ctypes.c_void_p(stream.cuda_stream))
        assert st == 0, f"ffbf_scan_static returned {st}"
        k = n.value
        assert k == ref.hit_offsets.size
        o = offs[:k].cpu().numpy().astype(np.uint64)
        s = ls[:k].cpu().numpy().astype(np.uint64)
        e = le[:k].cpu().numpy().astype(np.uint64)
        order = np.argsort(o, kind="stable")
        np.testing.assert_array_equal(o[order], ref.hit_offsets)
        # one line per distinct start, in text order
        starts, first = np.unique(s[order], return_index=True)
        np.testing.assert_array_equal(starts, ref.line_start)
        np.testing.assert_array_equal(e[order][first], ref.line_end)
        np.testing.assert_array_equal(d_ff.cpu().numpy().view(np.uint8), ff_ref)


def test_static_scan_rejects_oversized_text():
    lib = load_library()
    prm, _, _ = build_inputs("plain_small")
    n = ctypes.c_uint32()
    dummy = ctypes.c_void_p(256)
    st = lib.ffbf_scan_static(ctypes.byref(prm), dummy, dummy, dummy, (1 << 30) + 1, dummy, dummy, dummy,
                              ctypes.byref(n), None)
    assert st == 1
