"""Parity at the measured workloads' full sizes, against efficient/ffbf's own binary.

The benchmark workloads are checked here at the sizes they are timed at, with the benchmark's seed:
  * plain   10,000 printable patterns, 64 MiB text (LEN 20, 2^24 + 2^28 bits);
  * scale   1,000,000 Zipf-word patterns, 4 GiB text (LEN 32, 2^23 + 2^26 bits): the text ends exactly at
            2^32 bytes;
  * binary  4,000,000 random 16-byte signatures, 8 GiB random text (LEN 16, 2^24 + 2^28 bits): hits and
            lines lie on both sides of 2^32;
  * batched a sample of the 512 batched jobs covering the three geometries of its menu and both scan
            modes, run together through one batch launch.

The reference binary (oracle/_ref, built from the reference's ffbf.cpp) runs over line-aligned shards of
each text on all host cores (oracle/shards.py says why that gives the whole text's answer). The GPU runs
the whole text in one piece, through the device-resident path the benchmark times and through the
host-buffer path (chunked copies overlapping the scan). Compared bit for bit:
  main bit array and `__bloom_filter_` file        vs the reference's
  hit windows and flagged line spans               vs the C restatement (the reference prints neither)
  feed-forward bit array                           vs the OR of the reference shards' arrays
  stdout                                           vs each reference shard's stdout, formatted on that
                                                   shard's 512 KiB chunk grid (and, for texts without
                                                   NUL bytes, the whole text's stdout vs their
                                                   concatenation)
  pruned pattern file and __index_ file            vs the reference's filterPhrases over that array
  exact (offset, pattern id) matches               vs the C restatement
"""
import os
import time

import numpy as np
import pytest

import oracle
from oracle.shards import ReferenceShards, host_cores, line_shards, oracle_scan_shards

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

SEED = 2024  # the benchmark's seed


@pytest.fixture(scope="module", autouse=True)
def require_gpu():
    import torch
    assert torch.cuda.is_available(), "the gpu tests need a CUDA device"


def n_shards(nbytes):
    return max(1, min(2 * host_cores(), nbytes // (4 << 20)))


def check_job(f, prm, pats, text, got, ff, label):
    """Compares one scanned job (`got` = its ScanOutput, `ff` = its feed-forward array) with the reference
    binary run over line-aligned shards and with the C restatement. Returns a short summary."""
    from ffbf_b200.lib import format_spans

    binary = oracle.ref_binary(prm)
    assert binary is not None, f"no reference binary for {prm} in oracle/_ref"
    shards = line_shards(text, n_shards(text.size))
    t0 = time.time()
    with ReferenceShards(binary, pats, text, shards) as ref:
        ref.prepare()
        ref.run(dump_ff=True)
        main, _ = f.get_filters()
        assert np.array_equal(main, ref.main), f"{label}: main bit array differs from the reference's"
        assert f.save_filter() == ref.bloom, f"{label}: __bloom_filter_ file differs from the reference's"

        hits, ls, le, off_ff = oracle_scan_shards(prm, ref.main, text, shards)
        np.testing.assert_array_equal(got.hit_offsets, hits, err_msg=f"{label}: hit windows")
        np.testing.assert_array_equal(got.line_start, ls, err_msg=f"{label}: line starts")
        np.testing.assert_array_equal(got.line_end, le, err_msg=f"{label}: line ends")

        ref_ff = ref.ff_or()
        assert np.array_equal(ref_ff, off_ff), f"{label}: the restatement's feed-forward array differs (oracle)"
        assert np.array_equal(ff, ref_ff), f"{label}: feed-forward bit array differs from the reference's"

        # stdout, shard by shard on each shard's own chunk grid
        for i, (a, b) in enumerate(shards):
            lo, hi = np.searchsorted(got.line_start, [a, b])
            mine = format_spans(text[a:b], got.line_start[lo:hi] - np.uint64(a), got.line_end[lo:hi] - np.uint64(a))
            assert mine == ref.stdout(i), f"{label}: stdout of shard {i} [{a}, {b}) differs"
        if not any(np.any(text[i:i + (1 << 28)] == 0) for i in range(0, text.size, 1 << 28)):
            whole = f.format_lines(text)
            assert whole == b"".join(ref.stdout(i) for i in range(len(shards))), f"{label}: stdout differs"

        ids = f.filter_phrases()
        pruned, index = f.format_pruned()
        r_pruned, r_index = ref.prune_with_ff(ref_ff)
        assert pruned == r_pruned, f"{label}: pruned pattern file differs from the reference's"
        assert index == r_index, f"{label}: __index_ file differs from the reference's"

        off, pid = f.verify()
        o = oracle.Oracle.from_params(prm)
        ooff, opid = o.verify(pats, ids, text, hits)
        np.testing.assert_array_equal(off, ooff, err_msg=f"{label}: exact match offsets")
        np.testing.assert_array_equal(pid, opid, err_msg=f"{label}: exact match pattern ids")
    return dict(hits=int(hits.size), lines=int(ls.size), pruned=int(ids.size), matches=int(off.size),
                shards=len(shards), check_s=round(time.time() - t0, 1))


def scan_both_paths(f, text):
    """The device-resident scan (the benchmark's timed path) and the host-buffer scan; both must agree.
    Returns the scan output and the feed-forward array."""
    import torch

    n = int(text.size)
    d_text = torch.empty(n + 64, dtype=torch.uint8, device="cuda")
    d_text[:n].copy_(torch.from_numpy(text))
    torch.cuda.synchronize()
    f.clear_ff()
    f.process_device(d_text.data_ptr(), n)
    dev = f.collect()
    _, ff_dev = f.get_filters()
    del d_text
    torch.cuda.empty_cache()
    f.clear_ff()
    host = f.process(text)
    _, ff_host = f.get_filters()
    np.testing.assert_array_equal(dev.hit_offsets, host.hit_offsets)
    np.testing.assert_array_equal(dev.line_start, host.line_start)
    np.testing.assert_array_equal(dev.line_end, host.line_end)
    assert np.array_equal(ff_dev, ff_host)
    return host, ff_host


@pytest.mark.parametrize("name", ["plain", "scale", "binary"])
def test_full_size_workload_matches_reference(name):
    from ffbf_b200 import Filter
    from ffbf_b200 import datagen as dg

    wl = {"plain": dg.plain, "scale": dg.scale, "binary": dg.binary}[name]()
    pats = wl.patterns(SEED)
    text = wl.text(SEED, pats)
    with Filter(wl.params) as f:
        f.add_patterns(pats)
        got, ff = scan_both_paths(f, text)
        cfg = f.config()
        summary = check_job(f, wl.params, pats, text, got, ff, name)
    if name == "binary":
        # offsets on both sides of 2^32: a 32-bit truncation anywhere would show
        assert got.hit_offsets[0] < 2**32 < got.hit_offsets[-1]
        assert got.line_start[0] < 2**32 < got.line_start[-1]
    print(f"{name}: {wl.n_patterns} patterns, {text.size} text bytes, scan config {cfg}: {summary}")


def test_batched_sample_matches_reference():
    """Jobs of the batched workload (its seed, sizes and geometry menu) run together in one batch launch
    after the autotuner has picked each one's configuration; each job's results against the reference."""
    import torch

    from ffbf_b200 import Batch, Filter
    from ffbf_b200 import datagen as dg

    jobs = dg.batched(seed=SEED)
    picked = []
    for cache_bits in (1 << 20, 1 << 22, 1 << 23):
        mine = [j for j, w in enumerate(jobs) if w.params.cache_bits == cache_bits]
        mine.sort(key=lambda j: jobs[j].text_bytes)
        # the largest text of the geometry, a middle one and the smallest
        for j in (mine[-1], mine[len(mine) // 2], mine[0]):
            if j not in picked:
                picked.append(j)
    ws = [jobs[j] for j in picked]
    pats = [w.patterns(w.seed) for w in ws]
    texts = [w.text(w.seed, p) for w, p in zip(ws, pats)]
    offs, total = [], 0
    for t in texts:
        offs.append(total)
        total += (t.size + 255) // 256 * 256
    host = np.zeros(total + 64, dtype=np.uint8)
    for t, o in zip(texts, offs):
        host[o:o + t.size] = t
    d_all = torch.from_numpy(host).cuda()
    filters = [Filter(w.params) for w in ws]
    try:
        for f, p in zip(filters, pats):
            f.add_patterns(p)
        with Batch(0) as b:
            for f, t, o in zip(filters, texts, offs):
                b.add(f, d_all.data_ptr() + o, t.size)
            b.autotune(16 << 20)
            b.prepare()
            b.launch()
            b.wait()
            modes = set()
            for j, f, w, p, t in zip(picked, filters, ws, pats, texts):
                got = f.collect()
                _, ff = f.get_filters()
                modes.add(f.config()[1])
                s = check_job(f, w.params, p, t, got, ff, f"batched[{j}]")
                print(f"batched[{j}]: {w.n_patterns} patterns, {t.size} bytes, C=2^{w.params.cache_bits.bit_length() - 1}, "
                      f"config {f.config()}: {s}")
        assert 1 in modes and modes & {0, 2, 3}, f"the sample should run the dense and a shared-memory mode, ran {modes}"
    finally:
        for f in filters:
            f.close()
