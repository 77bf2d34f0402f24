"""The scan server (ffbf_server_*): every request's hits and candidate lines equal the oracle's scan of its
text, whether the request runs alone or batched with requests of other sets; each set's feed-forward filter
ends as the union of what its requests set, as successive ffbf_scan calls would leave it.

The sets cover the tuned kernel's sparse and dense modes, a geometry only the generic kernel handles, a
filter so full that a request overflows its slot's hit buffer (the server then grows it and rescans), and
request sizes from empty through ragged tile ends to several MiB. A small text arena and few slots make
admission wait for room.
"""
import time

import numpy as np
import pytest

import oracle
from cases import build_inputs
from ffbf_b200 import FFBFError, Filter, Server

pytestmark = pytest.mark.gpu

SETS = ["scale_small", "plain_small", "smem_cache", "k11_s0_len63", "hit_flood"]


def request_slices(n, seed):
    """(offset, length) pairs over a text of n bytes."""
    rng = np.random.default_rng(seed)
    sizes = [0, 100, 5000, 16384 + 7, 3 * 16384, 200_000, 1 << 20, n]
    out = []
    for sz in sizes:
        sz = min(sz, n)
        off = int(rng.integers(0, n - sz + 1)) if sz < n else 0
        out.append((off, sz))
    return out


@pytest.fixture(scope="module")
def workload():
    sets = []
    for i, name in enumerate(SETS):
        prm, pats, text = build_inputs(name)
        sets.append((name, prm, pats, text, request_slices(text.size, 100 + i)))
    # requests interleaved across sets: (set index, offset, length)
    reqs = []
    for k in range(max(len(s[4]) for s in sets)):
        for si, s in enumerate(sets):
            if k < len(s[4]):
                reqs.append((si,) + s[4][k])
    return sets, reqs


def expected(sets, reqs):
    """Oracle results per request and each set's feed-forward filter after all of its requests."""
    orcs = []
    for _, prm, pats, _, _ in sets:
        o = oracle.Oracle.from_params(prm)
        o.build(pats)
        orcs.append(o)
    res = []
    for si, off, ln in reqs:
        s = orcs[si].scan(sets[si][3][off:off + ln])
        res.append((s["hits"], s["line_start"], s["line_end"]))
    return res, [o.ff for o in orcs]


def make_filters(sets):
    fs = []
    for _, prm, pats, _, _ in sets:
        f = Filter(prm)
        f.add_patterns(pats)
        fs.append(f)
    return fs


def drain(srv, n, timeout=120.0):
    got = {}
    t_end = time.time() + timeout
    while len(got) < n:
        assert time.time() < t_end, f"server finished {len(got)} of {n} requests"
        for r in srv.poll(wait_us=100_000):
            got[r.request_id] = r
    return got


def check(results, want, reqs, ids, label):
    for i, (si, off, ln) in enumerate(reqs):
        r = results[ids[i]]
        assert r.status == 0, f"{label}: request {i} status {r.status}"
        assert r.text_len == ln
        hits, ls, le = want[i]
        np.testing.assert_array_equal(r.hit_offsets, hits, err_msg=f"{label} request {i} (set {si}, {ln} B)")
        np.testing.assert_array_equal(r.line_start, ls, err_msg=f"{label} request {i}")
        np.testing.assert_array_equal(r.line_end, le, err_msg=f"{label} request {i}")


def test_server_requests_alone_and_in_the_mix_equal_oracle(workload):
    sets, reqs = workload
    want, want_ff = expected(sets, reqs)
    largest = max(ln for _, _, ln in reqs)

    # alone: one request in the server at a time
    fs = make_filters(sets)
    with Server(0, arena_bytes=largest + (1 << 20), slots=2) as srv:
        sids = [srv.add_set(f) for f in fs]
        ids, results = [], {}
        for si, off, ln in reqs:
            rid = srv.submit(sids[si], sets[si][3][off:off + ln])
            ids.append(rid)
            results.update(drain(srv, 1))
        check(results, want, reqs, ids, "alone")
        assert srv.stats()["max_batch"] == 1
    for f, ff in zip(fs, want_ff):
        np.testing.assert_array_equal(f.get_filters()[1], ff)
        f.close()

    # in the mix: everything submitted at once; the arena holds about two of the largest texts and four
    # slots are free, so requests wait for admission and batches mix sets
    fs = make_filters(sets)
    with Server(0, arena_bytes=2 * largest + (1 << 20), slots=4) as srv:
        sids = [srv.add_set(f) for f in fs]
        ids = [srv.submit(sids[si], sets[si][3][off:off + ln]) for si, off, ln in reqs]
        results = drain(srv, len(reqs))
        check(results, want, reqs, ids, "mix")
        st = srv.stats()
        assert st["requests_done"] == len(reqs)
        assert st["max_batch"] > 1, "requests of several sets should have shared a launch"
        assert st["bytes_scanned"] == sum(ln for _, _, ln in reqs)
    for f, ff in zip(fs, want_ff):
        np.testing.assert_array_equal(f.get_filters()[1], ff)
        f.close()


def test_server_refuses_request_larger_than_arena():
    prm, pats, text = build_inputs("plain_small")
    with Filter(prm) as f:
        f.add_patterns(pats)
        with Server(0, arena_bytes=1 << 20, slots=2) as srv:
            sid = srv.add_set(f)
            with pytest.raises(FFBFError) as ei:
                srv.submit(sid, text[: 2 << 20])
            assert ei.value.status == 1  # FFBF_EINVAL
            rid = srv.submit(sid, text[:4096])
            got = drain(srv, 1)
            assert got[rid].status == 0
            # sets are fixed once requests flow
            with Filter(prm) as g:
                with pytest.raises(FFBFError):
                    srv.add_set(g)


def test_server_admission_waits_for_device_memory():
    """Admission follows the device's free memory, which every context's allocations reduce: while another
    allocation holds all but 1 GiB of it, a request larger than the room the server already holds waits (it is
    not refused and does not fail) and a request that fits that room still runs; once the memory is freed the
    waiting request is admitted and its results equal a plain ffbf_scan of its text. Room grown for it goes
    back to the device after the server has been idle for a while."""
    import torch

    prm, pats, text = build_inputs("plain_small")
    reps = (1280 << 20) // text.size + 1
    big = np.ascontiguousarray(np.tile(text, reps))  # ~1.25 GiB: more than the server's first segment
    small = text[: 1 << 20]
    with Filter(prm) as g:
        g.add_patterns(pats)
        want_big = g.process(big)
        want_small = g.process(small)
    with Filter(prm) as f:
        f.add_patterns(pats)
        with Server(0, arena_bytes=0, slots=4) as srv:
            sid = srv.add_set(f)
            first = srv.stats()["arena_bytes"]
            assert first < big.size
            free, _ = torch.cuda.mem_get_info()
            # 1 GiB stays free: the server may neither add a segment for the large text nor replace its first
            # one, since either would leave less than its 1 GiB reserve
            blocker = torch.empty(free - (1 << 30), dtype=torch.uint8, device="cuda")
            try:
                rid_small = srv.submit(sid, small)
                got = drain(srv, 1)
                assert got[rid_small].status == 0
                np.testing.assert_array_equal(got[rid_small].hit_offsets, want_small.hit_offsets)
                rid_big = srv.submit(sid, big)
                t_end = time.time() + 1.0
                while time.time() < t_end:
                    assert not srv.poll(wait_us=50_000), "the large request ran while the memory was held"
                assert srv.stats()["arena_bytes"] == first
            finally:
                del blocker
                torch.cuda.empty_cache()
            got = drain(srv, 1)
            r = got[rid_big]
            assert r.status == 0
            np.testing.assert_array_equal(r.hit_offsets, want_big.hit_offsets)
            np.testing.assert_array_equal(r.line_start, want_big.line_start)
            np.testing.assert_array_equal(r.line_end, want_big.line_end)
            assert r.t_admit - r.t_submit >= 0.9, "admission should have waited for the memory"
            assert srv.stats()["arena_bytes"] > first
            t_end = time.time() + 5.0
            while srv.stats()["arena_bytes"] > first and time.time() < t_end:
                time.sleep(0.05)
            assert srv.stats()["arena_bytes"] == first, "grown room should go back to the device when idle"


def test_server_cap_admits_a_request_larger_than_its_first_segment():
    """With a cap of 2 GiB the arena starts as one 1 GiB segment and may not grow past the cap by adding a
    second one, so a 1.5 GiB request is admitted by replacing the idle arena with one segment that holds it;
    once the server idles again the arena returns to its first size."""
    prm, pats, text = build_inputs("plain_small")
    big = np.ascontiguousarray(np.tile(text, (1536 << 20) // text.size + 1)[: 1536 << 20])
    with Filter(prm) as g:
        g.add_patterns(pats)
        want = g.process(big)
    with Filter(prm) as f:
        f.add_patterns(pats)
        with Server(0, arena_bytes=2 << 30, slots=2) as srv:
            sid = srv.add_set(f)
            first = srv.stats()["arena_bytes"]
            assert first == 1 << 30
            rid = srv.submit(sid, big)
            r = drain(srv, 1)[rid]
            assert r.status == 0
            np.testing.assert_array_equal(r.hit_offsets, want.hit_offsets)
            np.testing.assert_array_equal(r.line_start, want.line_start)
            t_end = time.time() + 5.0
            while srv.stats()["arena_bytes"] != first and time.time() < t_end:
                time.sleep(0.05)
            assert srv.stats()["arena_bytes"] == first
