"""The multi-GPU path's host logic (ffbf_b200.replicas) with two gloo ranks on CPU.

Each rank scans its own replica's workload (seed + rank) with the oracle and reports bytes and a time; the
whole-job throughput must be every rank's bytes over the slowest rank's time, on every rank. The replicas'
texts differ, and each replica's hits are its own workload's (no data crosses ranks).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    import oracle
    from ffbf_b200 import datagen as dg
    from ffbf_b200.replicas import Replicas

    rep = Replicas.from_env("gloo", timeout_s=60)
    try:
        wl = dg.plain(text_bytes=256 * 1024, n_patterns=200)
        seed = rep.seed(11)
        pats = wl.patterns(seed)
        text = wl.text(seed, pats)
        o = oracle.Oracle.from_params(wl.params)
        o.build(pats)
        hits = o.scan(text)["hits"]
        rep.barrier()
        seconds = 1.0 + rank  # a stand-in device time: rank 1 is the slowest
        thr = rep.throughput(text.size, seconds)
        q.put((rank, seed, int(text.size), int(hits.size), hash(text.tobytes()), thr, rep.max(rank * 10.0),
               rep.sum(1.0)))
    finally:
        rep.close()


@pytest.mark.timeout(300)
def test_two_gloo_replicas_report_whole_job_throughput():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
        assert p.exitcode == 0, f"rank exited with {p.exitcode}"
    got = sorted(q.get() for _ in range(world))
    seeds = [g[1] for g in got]
    assert seeds == [11, 12], "each replica scans its own seed's workload"
    assert got[0][4] != got[1][4], "replica texts must differ"
    total = sum(g[2] for g in got)
    for g in got:
        assert g[5] == pytest.approx(total / 2.0)  # all bytes over the slowest rank's 2.0 s
        assert g[6] == 10.0 and g[7] == 2.0
        assert g[3] > 0


def test_single_process_replicas_need_no_process_group(monkeypatch):
    from ffbf_b200.replicas import Replicas

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    rep = Replicas.from_env("gloo")
    assert (rep.world, rep.rank) == (1, 0)
    assert rep.seed(5) == 5
    rep.barrier()
    assert rep.throughput(1000, 2.0) == pytest.approx(500.0)
    assert np.isclose(rep.max(3.0), 3.0) and np.isclose(rep.sum(3.0), 3.0)
    rep.close()
