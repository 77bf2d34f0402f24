"""Batched scans (ffbf_batch_*) and the autotuner: every job's results equal the oracle's, alone or in the mix.

The batch mixes jobs that run in different launches of one graph: LEN 20/32/24/16 (one tuned launch per LEN
and configuration), sparse and dense filters, texts that are not a multiple of the 16 KiB tile (generic tail
tiles), a text shorter than one tile and a geometry only the generic kernel covers (LEN 63).
"""
import numpy as np
import pytest

import oracle
from cases import build_inputs
from ffbf_b200 import Batch, Filter

pytestmark = pytest.mark.gpu

BATCH_CASES = ["plain_small", "scale_small", "binary_small", "smem_cache", "dense_fp", "edge_chunks",
               "k11_s0_len63", "len19_default", "pats_no_newline", "hit_flood"]


def expected(name):
    prm, pats, text = build_inputs(name)
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    s = o.scan(text)
    return prm, pats, text, o, s


def test_batch_results_equal_oracle_on_two_launches():
    import torch

    dev = torch.device("cuda", 0)
    jobs = []
    with Batch(0) as b:
        for name in BATCH_CASES:
            prm, pats, text, o, s = expected(name)
            f = Filter(prm)
            f.add_patterns(pats)
            d_text = torch.from_numpy(text).to(dev) if text.size else torch.zeros(16, dtype=torch.uint8, device=dev)
            b.add(f, d_text.data_ptr(), text.size)
            jobs.append((name, f, d_text, o, s))
        # a tiny text: shorter than one 16 KiB tile
        prm, pats, text, o, _ = expected("plain_small")
        small = text[:5000].copy()
        o_small = oracle.Oracle.from_params(prm)
        o_small.build(pats)
        s_small = o_small.scan(small)
        f_small = Filter(prm)
        f_small.add_patterns(pats)
        d_small = torch.from_numpy(small).to(dev)
        b.add(f_small, d_small.data_ptr(), small.size)
        jobs.append(("tiny", f_small, d_small, o_small, s_small))
        b.prepare()
        for launch in range(2):
            if launch == 1:
                # tuning between launches changes configurations, never results
                assert b.autotune(1 << 20) >= 1
            b.launch()
            b.wait()
            for name, f, _, o, s in jobs:
                r = f.collect()
                np.testing.assert_array_equal(r.hit_offsets, s["hits"], err_msg=f"{name} launch {launch}")
                np.testing.assert_array_equal(r.line_start, s["line_start"], err_msg=name)
                np.testing.assert_array_equal(r.line_end, s["line_end"], err_msg=name)
                np.testing.assert_array_equal(f.get_filters()[1], o.ff, err_msg=name)
    for _, f, _, _, _ in jobs:
        f.close()


def test_batch_job_equals_plain_scan_of_same_job():
    """A job's results do not depend on which other jobs share the launch."""
    import torch

    dev = torch.device("cuda", 0)
    prm, pats, text, o, s = expected("scale_small")
    with Filter(prm) as alone:
        alone.add_patterns(pats)
        ref = alone.process(text)
    with Batch(0) as b:
        filters = []
        texts = []
        for k in range(5):  # the same job five times, in five contexts
            f = Filter(prm)
            f.add_patterns(pats)
            t = torch.from_numpy(text).to(dev)
            b.add(f, t.data_ptr(), text.size)
            filters.append(f)
            texts.append(t)
        b.launch()
        b.wait()
        for f in filters:
            r = f.collect()
            np.testing.assert_array_equal(r.hit_offsets, ref.hit_offsets)
            np.testing.assert_array_equal(r.line_start, ref.line_start)
            f.close()


@pytest.mark.parametrize("name", ["scale_small", "plain_small"])
def test_autotune_keeps_results(name):
    import torch

    prm, pats, text, o, s = expected(name)
    with Filter(prm) as f:
        f.add_patterns(pats)
        d = torch.from_numpy(text).to("cuda")
        threads, mode = f.autotune(d.data_ptr(), (text.size // 16384) * 16384)
        assert threads in (192, 256, 384, 512) and mode in (0, 1, 2, 3)
        assert not f.get_filters()[1].any(), "autotuning must not leave feed-forward bits behind"
        r = f.process(text)
        np.testing.assert_array_equal(r.hit_offsets, s["hits"])
        np.testing.assert_array_equal(f.get_filters()[1], o.ff)
