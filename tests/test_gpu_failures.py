"""Failure detection without a GPU fault: a device wait that runs out returns a status, and the context
stays usable.

The tuned scan can be gated on a device word that the host publishes; ffbf_debug_scan_unpublished never
publishes it. The kernel polls it a bounded number of times, records the timeout and ends before issuing
any load, so nothing is left in flight; the call reports FFBF_ETIMEOUT. A normal scan on the same context
must then give the oracle's results.
"""
import time

import numpy as np
import pytest

import oracle
from cases import build_inputs
from ffbf_b200 import FFBFError, Filter

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["plain_small", "scale_small"])
def test_unpublished_scan_times_out_and_context_stays_usable(name):
    import torch

    prm, pats, text = build_inputs(name)
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    s = o.scan(text)
    with Filter(prm) as f:
        f.add_patterns(pats)
        d = torch.from_numpy(text).to("cuda")
        n = text.size // 16384 * 16384
        t0 = time.perf_counter()
        with pytest.raises(FFBFError) as ei:
            f.debug_scan_unpublished(d.data_ptr(), n, spins=2000)
        assert ei.value.status == 4, ei.value  # FFBF_ETIMEOUT
        assert time.perf_counter() - t0 < 30.0
        assert not f.get_filters()[1].any(), "a scan that never started sets no feed-forward bits"
        r = f.process(text)
        np.testing.assert_array_equal(r.hit_offsets, s["hits"])
        np.testing.assert_array_equal(r.line_start, s["line_start"])
        np.testing.assert_array_equal(f.get_filters()[1], o.ff)
