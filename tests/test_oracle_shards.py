"""The shard machinery (oracle/shards.py) that the full-size parity tests rest on, checked on the CPU against
single whole-text runs of the reference binary: the OR of the shards' feed-forward arrays, the pruned file
and index that filterPhrases prints from it, the concatenated stdout, and the restatement's hits."""
import numpy as np
import pytest

import oracle
from ffbf_b200 import datagen as dg
from oracle.shards import ReferenceShards, line_shards, oracle_scan_shards


def test_line_shards_cover_the_text_at_line_ends():
    rng = np.random.default_rng(3)
    text = rng.integers(32, 127, 1 << 20, dtype=np.uint8)
    text[rng.integers(0, text.size, 300)] = 10
    for n in (1, 2, 7, 64):
        sh = line_shards(text, n)
        assert sh[0][0] == 0 and sh[-1][1] == text.size
        assert all(b == c for (_, b), (c, _) in zip(sh, sh[1:]))
        assert all(text[b - 1] == 10 for _, b in sh[:-1])
    no_nl = np.full(1000, 65, dtype=np.uint8)
    assert line_shards(no_nl, 4) == [(0, 1000)]
    one = no_nl.copy()
    one[-1] = 10
    assert line_shards(one, 4) == [(0, 1000)]


@pytest.mark.parametrize("kind", ["plain", "binary"])
def test_sharded_reference_equals_one_whole_run(kind):
    if kind == "plain":
        wl = dg.plain(text_bytes=6 << 20, n_patterns=3000)
    else:
        wl = dg.binary(text_bytes=6 << 20, n_patterns=200_000)
    binary = oracle.ref_binary(wl.params)
    if binary is None:
        pytest.skip("reference binary for this geometry not built (oracle/_ref)")
    pats = wl.patterns(11)
    text = wl.text(11, pats)
    whole = oracle.run_reference(binary, pats, text=text.tobytes())
    nb = wl.params.nbits // 8
    shards = line_shards(text, 5)
    assert len(shards) == 5
    o = oracle.Oracle.from_params(wl.params)
    o.build(pats)
    s = o.scan(text)
    with ReferenceShards(binary, pats, text, shards) as ref:
        ref.prepare()
        ref.run(procs=3, dump_ff=True)
        assert ref.bloom == whole["bloom"]
        assert np.array_equal(ref.main, np.frombuffer(whole["dump"], np.uint8)[:nb])
        ff = ref.ff_or()
        assert np.array_equal(ff, np.frombuffer(whole["dump"], np.uint8)[nb:])
        assert ref.prune_with_ff(ff) == (whole["pruned"], whole["index"])
        hits, ls, le, off = oracle_scan_shards(wl.params, ref.main, text, shards, threads=3)
        np.testing.assert_array_equal(hits, s["hits"])
        np.testing.assert_array_equal(ls, s["line_start"])
        np.testing.assert_array_equal(le, s["line_end"])
        assert np.array_equal(off, o.ff)
        for i, (a, b) in enumerate(shards):
            # each shard's stdout is the restatement's for that shard's bytes on its own chunk grid
            so = oracle.Oracle.from_params(wl.params)
            so.main[:] = ref.main
            assert ref.stdout(i) == so.scan(text[a:b])["out"]
        if kind == "plain":  # no NUL bytes and short lines: the cut does not show in stdout
            assert b"".join(ref.stdout(i) for i in range(len(shards))) == whole["stdout"]
