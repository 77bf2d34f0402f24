"""The oracle (oracle/ffbf_oracle.c) against the reference binary's outputs stored in tests/golden/.

This pins the C restatement to efficient/ffbf's own x86 build: every artefact the reference writes
(__bloom_filter_ file, stdout, pruned patterns, __index_ file) and its feed-forward bit array must match
byte for byte on every case, including the edge cases of tests/golden/cases.py.
"""
import os

import numpy as np
import pytest

import oracle
from cases import CASES, build_inputs, digest
from conftest import Golden


def delta(bits):
    return np.diff(np.concatenate([[0], np.asarray(bits, dtype=np.uint64)])).astype("<u4").tobytes()


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_reference(name):
    g = Golden(name)
    prm, pats, text = build_inputs(name)
    assert digest(pats, text) == g.meta["input_sha256"], "generator output drifted from the fixture"
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    assert g.matches("bloom", o.save_filter())
    s = o.scan(text)
    assert g.matches("stdout", s["out"])
    assert g.matches("ff", delta(oracle.set_bits(o.ff)))
    pr = o.prune(pats)
    assert g.matches("pruned", pr["out"])
    assert g.matches("index", pr["index"])
    # internal consistency of the restatement's extra outputs
    assert np.all(np.diff(s["hits"].astype(np.int64)) > 0)
    assert s["line_start"].size == len([1 for _ in s["line_start"]])
    if s["hits"].size:
        assert s["line_start"].size >= 1


@pytest.mark.parametrize("name", ["plain_small", "edge_mixed", "dense_fp"])
def test_oracle_filter_file_roundtrip(name):
    prm, pats, _ = build_inputs(name)
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    data = o.save_filter()
    o2 = oracle.Oracle.from_params(prm)
    assert o2.load_filter(data)
    assert np.array_equal(o.main, o2.main)
    assert np.array_equal(oracle.decode_filter_file(data), oracle.set_bits(o.main))


def test_oracle_verify_finds_planted():
    from ffbf_b200 import datagen as dg
    prm, pats, text = build_inputs("plain_small")
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    s = o.scan(text)
    pr = o.prune(pats)
    off, pid = o.verify(pats, pr["ids"], text, s["hits"])
    # every planted occurrence that survived later plants is found
    offs, ids = dg.plant(7, np.frombuffer(pats, np.uint8), np.zeros(text.size, np.uint8), 100)
    lines = pats.split(b"\n")
    found = set(zip(off.tolist(), pid.tolist()))
    for o_, i_ in zip(offs.tolist(), ids.tolist()):
        p = lines[i_]
        if bytes(text[o_:o_ + len(p)]) == p:
            assert (o_, i_) in found


def test_oracle_test_line_semantics():
    prm, pats, text = build_inputs("plain_small")
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    first = pats.split(b"\n")[0]
    assert o.test_line(b"xx" + first + b"yy")
    assert not o.test_line(first[: prm.len - 1])
    # operator[] hashes '\n' like any other byte, so a pattern split by a newline does not hit
    assert not o.test_line(first[:5] + b"\n" + first[5:])


@pytest.mark.parametrize("name", ["edge_mixed", "pats_no_newline"])
def test_fixtures_are_current(name):
    """Re-runs the reference binary and compares with the stored fixture (catches stale goldens)."""
    g = Golden(name)
    prm, pats, text = build_inputs(name)
    binary = oracle.ref_binary(prm)
    if binary is None:
        pytest.skip("reference binary for this geometry not built (oracle/_ref)")
    r = oracle.run_reference(binary, pats, text=text.tobytes())
    assert g.matches("stdout", r["stdout"]) and g.matches("bloom", r["bloom"])
    assert g.matches("pruned", r["pruned"]) and g.matches("index", r["index"])


def test_hashbench_restatement_matches_reference_output():
    """oracle.hashbench_lines reproduces `hashbench -l` (the reference's own binary, tests/golden/hashbench)
    byte for byte: fgets pieces of at most 4094 bytes, hashing stopped at a NUL, raw bytes >= 0x80."""
    import gzip
    import os

    import oracle

    d = os.path.join(os.path.dirname(__file__), "golden", "hashbench")
    text = gzip.open(os.path.join(d, "input.bin.gz")).read()
    want = gzip.open(os.path.join(d, "lines.out.gz")).read()
    assert oracle.hashbench_lines(text) == want


def test_hash_xor_restatement_is_the_rolling_hash():
    """oracle.hash_xor follows hash_rot_sbox_pre_2::update byte by byte (checked against the window closed
    form on random bytes)."""
    import numpy as np

    import oracle

    import os
    import re

    hdr = open(os.path.join(os.path.dirname(os.path.dirname(__file__)), "ffbf_b200", "csrc", "ffbf_sbox.h")).read()
    sbox = [int(w, 16) for w in re.findall(r"0x([0-9a-fA-F]+)ull", hdr)]
    assert len(sbox) == 256
    rng = np.random.default_rng(5)
    t = rng.integers(0, 256, 3000, dtype=np.uint8)

    def rol(w, s):
        s %= 64
        return ((w << s) | (w >> (64 - s))) & 0xFFFFFFFFFFFFFFFF if s else w

    acc = 0
    for i in range(t.size):
        h = 0
        for j in range(max(0, i - 18), i + 1):
            h ^= rol(int(sbox[t[j]]), i - j)
        acc ^= h
    assert oracle.hash_xor(t) == acc
