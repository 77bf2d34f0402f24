"""GPU hash benchmark (ffbf_hashbench_*, the `hashbench` CLI) against the reference's own hashbench output
(tests/golden/hashbench) and the oracle's rolling hash."""
import gzip
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT
from ffbf_b200.lib import hashbench_file, hashbench_lines

pytestmark = pytest.mark.gpu

GOLD = os.path.join(ROOT, "tests", "golden", "hashbench")
CLI = os.path.join(ROOT, "ffbf_b200", "_lib", "hashbench")


def golden():
    return gzip.open(os.path.join(GOLD, "input.bin.gz")).read(), gzip.open(os.path.join(GOLD, "lines.out.gz")).read()


def test_hash_lines_equal_reference_output():
    text, want = golden()
    assert hashbench_lines(text) == want
    assert hashbench_lines(b"") == b""


def test_cli_lines_and_file_modes(tmp_path):
    text, want = golden()
    p = tmp_path / "input.bin"
    p.write_bytes(text)
    r = subprocess.run([CLI, "-l", str(p)], capture_output=True, check=True)
    assert r.stdout == want
    r = subprocess.run([CLI, "-f", str(p)], capture_output=True, check=True, text=True)
    lines = r.stdout.splitlines()
    assert lines[0].startswith("# hashbench.c ") and lines[1] == "# hashfn: hash_rot_sbox_pre_2"
    assert lines[-2] == "# bytes     execution time (seconds)"
    assert int(lines[-1].split()[0]) == len(text)


@pytest.mark.parametrize("size", [0, 1, 18, 19, 20, 16383, 16384, 16403, 64 << 20])
def test_hash_file_xor_equals_oracle(size):
    rng = np.random.default_rng(size)
    text = rng.integers(0, 256, size, dtype=np.uint8)
    x, secs = hashbench_file(text)
    assert x == oracle.hash_xor(text)
    assert secs >= 0
