"""Shared test setup: repository root on sys.path, the `gpu` marker, native builds, golden fixtures."""
import gzip
import hashlib
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")
    config.addinivalue_line("markers", "slow: large inputs; minutes of runtime")


@pytest.fixture(scope="session", autouse=True)
def native_build():
    """Builds libffbf.so, the CLI, the data generator and the oracle library if they are stale."""
    from ffbf_b200 import build as b
    b.build()
    import oracle
    oracle.build_lib()


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


class Golden:
    """Outputs of the reference binary for one case of tests/golden/cases.py."""

    def __init__(self, name):
        self.name = name
        self.dir = os.path.join(GOLDEN, name)
        with open(os.path.join(self.dir, "meta.json")) as f:
            self.meta = json.load(f)

    def has(self, what):
        return os.path.exists(os.path.join(self.dir, what + ".gz"))

    def read(self, what):
        with gzip.open(os.path.join(self.dir, what + ".gz"), "rb") as f:
            return f.read()

    def matches(self, what, data):
        """True when `data` equals the stored artefact (content or, for large ones, length + sha256)."""
        if self.has(what):
            return self.read(what) == data
        with open(os.path.join(self.dir, what + ".sha256")) as f:
            n, h = f.read().split()
        return len(data) == int(n) and hashlib.sha256(data).hexdigest() == h


def golden_cases():
    from cases import CASES
    return list(CASES)
