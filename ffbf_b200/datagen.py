"""Seeded synthetic workloads (ffbf_b200/csrc/datagen.c) and the filter geometry each is run with.

Workloads (one uint64 seed each; patterns, then text, then planted occurrences):
  plain       10,000 printable patterns of 20-40 bytes, LEN 20; 64 MiB printable text, '\\n' after
              geometric(mean 80) bytes; 500 planted occurrences. Geometry: the reference's defaults
              with LEN 20 (K 5, S 2, 2^24 cache bits, 2^28 external bits).
  scale       1,000,000 Zipf-letter "word" patterns of 32-64 bytes, LEN 32; 4 GiB text of the same
              letters, '\\n' every geometric(mean 100) bytes; 20,000 planted occurrences. Geometry:
              K 5, S 2, 2^23 cache bits (1 MiB), 2^26 external bits (8 MiB).
  binary      4,000,000 signatures of 16 uniform bytes ('\\n' redrawn), LEN 16; 8 GiB uniform text;
              100,000 planted. Geometry: the reference's defaults with LEN 16.
  batched     512 independent jobs. Per job: a pattern count log-uniform in [1k, 256k] (printable, 24-48
              bytes, LEN 24) and a text size log-uniform in [256 KiB, 256 MiB] (printable, '\\n' after
              geometric(mean 80) bytes), with planted occurrences at 0.01% of the text's windows. Geometry
              from a menu keyed on the pattern count: (2^20, 2^24) cache/external bits below 16k patterns,
              (2^22, 2^26) below 64k, (2^23, 2^27) otherwise; K 5, S 2.
Text sizes and plant counts scale together for the smaller parity cases (same densities).
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

from .lib import Params

_HERE = os.path.dirname(os.path.abspath(__file__))
GEN_PATH = os.path.join(_HERE, "_lib", "libffbf_datagen.so")

PRINTABLE, ZIPF_WORDS, BINARY = 0, 1, 2

_gen = None


def _lib():
    global _gen
    if _gen is None:
        if not os.path.exists(GEN_PATH):
            raise FileNotFoundError(f"{GEN_PATH} is missing: build it with `python -m ffbf_b200.build`")
        g = ctypes.CDLL(GEN_PATH)
        u64, u32, vp, sz = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_size_t
        g.ffbf_gen_patterns.restype = sz
        g.ffbf_gen_patterns.argtypes = [u64, ctypes.c_int, u64, u32, u32, vp]
        g.ffbf_gen_text.restype = ctypes.c_int
        g.ffbf_gen_text.argtypes = [u64, ctypes.c_int, u32, vp, sz, ctypes.c_int]
        g.ffbf_gen_plant.restype = ctypes.c_int
        g.ffbf_gen_plant.argtypes = [u64, vp, sz, vp, sz, u64, vp, vp]
        g.ffbf_gen_u64.restype = None
        g.ffbf_gen_u64.argtypes = [u64, u64, vp, sz]
        _gen = g
    return _gen


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def gen_patterns(seed, kind, n, len_lo, len_hi):
    out = np.empty(n * (len_hi + 1) + 1, dtype=np.uint8)
    m = _lib().ffbf_gen_patterns(seed, kind, n, len_lo, len_hi, _ptr(out))
    return out[:m]


def gen_text(seed, kind, nbytes, newline_mean, out=None, threads=None):
    """Fills `out` (a uint8 array of nbytes, e.g. pinned memory) or a new array."""
    if out is None:
        out = np.empty(nbytes, dtype=np.uint8)
    assert out.dtype == np.uint8 and out.size >= nbytes and out.flags.c_contiguous
    threads = threads or min(32, os.cpu_count() or 1)
    if _lib().ffbf_gen_text(seed, kind, newline_mean, _ptr(out), nbytes, threads) != 0:
        raise RuntimeError("text generation failed")
    return out


def plant(seed, patterns, text, n_plant, nbytes=None):
    nbytes = text.size if nbytes is None else nbytes
    offs = np.zeros(max(n_plant, 1), dtype=np.uint64)
    ids = np.zeros(max(n_plant, 1), dtype=np.uint64)
    if _lib().ffbf_gen_plant(seed, _ptr(patterns), patterns.size, _ptr(text), nbytes, n_plant, _ptr(offs), _ptr(ids)):
        raise RuntimeError("planting failed")
    return offs[:n_plant], ids[:n_plant]


def gen_u64(seed, stream, n):
    out = np.empty(n, dtype=np.uint64)
    _lib().ffbf_gen_u64(seed, stream, _ptr(out), n)
    return out


@dataclass
class Workload:
    name: str
    params: Params
    kind: int
    n_patterns: int
    len_lo: int
    len_hi: int
    newline_mean: int
    text_bytes: int
    n_plant: int

    def patterns(self, seed):
        return gen_patterns(seed, self.kind, self.n_patterns, self.len_lo, self.len_hi)

    def text(self, seed, patterns, out=None):
        t = gen_text(seed, self.kind, self.text_bytes, self.newline_mean, out=out)
        plant(seed, patterns, t, self.n_plant, nbytes=self.text_bytes)
        return t


MiB = 1 << 20
GiB = 1 << 30


def plain(text_bytes=64 * MiB, n_patterns=10_000):
    return Workload("plain", Params(20, 5, 2, 1 << 24, 1 << 28), PRINTABLE, n_patterns, 20, 40, 80, text_bytes,
                    max(1, round(500 * text_bytes / (64 * MiB))))


def scale(text_bytes=4 * GiB, n_patterns=1_000_000):
    return Workload("scale", Params(32, 5, 2, 1 << 23, 1 << 26), ZIPF_WORDS, n_patterns, 32, 64, 100, text_bytes,
                    max(1, round(20_000 * text_bytes / (4 * GiB))))


def binary(text_bytes=8 * GiB, n_patterns=4_000_000):
    return Workload("binary", Params(16, 5, 2, 1 << 24, 1 << 28), BINARY, n_patterns, 16, 16, 0, text_bytes,
                    max(1, round(100_000 * text_bytes / (8 * GiB))))


def batch_geometry(n_patterns):
    """The batched workload's geometry menu, keyed on the job's pattern count."""
    if n_patterns < 16_000:
        return Params(24, 5, 2, 1 << 20, 1 << 24)
    if n_patterns < 64_000:
        return Params(24, 5, 2, 1 << 22, 1 << 26)
    return Params(24, 5, 2, 1 << 23, 1 << 27)


def batched(n_jobs=512, pat_lo=1_000, pat_hi=256_000, text_lo=256 * 1024, text_hi=256 * MiB, seed=2024):
    """The batched workload's jobs: one Workload per job, each with its own seed (Workload.seed).

    Draws come from gen_u64 stream 3 of `seed`: per job one draw for its seed, one for the pattern count and
    one for the text size, both log-uniform over [lo, hi] (floor(lo * (hi/lo)^u), u = draw / 2^64).
    """
    d = gen_u64(seed, 3, 3 * n_jobs).reshape(n_jobs, 3)
    u_pat = d[:, 1].astype(np.float64) / 2.0**64
    u_txt = d[:, 2].astype(np.float64) / 2.0**64
    jobs = []
    for j in range(n_jobs):
        npat = int(pat_lo * (pat_hi / pat_lo) ** u_pat[j])
        nbytes = int(text_lo * (text_hi / text_lo) ** u_txt[j])
        n_windows = max(nbytes - 24 + 1, 0)
        w = Workload(f"batched[{j}]", batch_geometry(npat), PRINTABLE, npat, 24, 48, 80, nbytes,
                     max(1, round(1e-4 * n_windows)))
        w.seed = int(d[j, 0])
        jobs.append(w)
    return jobs
