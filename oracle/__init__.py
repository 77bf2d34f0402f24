"""TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

The oracle for efficient/ffbf's x86 rabin-karp path:
  * `Oracle` -- ctypes access to the C restatement in oracle/ffbf_oracle.c (built into oracle/_build/);
  * `run_reference` -- runs the reference's own ffbf binary (built from its sources by oracle/Makefile into
    oracle/_ref/) in a scratch directory and returns every file it writes.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this package, and only as the
checker or as the timed CPU baseline. Nothing in ffbf_b200/ imports it.
"""
import ctypes
import os
import re
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libffbf_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_ENV = "FFBF_REFERENCE"  # names a checkout of efficient/ffbf; needed only to (re)build oracle/_ref


def reference_source():
    """The efficient/ffbf checkout named by FFBF_REFERENCE, or None when it is unset or not a checkout."""
    src = os.environ.get(REF_ENV)
    if src and os.path.exists(os.path.join(src, "src", "rabin-karp", "ffbf.cpp")):
        return src
    return None


class OParams(ctypes.Structure):
    _fields_ = [("len", ctypes.c_int), ("k", ctypes.c_int), ("s", ctypes.c_int),
                ("cache_bits", ctypes.c_uint64), ("ext_bits", ctypes.c_uint64)]


class _Scan(ctypes.Structure):
    _fields_ = [("out", ctypes.c_void_p), ("out_len", ctypes.c_size_t), ("hits", ctypes.c_void_p),
                ("n_hits", ctypes.c_size_t), ("line_start", ctypes.c_void_p), ("line_end", ctypes.c_void_p),
                ("n_lines", ctypes.c_size_t)]


class _Prune(ctypes.Structure):
    _fields_ = [("out", ctypes.c_void_p), ("out_len", ctypes.c_size_t), ("idx", ctypes.c_void_p),
                ("idx_len", ctypes.c_size_t), ("ids", ctypes.c_void_p), ("n_ids", ctypes.c_size_t)]


class _Matches(ctypes.Structure):
    _fields_ = [("off", ctypes.c_void_p), ("pid", ctypes.c_void_p), ("n", ctypes.c_size_t)]


def build_lib():
    subprocess.run(["make", "-s", "-C", HERE, "lib"], check=True)


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build_lib()
        lib = ctypes.CDLL(LIB)
        vp, sz, P = ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER
        lib.orc_window_hash.restype = ctypes.c_uint64
        lib.orc_window_hash.argtypes = [vp, ctypes.c_int]
        lib.orc_index.restype = ctypes.c_uint32
        lib.orc_index.argtypes = [P(OParams), ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        lib.orc_build.restype = ctypes.c_long
        lib.orc_build.argtypes = [P(OParams), vp, sz, vp]
        lib.orc_scan.restype = ctypes.c_int
        lib.orc_scan.argtypes = [P(OParams), vp, vp, vp, sz, sz, P(_Scan)]
        lib.orc_prune.restype = ctypes.c_int
        lib.orc_prune.argtypes = [P(OParams), vp, vp, sz, sz, P(_Prune)]
        lib.orc_test_line.restype = ctypes.c_int
        lib.orc_test_line.argtypes = [P(OParams), vp, vp, sz]
        lib.orc_save_filter.restype = ctypes.c_int
        lib.orc_save_filter.argtypes = [P(OParams), vp, P(vp), P(sz)]
        lib.orc_load_filter.restype = ctypes.c_int
        lib.orc_load_filter.argtypes = [P(OParams), vp, sz, vp]
        lib.orc_verify.restype = ctypes.c_int
        lib.orc_verify.argtypes = [P(OParams), vp, sz, vp, sz, vp, sz, vp, sz, P(_Matches)]
        lib.orc_hashbench_lines.restype = ctypes.c_long
        lib.orc_hashbench_lines.argtypes = [vp, sz, P(vp)]
        lib.orc_hash_xor.restype = ctypes.c_uint64
        lib.orc_hash_xor.argtypes = [vp, sz, ctypes.c_int]
        lib.orc_free.restype = None
        lib.orc_free.argtypes = [vp]
        _lib = lib
    return _lib


def _np(data):
    a = np.ascontiguousarray(np.frombuffer(data, dtype=np.uint8) if isinstance(data, (bytes, bytearray)) else data,
                             dtype=np.uint8)
    return a


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _take(lib, ptr, n, dtype):
    if not n:
        if ptr:
            lib.orc_free(ptr)
        return np.zeros(0, dtype=dtype)
    a = np.frombuffer(ctypes.string_at(ptr, n * np.dtype(dtype).itemsize), dtype=dtype).copy()
    lib.orc_free(ptr)
    return a


class Oracle:
    """The C restatement for one geometry (len, k, s, cache_bits, ext_bits)."""

    def __init__(self, len=19, k=5, s=2, cache_bits=1 << 24, ext_bits=1 << 28):
        self.lib = _load()
        self.p = OParams(len, k, s, cache_bits, ext_bits)
        self.nbytes = (cache_bits + ext_bits) // 8
        self.main = np.zeros(self.nbytes, dtype=np.uint8)
        self.ff = np.zeros(self.nbytes, dtype=np.uint8)

    @classmethod
    def from_params(cls, prm):
        return cls(prm.len, prm.k, prm.s, prm.cache_bits, prm.ext_bits)

    def window_hash(self, window):
        w = _np(window)
        return int(self.lib.orc_window_hash(_p(w), self.p.len))

    def index(self, h, i, order):
        return int(self.lib.orc_index(ctypes.byref(self.p), h, i, order))

    def build(self, patterns):
        pa = _np(patterns)
        return int(self.lib.orc_build(ctypes.byref(self.p), _p(pa), pa.size, _p(self.main)))

    def scan(self, text, chunk=512 * 1024):
        """processFile: returns dict(out=stdout bytes, hits, line_start, line_end); updates self.ff."""
        t = _np(text)
        r = _Scan()
        if self.lib.orc_scan(ctypes.byref(self.p), _p(self.main), _p(self.ff), _p(t), t.size, chunk, ctypes.byref(r)):
            raise MemoryError("oracle scan failed")
        out = _take(self.lib, r.out, r.out_len, np.uint8).tobytes()
        return dict(out=out, hits=_take(self.lib, r.hits, r.n_hits, np.uint64),
                    line_start=_take(self.lib, r.line_start, r.n_lines, np.uint64),
                    line_end=_take(self.lib, r.line_end, r.n_lines, np.uint64))

    def prune(self, patterns, chunk=512 * 1024):
        """filterPhrases: returns dict(out=pruned file, index=__index_ file, ids)."""
        pa = _np(patterns)
        r = _Prune()
        if self.lib.orc_prune(ctypes.byref(self.p), _p(self.ff), _p(pa), pa.size, chunk, ctypes.byref(r)):
            raise MemoryError("oracle prune failed")
        return dict(out=_take(self.lib, r.out, r.out_len, np.uint8).tobytes(),
                    index=_take(self.lib, r.idx, r.idx_len, np.uint8).tobytes(),
                    ids=_take(self.lib, r.ids, r.n_ids, np.uint64))

    def test_line(self, line):
        la = _np(line)
        return bool(self.lib.orc_test_line(ctypes.byref(self.p), _p(self.main), _p(la), la.size))

    def save_filter(self):
        out, n = ctypes.c_void_p(), ctypes.c_size_t()
        if self.lib.orc_save_filter(ctypes.byref(self.p), _p(self.main), ctypes.byref(out), ctypes.byref(n)):
            raise MemoryError("oracle save failed")
        return _take(self.lib, out.value, n.value, np.uint8).tobytes()

    def load_filter(self, data):
        d = _np(data)
        return self.lib.orc_load_filter(ctypes.byref(self.p), _p(d), d.size, _p(self.main)) == 0

    def verify(self, patterns, ids, text, hits):
        pa, t = _np(patterns), _np(text)
        ids = np.ascontiguousarray(ids, dtype=np.uint64)
        hits = np.ascontiguousarray(hits, dtype=np.uint64)
        m = _Matches()
        if self.lib.orc_verify(ctypes.byref(self.p), _p(pa), pa.size, _p(ids), ids.size, _p(t), t.size, _p(hits),
                               hits.size, ctypes.byref(m)):
            raise MemoryError("oracle verify failed")
        n = m.n
        return _take(self.lib, m.off, n, np.uint64), _take(self.lib, m.pid, n, np.uint64)


# ---- the reference binary ------------------------------------------------------------------------
def ref_name(prm):
    return f"ffbf_ref_L{prm.len}_K{prm.k}_S{prm.s}_C{prm.cache_bits:#x}_E{prm.ext_bits:#x}"


def ref_binary(prm, ref_src=None, build=True):
    """Path of the reference binary for this geometry. A missing (or, with sources at hand, stale) binary is
    built when `build` is set and the reference sources are given (`ref_src` or FFBF_REFERENCE)."""
    path = os.path.join(REF_DIR, ref_name(prm))
    src = ref_src or reference_source()
    if not build or src is None:
        return path if os.path.exists(path) else None
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={src}", f"LEN={prm.len}", f"K={prm.k}", f"S={prm.s}",
                    f"CACHE={prm.cache_bits:#x}", f"EXT={prm.ext_bits:#x}"], check=True)
    return path


def run_reference(binary, patterns, text_path=None, text=None, dump_ff=True, workdir=None, filter_cache=None):
    """Runs `ffbf pats out < text` in a scratch directory (regular-file stdin, as the reference expects).

    Returns dict(stdout, pruned, index, bloom (the __bloom_filter_ file, or None when it was loaded from
    `filter_cache`), dump (main+FF arrays when dump_ff), times {label: seconds}, wall).
    """
    own = workdir is None
    wd = workdir or tempfile.mkdtemp(prefix="ffbf_ref_")
    try:
        with open(os.path.join(wd, "pats"), "wb") as f:
            f.write(bytes(patterns))
        if text_path is None:
            text_path = os.path.join(wd, "text")
            with open(text_path, "wb") as f:
                f.write(bytes(text))
        if filter_cache is not None:
            with open(os.path.join(wd, "__bloom_filter_pats"), "wb") as f:
                f.write(filter_cache)
        env = dict(os.environ)
        if dump_ff:
            env["FFBF_REF_DUMP"] = os.path.join(wd, "dump.bin")
        t0 = time.time()
        with open(text_path, "rb") as fin, open(os.path.join(wd, "stdout"), "wb") as fout:
            r = subprocess.run([binary, "pats", "out"], stdin=fin, stdout=fout, stderr=subprocess.PIPE, cwd=wd,
                               env=env)
        wall = time.time() - t0
        err = r.stderr.decode(errors="replace")
        if r.returncode != 0:
            raise RuntimeError(f"reference exited {r.returncode}: {err}")
        times = {m.group(1): float(m.group(2)) for m in re.finditer(r"^(.*) time: ([0-9.]+)$", err, re.M)}

        def rd(name):
            p = os.path.join(wd, name)
            return open(p, "rb").read() if os.path.exists(p) else None

        res = dict(stdout=rd("stdout"), pruned=rd("out"), index=rd("__index_out"),
                   bloom=None if filter_cache is not None else rd("__bloom_filter_pats"),
                   dump=rd("dump.bin") if dump_ff else None, times=times, wall=wall, stderr=err)
        return res
    finally:
        if own:
            for fn in os.listdir(wd):
                os.unlink(os.path.join(wd, fn))
            os.rmdir(wd)


def set_bits(bitarray_bytes):
    """Ascending indices of the set bits of a bit array in the reference's byte layout."""
    a = np.frombuffer(bitarray_bytes, dtype=np.uint8) if isinstance(bitarray_bytes, (bytes, bytearray)) else bitarray_bytes
    bits = np.unpackbits(a, bitorder="little")
    return np.flatnonzero(bits).astype(np.uint64)


def decode_filter_file(data):
    """Set-bit indices stored in a __bloom_filter_ image (cumulative uint32 deltas)."""
    d = np.frombuffer(data[: len(data) // 4 * 4], dtype="<u4").astype(np.uint64)
    return (np.cumsum(d) & 0xFFFFFFFF).astype(np.uint64)


def hashbench_lines(text):
    """What `hashbench -l` prints for `text` (hash_rot_sbox_pre_2<19>, hashbench.cc:108-127)."""
    lib = _load()
    t = _np(text)
    out = ctypes.c_void_p()
    n = lib.orc_hashbench_lines(_p(t), t.size, ctypes.byref(out))
    if n < 0:
        raise MemoryError("oracle hashbench failed")
    return _take(lib, out.value, n, np.uint8).tobytes()


def hash_xor(text, length=19):
    """XOR of the rolling hash after every byte of `text` (no resets): the checkable result of hashbench -f."""
    t = _np(text)
    return int(_load().orc_hash_xor(_p(t), t.size, length))
