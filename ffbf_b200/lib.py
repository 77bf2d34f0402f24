"""Python access to the C ABI in include/ffbf.h (ffbf_b200/_lib/libffbf.so).

`Filter` mirrors efficient/ffbf's Filter<H, LEN> (src/rabin-karp/ffbf.h:43-93) member for member:

    reference (C++)                         here
    filter << phrase  (per getline line)    Filter.add_patterns(file_bytes)
    filter[line]                            Filter.test_line(line)
    processFile(fd)                         Filter.process(text) / Filter.process_device(ptr, n)
    filterPhrases(pfd, out, outIndex)       Filter.filter_phrases() + Filter.format_pruned()
    loadFilterFromFile(fd)                  Filter.load_filter(data) / load_filter_from_file(path)
    saveFilterToFile(fd)                    Filter.save_filter() / save_filter_to_file(path)

Failures raise FFBFError (the reference throws FilterError, ffbf.h:31-41) carrying the C status and
ffbf_last_error(). There is no fallback: if the native library is missing this module raises on load.
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libffbf.so")

# processFile and filterPhrases read() 512 KiB at a time (src/rabin-karp/ffbf.cpp:313,397); a regular
# file returns full chunks, which is what the output rules depend on.
DEFAULT_CHUNK = 512 * 1024

STATUS = {0: "FFBF_OK", 1: "FFBF_EINVAL", 2: "FFBF_ENOMEM_DEVICE", 3: "FFBF_EIO", 4: "FFBF_ETIMEOUT",
          5: "FFBF_ECUDA", 6: "FFBF_ESTATE", 7: "FFBF_ENOMEM_HOST"}

EXPORTED = [
    "ffbf_params_default", "ffbf_create", "ffbf_destroy", "ffbf_last_error", "ffbf_status_string",
    "ffbf_set_hbm_budget", "ffbf_set_patterns", "ffbf_build", "ffbf_add_patterns", "ffbf_load_filter",
    "ffbf_save_filter", "ffbf_load_filter_file", "ffbf_save_filter_file", "ffbf_scan", "ffbf_scan_device",
    "ffbf_scan_collect", "ffbf_format_lines", "ffbf_prune", "ffbf_format_pruned", "ffbf_verify",
    "ffbf_test_line", "ffbf_clear_ff", "ffbf_get_filters", "ffbf_filter_bytes", "ffbf_free", "ffbf_format_spans",
    "ffbf_stream", "ffbf_kernel_launches", "ffbf_scan_static", "ffbf_batch_create", "ffbf_batch_add",
    "ffbf_batch_prepare", "ffbf_batch_launch", "ffbf_batch_wait", "ffbf_batch_stream", "ffbf_batch_last_error",
    "ffbf_batch_destroy", "ffbf_batch_autotune", "ffbf_autotune", "ffbf_get_scan_config", "ffbf_get_probe_order", "ffbf_debug_scan_unpublished", "ffbf_hashbench_lines", "ffbf_hashbench_file", "ffbf_host_alloc", "ffbf_host_free", "ffbf_server_create", "ffbf_server_add_set", "ffbf_server_submit",
    "ffbf_server_poll", "ffbf_server_release", "ffbf_server_get_stats", "ffbf_server_last_error",
    "ffbf_server_destroy",
]


class FFBFError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Params(ctypes.Structure):
    """ffbf_params: len=DEF_PATT_LEN, k=DEF_K, s=DEF_S, cache_bits=DEF_CACHE_SIZE, ext_bits=DEF_EXT_SIZE."""
    _fields_ = [("len", ctypes.c_uint32), ("k", ctypes.c_uint32), ("s", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("cache_bits", ctypes.c_uint64), ("ext_bits", ctypes.c_uint64)]

    def __init__(self, len=19, k=5, s=2, cache_bits=1 << 24, ext_bits=1 << 28):
        super().__init__(len, k, s, 0, cache_bits, ext_bits)

    @property
    def nbits(self):
        return self.cache_bits + self.ext_bits

    def as_tuple(self):
        return (self.len, self.k, self.s, self.cache_bits, self.ext_bits)

    def __repr__(self):
        return f"Params(len={self.len}, k={self.k}, s={self.s}, cache_bits={self.cache_bits:#x}, ext_bits={self.ext_bits:#x})"


class _RequestResult(ctypes.Structure):
    _fields_ = [("request_id", ctypes.c_uint64), ("set_id", ctypes.c_uint32), ("status", ctypes.c_int),
                ("text_len", ctypes.c_uint64), ("n_hits", ctypes.c_uint64),
                ("hit_offsets", ctypes.POINTER(ctypes.c_uint64)), ("n_lines", ctypes.c_uint64),
                ("line_start", ctypes.POINTER(ctypes.c_uint64)), ("line_end", ctypes.POINTER(ctypes.c_uint64)),
                ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_launch", ctypes.c_double),
                ("t_done", ctypes.c_double)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("requests_done", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("bytes_scanned", ctypes.c_uint64),
                ("max_batch", ctypes.c_uint64), ("arena_bytes", ctypes.c_uint64), ("slots", ctypes.c_uint32)]


class _ScanResult(ctypes.Structure):
    _fields_ = [("text_len", ctypes.c_uint64), ("n_hits", ctypes.c_uint64),
                ("hit_offsets", ctypes.POINTER(ctypes.c_uint64)), ("n_lines", ctypes.c_uint64),
                ("line_start", ctypes.POINTER(ctypes.c_uint64)), ("line_end", ctypes.POINTER(ctypes.c_uint64))]


class _PruneResult(ctypes.Structure):
    _fields_ = [("n_ids", ctypes.c_uint64), ("ids", ctypes.POINTER(ctypes.c_uint64))]


class _Matches(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("offsets", ctypes.POINTER(ctypes.c_uint64)),
                ("pattern_ids", ctypes.POINTER(ctypes.c_uint64))]


_lib = None


def load_library(path=LIB_PATH):
    """Loads libffbf.so once. Raises FileNotFoundError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -m ffbf_b200.build`")
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    u8p, vp, sz = P(ctypes.c_uint8), ctypes.c_void_p, ctypes.c_size_t
    sig = {
        "ffbf_params_default": (ctypes.c_int, [P(Params)]),
        "ffbf_create": (ctypes.c_int, [P(Params), ctypes.c_int, P(vp)]),
        "ffbf_destroy": (None, [vp]),
        "ffbf_last_error": (ctypes.c_char_p, [vp]),
        "ffbf_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "ffbf_set_hbm_budget": (ctypes.c_int, [vp, ctypes.c_uint64]),
        "ffbf_set_patterns": (ctypes.c_int, [vp, vp, sz]),
        "ffbf_build": (ctypes.c_int, [vp]),
        "ffbf_add_patterns": (ctypes.c_int, [vp, vp, sz]),
        "ffbf_load_filter": (ctypes.c_int, [vp, vp, sz]),
        "ffbf_save_filter": (ctypes.c_int, [vp, P(u8p), P(sz)]),
        "ffbf_load_filter_file": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "ffbf_save_filter_file": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "ffbf_scan": (ctypes.c_int, [vp, vp, sz, P(_ScanResult)]),
        "ffbf_scan_device": (ctypes.c_int, [vp, vp, sz]),
        "ffbf_scan_collect": (ctypes.c_int, [vp, P(_ScanResult)]),
        "ffbf_format_lines": (ctypes.c_int, [vp, vp, sz, sz, P(u8p), P(sz)]),
        "ffbf_prune": (ctypes.c_int, [vp, P(_PruneResult)]),
        "ffbf_format_pruned": (ctypes.c_int, [vp, sz, P(u8p), P(sz), P(u8p), P(sz)]),
        "ffbf_verify": (ctypes.c_int, [vp, P(_Matches)]),
        "ffbf_test_line": (ctypes.c_int, [vp, vp, sz, P(ctypes.c_int)]),
        "ffbf_clear_ff": (ctypes.c_int, [vp]),
        "ffbf_get_filters": (ctypes.c_int, [vp, vp, vp]),
        "ffbf_filter_bytes": (ctypes.c_uint64, [vp]),
        "ffbf_free": (None, [vp]),
        "ffbf_format_spans": (ctypes.c_int, [vp, sz, vp, vp, sz, sz, P(u8p), P(sz)]),
        "ffbf_stream": (vp, [vp]),
        "ffbf_kernel_launches": (ctypes.c_uint64, []),
        "ffbf_scan_static": (ctypes.c_int, [P(Params), vp, vp, vp, ctypes.c_uint64, vp, vp, vp,
                                            P(ctypes.c_uint32), vp]),
        "ffbf_batch_create": (ctypes.c_int, [ctypes.c_int, P(vp)]),
        "ffbf_batch_add": (ctypes.c_int, [vp, vp, vp, sz]),
        "ffbf_batch_prepare": (ctypes.c_int, [vp]),
        "ffbf_batch_launch": (ctypes.c_int, [vp]),
        "ffbf_batch_wait": (ctypes.c_int, [vp]),
        "ffbf_batch_stream": (vp, [vp]),
        "ffbf_batch_last_error": (ctypes.c_char_p, [vp]),
        "ffbf_batch_destroy": (None, [vp]),
        "ffbf_batch_autotune": (ctypes.c_int, [vp, sz, P(ctypes.c_uint32)]),
        "ffbf_get_scan_config": (ctypes.c_int, [vp, P(ctypes.c_int), P(ctypes.c_int)]),
        "ffbf_get_probe_order": (ctypes.c_int, [vp, P(ctypes.c_int)]),
        "ffbf_debug_scan_unpublished": (ctypes.c_int, [vp, vp, sz, ctypes.c_uint32]),
        "ffbf_hashbench_lines": (ctypes.c_int, [ctypes.c_int, vp, sz, P(u8p), P(sz)]),
        "ffbf_host_alloc": (vp, [sz]),
        "ffbf_host_free": (None, [vp]),
        "ffbf_hashbench_file": (ctypes.c_int, [ctypes.c_int, vp, sz, P(ctypes.c_uint64), P(ctypes.c_double)]),
        "ffbf_autotune": (ctypes.c_int, [vp, vp, sz, P(ctypes.c_int), P(ctypes.c_int)]),
        "ffbf_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32, P(vp)]),
        "ffbf_server_add_set": (ctypes.c_int, [vp, vp, P(ctypes.c_uint32)]),
        "ffbf_server_submit": (ctypes.c_int, [vp, ctypes.c_uint32, vp, sz, P(ctypes.c_uint64)]),
        "ffbf_server_poll": (ctypes.c_int, [vp, P(_RequestResult), ctypes.c_uint32, P(ctypes.c_uint32),
                                            ctypes.c_uint32]),
        "ffbf_server_release": (ctypes.c_int, [vp, ctypes.c_uint64]),
        "ffbf_server_get_stats": (ctypes.c_int, [vp, P(_ServerStats)]),
        "ffbf_server_last_error": (ctypes.c_char_p, [vp]),
        "ffbf_server_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _buf(data):
    """(pointer, length, keepalive) for bytes / bytearray / numpy uint8 data without copying numpy."""
    if isinstance(data, np.ndarray):
        a = np.ascontiguousarray(data, dtype=np.uint8)
        return a.ctypes.data_as(ctypes.c_void_p), a.nbytes, a
    if isinstance(data, (bytes, bytearray, memoryview)):
        a = np.frombuffer(bytes(data) if isinstance(data, memoryview) else data, dtype=np.uint8)
        return (a.ctypes.data_as(ctypes.c_void_p) if a.size else None), a.size, a
    raise TypeError(f"expected bytes or a uint8 array, got {type(data).__name__}")


def _arr(ptr, n):
    if n == 0:
        return np.zeros(0, dtype=np.uint64)
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def _take_bytes(lib, p, n):
    try:
        return ctypes.string_at(p, n.value) if n.value else b""
    finally:
        lib.ffbf_free(ctypes.cast(p, ctypes.c_void_p))


def kernel_launches():
    """Kernels the library has launched in this process so far."""
    return int(load_library().ffbf_kernel_launches())


def format_spans(buf, starts, ends, chunk=DEFAULT_CHUNK):
    """ffbf_format_spans: the reference's stdout bytes for the given flagged line spans of `buf` (host only)."""
    lib = load_library()
    p, n, keep = _buf(buf)
    st = np.ascontiguousarray(starts, dtype=np.uint64)
    en = np.ascontiguousarray(ends, dtype=np.uint64)
    out, m = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
    rc = lib.ffbf_format_spans(p, n, st.ctypes.data_as(ctypes.c_void_p), en.ctypes.data_as(ctypes.c_void_p), st.size,
                               chunk, ctypes.byref(out), ctypes.byref(m))
    if rc != 0:
        raise FFBFError(rc, "ffbf_format_spans rejected its arguments")
    return _take_bytes(lib, out, m)


@dataclass
class ScanOutput:
    text_len: int
    hit_offsets: np.ndarray  # uint64, ascending window start offsets
    line_start: np.ndarray   # uint64, flagged lines in text order
    line_end: np.ndarray     # uint64, exclusive, excludes the '\n'


class Filter:
    """One device-resident pair of bit arrays (main + feed-forward) with the reference's operations."""

    def __init__(self, params=None, device=0):
        self._lib = load_library()
        self.params = params if params is not None else Params()
        h = ctypes.c_void_p()
        st = self._lib.ffbf_create(ctypes.byref(self.params), device, ctypes.byref(h))
        if st != 0:
            raise FFBFError(st, "ffbf_create failed (bad geometry or no usable CUDA device)")
        self._h = h

    # -- plumbing -----------------------------------------------------------------------------
    def _check(self, st):
        if st != 0:
            raise FFBFError(st, self._lib.ffbf_last_error(self._h).decode(errors="replace"))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ffbf_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def filter_bytes(self):
        return int(self._lib.ffbf_filter_bytes(self._h))

    @property
    def stream(self):
        """The context's cudaStream_t as an integer handle (e.g. for torch.cuda.ExternalStream)."""
        return int(self._lib.ffbf_stream(self._h) or 0)

    def set_hbm_budget(self, nbytes):
        self._check(self._lib.ffbf_set_hbm_budget(self._h, nbytes))

    # -- build ---------------------------------------------------------------------------------
    def set_patterns(self, file_bytes):
        p, n, keep = _buf(file_bytes)
        self._check(self._lib.ffbf_set_patterns(self._h, p, n))

    def build(self):
        self._check(self._lib.ffbf_build(self._h))

    def add_patterns(self, file_bytes):
        """main()'s getline loop of `filter << phrase` (ffbf.cpp:556-571)."""
        p, n, keep = _buf(file_bytes)
        self._check(self._lib.ffbf_add_patterns(self._h, p, n))

    def load_filter(self, data):
        p, n, keep = _buf(data)
        self._check(self._lib.ffbf_load_filter(self._h, p, n))

    def save_filter(self):
        out, n = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
        self._check(self._lib.ffbf_save_filter(self._h, ctypes.byref(out), ctypes.byref(n)))
        return _take_bytes(self._lib, out, n)

    def load_filter_from_file(self, path):
        self._check(self._lib.ffbf_load_filter_file(self._h, os.fsencode(path)))

    def save_filter_to_file(self, path):
        self._check(self._lib.ffbf_save_filter_file(self._h, os.fsencode(path)))

    # -- scan ----------------------------------------------------------------------------------
    def _result(self, r):
        return ScanOutput(int(r.text_len), _arr(r.hit_offsets, r.n_hits), _arr(r.line_start, r.n_lines),
                          _arr(r.line_end, r.n_lines))

    def process(self, text):
        """processFile over a host text image."""
        p, n, keep = _buf(text)
        r = _ScanResult()
        self._check(self._lib.ffbf_scan(self._h, p, n, ctypes.byref(r)))
        return self._result(r)

    def process_device(self, dev_ptr, n):
        """Enqueues the scan of n bytes already on the device (16-byte aligned pointer)."""
        self._check(self._lib.ffbf_scan_device(self._h, ctypes.c_void_p(dev_ptr), n))

    def collect(self):
        r = _ScanResult()
        self._check(self._lib.ffbf_scan_collect(self._h, ctypes.byref(r)))
        return self._result(r)

    def format_lines(self, text, chunk=DEFAULT_CHUNK):
        """The bytes processFile writes to stdout for the last scan."""
        p, n, keep = _buf(text)
        out, m = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
        self._check(self._lib.ffbf_format_lines(self._h, p, n, chunk, ctypes.byref(out), ctypes.byref(m)))
        return _take_bytes(self._lib, out, m)

    # -- feed-forward prune and verification ---------------------------------------------------
    def filter_phrases(self):
        """Ascending 0-based line numbers of the patterns that pass the feed-forward filter."""
        r = _PruneResult()
        self._check(self._lib.ffbf_prune(self._h, ctypes.byref(r)))
        return _arr(r.ids, r.n_ids)

    def format_pruned(self, chunk=DEFAULT_CHUNK):
        """(pruned pattern file, __index_ file) bytes for the last filter_phrases()."""
        o, on = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
        i, inn = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
        self._check(self._lib.ffbf_format_pruned(self._h, chunk, ctypes.byref(o), ctypes.byref(on), ctypes.byref(i),
                                                 ctypes.byref(inn)))
        return _take_bytes(self._lib, o, on), _take_bytes(self._lib, i, inn)

    def verify(self):
        """Exact (offset, pattern id) pairs, sorted."""
        m = _Matches()
        self._check(self._lib.ffbf_verify(self._h, ctypes.byref(m)))
        return _arr(m.offsets, m.n), _arr(m.pattern_ids, m.n)

    def test_line(self, line):
        """operator[] (ffbf.cpp:285-308)."""
        p, n, keep = _buf(line)
        hit = ctypes.c_int()
        self._check(self._lib.ffbf_test_line(self._h, p, n, ctypes.byref(hit)))
        return bool(hit.value)

    def autotune(self, dev_ptr, n):
        """Times the tuned scan's configurations on n device bytes; keeps the fastest. Returns (threads, mode)."""
        t, m = ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.ffbf_autotune(self._h, ctypes.c_void_p(dev_ptr), n, ctypes.byref(t), ctypes.byref(m)))
        return t.value, m.value

    def debug_scan_unpublished(self, dev_ptr, n, spins=2000):
        """Failure-detection check: a scan gated on a word that is never published; raises FFBFError with
        FFBF_ETIMEOUT (4) after `spins` polls of about a microsecond."""
        self._check(self._lib.ffbf_debug_scan_unpublished(self._h, ctypes.c_void_p(dev_ptr), n, spins))

    def config(self):
        """(threads, mode) of the tuned scan for this filter (mode 0: shared-memory stage, 1: L2 probes, 2:
        shared-memory stage with candidates deferred to the end of each 32-byte block, 3: mode 0 with
        per-stage barriers instead of a block barrier per stage)."""
        t, m = ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.ffbf_get_scan_config(self._h, ctypes.byref(t), ctypes.byref(m)))
        return t.value, m.value

    def probe_order(self):
        """The dense mode's probe plan (0: f0/f1; 1: f2/f3; 2: f0/f1 behind a shared-memory prefilter)."""
        o = ctypes.c_int()
        self._check(self._lib.ffbf_get_probe_order(self._h, ctypes.byref(o)))
        return o.value

    def clear_ff(self):
        self._check(self._lib.ffbf_clear_ff(self._h))

    def get_filters(self):
        nb = self.filter_bytes
        main = np.zeros(nb, dtype=np.uint8)
        ff = np.zeros(nb, dtype=np.uint8)
        self._check(self._lib.ffbf_get_filters(self._h, main.ctypes.data_as(ctypes.c_void_p),
                                               ff.ctypes.data_as(ctypes.c_void_p)))
        return main, ff


class Batch:
    """Many (Filter, device text) scan jobs in one graph launch (ffbf_batch_*)."""

    def __init__(self, device=0):
        self._lib = load_library()
        h = ctypes.c_void_p()
        st = self._lib.ffbf_batch_create(device, ctypes.byref(h))
        if st != 0:
            raise FFBFError(st, "ffbf_batch_create failed")
        self._h = h
        self._filters = []

    def _check(self, st):
        if st != 0:
            raise FFBFError(st, self._lib.ffbf_batch_last_error(self._h).decode(errors="replace"))

    def add(self, filt, dev_ptr, n):
        self._check(self._lib.ffbf_batch_add(self._h, filt._h, ctypes.c_void_p(dev_ptr), n))
        self._filters.append(filt)

    def prepare(self):
        self._check(self._lib.ffbf_batch_prepare(self._h))

    def autotune(self, sample_bytes=16 << 20):
        """Tunes the jobs' scan configurations by class; returns the number of classes."""
        n = ctypes.c_uint32()
        self._check(self._lib.ffbf_batch_autotune(self._h, sample_bytes, ctypes.byref(n)))
        return n.value

    def launch(self):
        self._check(self._lib.ffbf_batch_launch(self._h))

    def wait(self):
        self._check(self._lib.ffbf_batch_wait(self._h))

    @property
    def stream(self):
        return int(self._lib.ffbf_batch_stream(self._h) or 0)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ffbf_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class RequestResult:
    """One finished server request: its hits and candidate lines (as Filter.process returns them) and the
    server's timestamps (seconds since the server started)."""
    request_id: int
    set_id: int
    status: int
    text_len: int
    hit_offsets: np.ndarray
    line_start: np.ndarray
    line_end: np.ndarray
    t_submit: float
    t_admit: float
    t_launch: float
    t_done: float

    @property
    def latency(self):
        return self.t_done - self.t_submit


class Server:
    """Scan server (ffbf_server_*): resident pattern sets, admission by free slots and free device memory,
    continuous batching of the admitted requests on one GPU."""

    def __init__(self, device=0, arena_bytes=0, slots=0):
        self._lib = load_library()
        h = ctypes.c_void_p()
        st = self._lib.ffbf_server_create(device, arena_bytes, slots, ctypes.byref(h))
        if st != 0:
            raise FFBFError(st, "ffbf_server_create failed")
        self._h = h
        self._texts = {}  # request id -> the submitted buffer, kept alive until the request is polled
        self._sets = []

    def _check(self, st):
        if st != 0:
            raise FFBFError(st, self._lib.ffbf_server_last_error(self._h).decode(errors="replace"))

    def add_set(self, filt):
        sid = ctypes.c_uint32()
        self._check(self._lib.ffbf_server_add_set(self._h, filt._h, ctypes.byref(sid)))
        self._sets.append(filt)
        return sid.value

    def submit(self, set_id, text):
        """Queues a scan of `text` (a uint8 numpy array, ideally in pinned memory) against a set."""
        a = np.ascontiguousarray(text, dtype=np.uint8)
        rid = ctypes.c_uint64()
        self._check(self._lib.ffbf_server_submit(self._h, set_id, a.ctypes.data_as(ctypes.c_void_p), a.size,
                                                 ctypes.byref(rid)))
        self._texts[rid.value] = a
        return rid.value

    def poll(self, max_results=256, wait_us=0):
        out = (_RequestResult * max_results)()
        n = ctypes.c_uint32()
        self._check(self._lib.ffbf_server_poll(self._h, out, max_results, ctypes.byref(n), wait_us))
        res = []
        for i in range(n.value):
            r = out[i]
            res.append(RequestResult(int(r.request_id), int(r.set_id), int(r.status), int(r.text_len),
                                     _arr(r.hit_offsets, r.n_hits), _arr(r.line_start, r.n_lines),
                                     _arr(r.line_end, r.n_lines), r.t_submit, r.t_admit, r.t_launch, r.t_done))
            self._lib.ffbf_server_release(self._h, r.request_id)
            self._texts.pop(int(r.request_id), None)
        return res

    def stats(self):
        s = _ServerStats()
        self._check(self._lib.ffbf_server_get_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ffbf_server_destroy(self._h)
            self._h = None
            self._texts.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hashbench_lines(text, device=0):
    """What the reference's `hashbench -l` prints for `text` (hash_rot_sbox_pre_2<19>), hashed on the GPU."""
    lib = load_library()
    p, n, keep = _buf(text)
    out, out_len = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
    st = lib.ffbf_hashbench_lines(device, p, n, ctypes.byref(out), ctypes.byref(out_len))
    if st != 0:
        raise FFBFError(st, "ffbf_hashbench_lines failed")
    return _take_bytes(lib, out, out_len)


def hashbench_file(text, device=0):
    """`hashbench -f` on the GPU: (XOR of the rolling hash after every byte, device seconds)."""
    lib = load_library()
    p, n, keep = _buf(text)
    x, sec = ctypes.c_uint64(), ctypes.c_double()
    st = lib.ffbf_hashbench_file(device, p, n, ctypes.byref(x), ctypes.byref(sec))
    if st != 0:
        raise FFBFError(st, "ffbf_hashbench_file failed")
    return int(x.value), float(sec.value)
