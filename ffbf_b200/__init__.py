"""ffbf_b200: a B200-native (sm_100a) feed-forward Bloom filter matcher.

A drop-in for the x86 rabin-karp path of efficient/ffbf: the filter build, the text scan that sets
feed-forward bits, the feed-forward pattern prune and exact verification all run as CUDA kernels behind the
C ABI in include/ffbf.h. This package gives Python access to that ABI (lib.Filter) and to the seeded
workload generator (datagen).
"""
from .lib import DEFAULT_CHUNK, EXPORTED, Batch, FFBFError, Filter, Params, RequestResult, ScanOutput, Server, format_spans, kernel_launches, load_library  # noqa: F401

__all__ = ["Batch", "DEFAULT_CHUNK", "EXPORTED", "FFBFError", "Filter", "Params", "RequestResult", "ScanOutput", "Server", "format_spans", "kernel_launches", "load_library"]
