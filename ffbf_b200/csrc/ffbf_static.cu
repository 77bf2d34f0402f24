// ffbf_static.cu -- ffbf_scan_static: a scan that allocates no memory.
//
// Some callers cannot let a library call cudaMalloc: a service whose own allocator owns all of the GPU's
// memory (the library would fail or break its accounting), a plug-in host that forbids allocation inside
// callbacks, or a latency-critical loop where an allocation's implicit device synchronisation is not
// acceptable. For them this entry point runs the generic scan and the hit-to-line resolution with every
// piece of scratch memory (hit records, counters, per-tile newline summaries, line spans) taken from one
// file-scope __device__ array of fixed size. The caller still provides the inputs (text, main filter) and
// the outputs (feed-forward filter, hit and line arrays) in device memory it owns.
//
// The array lives in every GPU that loads this library until the process exits. Its device address is
// looked up on every call, in the context current at the call (a lookup allocates nothing), so a
// cudaDeviceReset between calls, or a driver-API context of the caller's own, gets the array of the
// context it runs in. The first call on a device loads the module that holds the array there.
#include <cuda_runtime.h>

#include "../../include/ffbf.h"
#include "ffbf_kernels.cuh"

namespace {

constexpr uint64_t kMaxText = FFBF_STATIC_MAX_TEXT;
constexpr uint32_t kMaxHits = FFBF_STATIC_MAX_HITS;
constexpr uint64_t kMaxTiles = kMaxText / ffbf::kScanTile;

// Scratch layout, in bytes from the start of the array.
constexpr size_t kOffCounters = 0;
constexpr size_t kOffHits = 256;
constexpr size_t kOffLines = kOffHits + sizeof(ffbf::HitRec) * kMaxHits;
constexpr size_t kOffTiles = kOffLines + sizeof(ffbf::HitLine) * kMaxHits;
constexpr size_t kScratchBytes = kOffTiles + 4 * sizeof(long long) * kMaxTiles;
static_assert(kScratchBytes == FFBF_STATIC_SCRATCH_BYTES, "scratch size in include/ffbf.h is stale");

// In host code this name is only a host-side stand-in for the device array: kernels get the address
// cudaGetSymbolAddress returns for the current device, never &g_scan_scratch.
static __device__ __align__(256) unsigned char g_scan_scratch[kScratchBytes];

// The array's device address in the current context. Looked up on every call rather than cached: after a
// cudaDeviceReset the module is loaded again and the array may move, and a caller's own driver-API context
// on the same device has an array of its own.
ffbf_status scratch_for_current_context(unsigned char** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scan_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return FFBF_ECUDA;
    }
    *out = static_cast<unsigned char*>(p);
    return FFBF_OK;
}

__global__ void k_split(const ffbf::HitRec* hits, const ffbf::HitLine* lines, uint32_t n, uint64_t* off,
                        uint64_t* ls, uint64_t* le) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    off[i] = hits[i].off;
    ls[i] = lines[i].start;
    le[i] = lines[i].end;
}

bool pow2(uint64_t x) { return x && !(x & (x - 1)); }

}  // namespace

extern "C" ffbf_status ffbf_scan_static(const ffbf_params* p, const uint32_t* d_main, uint32_t* d_ff,
                                        const uint8_t* d_text, uint64_t len, uint64_t* d_hit_offsets,
                                        uint64_t* d_line_start, uint64_t* d_line_end, uint32_t* n_hits,
                                        void* stream) {
    if (!p || !d_main || !d_ff || !n_hits || !d_hit_offsets || !d_line_start || !d_line_end) return FFBF_EINVAL;
    if (p->len < 1 || p->len > 63 || p->k < 1 || p->k > 11 || p->s > p->k || p->reserved ||
        !pow2(p->cache_bits) || !pow2(p->ext_bits) || p->cache_bits < 32 || p->ext_bits < 32 ||
        p->cache_bits + p->ext_bits > (1ull << 31))
        return FFBF_EINVAL;
    if (len > kMaxText) return FFBF_EINVAL;  // the fixed scratch covers at most FFBF_STATIC_MAX_TEXT bytes
    if (len && (!d_text || ((uintptr_t)d_text & 15))) return FFBF_EINVAL;
    *n_hits = 0;
    unsigned char* scratch = nullptr;
    ffbf_status s = scratch_for_current_context(&scratch);
    if (s != FFBF_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    uint32_t* counters = reinterpret_cast<uint32_t*>(scratch + kOffCounters);
    ffbf::HitRec* hits = reinterpret_cast<ffbf::HitRec*>(scratch + kOffHits);
    ffbf::HitLine* lines = reinterpret_cast<ffbf::HitLine*>(scratch + kOffLines);
    long long* tiles = reinterpret_cast<long long*>(scratch + kOffTiles);

    // The array keeps the previous call's contents; only the counters must start at zero (hit records
    // and tile summaries are written before they are read).
    if (cudaMemsetAsync(counters, 0, ffbf::CNT_WORDS * sizeof(uint32_t), st) != cudaSuccess) {
        cudaGetLastError();
        return FFBF_ECUDA;
    }
    const uint64_t ntiles = (len + ffbf::kScanTile - 1) / ffbf::kScanTile;
    ffbf::ScanArgs a{};
    a.text = d_text;
    a.n = len;
    a.g.len = p->len;
    a.g.k = p->k;
    a.g.s = p->s;
    a.g.cache_bits = (uint32_t)p->cache_bits;
    a.g.cache_mask = (uint32_t)(p->cache_bits - 1);
    a.g.ext_mask = (uint32_t)(p->ext_bits - 1);
    a.g.nbits = (uint32_t)(p->cache_bits + p->ext_bits);
    a.main_words = d_main;
    a.ff_words = d_ff;
    a.hits = hits;
    a.hits_cap = kMaxHits;
    a.counters = counters;
    a.tile_first_nl = tiles;
    a.tile_last_nl = tiles + kMaxTiles;
    a.ntiles = ntiles;
    a.tile_begin = 0;
    a.cache_in_smem = p->cache_bits <= ffbf::kSmemCacheMaxBits;
    if (ntiles) {
        const int grid = ffbf::scan_generic_grid(a.g, a.cache_in_smem, ntiles);
        if (grid <= 0 || ffbf::scan_generic(a, grid, st) != cudaSuccess) {
            cudaGetLastError();
            return FFBF_ECUDA;
        }
    }
    uint32_t found = 0;
    if (cudaMemcpyAsync(&found, counters + ffbf::CNT_HITS, sizeof found, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return FFBF_ECUDA;
    }
    const uint32_t n = found < kMaxHits ? found : kMaxHits;
    if (n) {
        if (ffbf::resolve_lines(d_text, len, p->len, hits, n, tiles, tiles + kMaxTiles, tiles + 2 * kMaxTiles,
                                tiles + 3 * kMaxTiles, ntiles, lines, st) != cudaSuccess) {
            cudaGetLastError();
            return FFBF_ECUDA;
        }
        k_split<<<(n + 255) / 256, 256, 0, st>>>(hits, lines, n, d_hit_offsets, d_line_start, d_line_end);
        ffbf::note_launches(1);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return FFBF_ECUDA;
        }
    }
    *n_hits = found;
    return found > kMaxHits ? FFBF_ENOMEM_DEVICE : FFBF_OK;
}
