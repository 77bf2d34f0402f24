// ffbf_scan_fast.cu -- the tuned sm_100a scan of processFile (src/rabin-karp/ffbf.cpp:310-392).
//
// Work decomposition. The text is cut into streams of SLEN = rows * 128 bytes. A CTA of THREADS threads
// owns THREADS consecutive streams (a "supertile") at a time, one stream per thread, and walks them row by
// row. Each thread rolls the hash over its stream without restarting, so the LEN-byte warm-up is paid once
// per stream (from a 32-byte halo) instead of once per tile.
//
// Staging. Row r of all THREADS streams is one TMA load of a 3-D box {128 bytes, 1 row, THREADS streams}
// (cp.async.bulk.tensor, 128B swizzle, no multicast) into a double-buffered shared-memory stage, completed on
// an mbarrier. The 128B swizzle puts chunk c of thread t's row at chunk c ^ (t & 7), so the eight 16-byte
// reads a quarter-warp issues hit eight different bank groups.
//
// Hash. h <- rol64(h,1) ^ S[in] ^ rol64(S[out], LEN) (hash_rot_sbox_pre_2.h:42-51 with the ring folded
// into the outgoing byte, which is still in registers). S is kept in shared memory as 16 interleaved
// copies, 8 bytes per entry, so the 16 lanes of each half-warp read disjoint banks whatever their bytes.
// Bytes with the high bit set index entries that hold S[0] (ffbf.cpp:127-130).
//
// Probes. The first S index functions (h1, h2 & (C-1)) are tested against a shared-memory copy of the
// cache region (C <= 2^20 bits) or against an exact OR-summary of it (bit j = OR of cache bits
// [j<<sh, (j+1)<<sh)), which can only reject windows the full test rejects. Windows that pass go to the
// full K-bit test on the global bit array, in the reference order (checkInFilter, ffbf.cpp:214-239).
//
// Validity. A window is tested only when its LEN bytes hold no '\n' (processFile resets the hash at '\n').
// The position of the last '\n' is tracked per thread; its first and last '\n' per stream feed the
// per-16 KiB-tile newline summaries the line resolver uses.
//
// Every mbarrier wait is bounded; on timeout the CTA records an error flag and stops.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <climits>

#include "ffbf_scan_fast.cuh"

namespace ffbf {

namespace {

constexpr int kFastThreads = 256;
constexpr int kRowBytes = 128;
constexpr int kStageBytes = kFastThreads * kRowBytes;  // 32 KiB per stage
constexpr int kTabBytes = 256 * 16 * 8;                // 32 KiB: 16 copies of the S-box
constexpr uint32_t kMaxCacheWords = (1u << 20) / 32;   // 128 KiB of cache copy / summary
constexpr uint32_t kWaitLimit = 1u << 24;

struct FastArgs {
    uint64_t n_streams;      // streams covered by the tensor map
    uint32_t rows;           // rows per stream
    uint32_t n_supertiles;   // ceil(n_streams / kFastThreads)
    uint32_t streams_per_tile_log2;  // log2(16384 / (rows * 128))
    Geom g;
    const uint32_t* main_words;
    uint32_t* ff_words;
    const uint32_t* stage1_words;  // cache region copy or its summary (global), copied into smem
    uint32_t stage1_nwords;
    uint32_t stage1_shift;         // index >> shift before the smem lookup (0: exact copy)
    HitRec* hits;
    uint32_t hits_cap;
    uint32_t* counters;
    long long* tile_first_nl;
    long long* tile_last_nl;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

__device__ __forceinline__ uint32_t byte_of(const uint32_t (&w)[32], int pos) {
    return (w[pos >> 2] >> (8 * (pos & 3))) & 0xFFu;
}


template <int L>
__device__ __forceinline__ uint64_t rolL(uint64_t x) {
    return L == 32 ? ((x << 32) | (x >> 32)) : ((x << L) | (x >> (64 - L)));
}

// Full K-bit test on the global main filter, reference order, early exit.
__device__ __noinline__ bool full_check(const Geom g, const uint32_t* __restrict__ words, uint64_t h) {
    for (uint32_t i = 0; i < g.k; i++) {
        uint32_t b = bit_index<1>(g, h, i);
        if (!((__ldg(words + (b >> 5)) >> (b & 31)) & 1u)) return false;
    }
    return true;
}

__device__ __noinline__ void record_hit(const Geom g, uint32_t* ff_words, HitRec* hits, uint32_t cap,
                                       uint32_t* counters, uint64_t start, uint64_t h) {
    set_all<2>(g, ff_words, h);
    uint32_t slot = atomicAdd(counters + CNT_HITS, 1u);
    if (slot < cap) hits[slot] = HitRec{start, h};
}

// First '\n' position (0..127) in a row held as 32 words, or -1.
__device__ __forceinline__ int first_newline(const uint32_t (&w)[32]) {
    for (int k = 0; k < 32; k++) {
        uint32_t t = w[k] ^ 0x0A0A0A0Au;
        uint32_t z = ~(((t & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | t) & 0x80808080u;
        if (z) return 4 * k + (__ffs(z) - 1) / 8;
    }
    return -1;
}

template <int L>
__global__ void __launch_bounds__(kFastThreads, 1) k_scan_fast(const __grid_constant__ CUtensorMap tmap, FastArgs a) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* smem = smem_raw + (base - raw);
    const uint32_t stage0 = base;                       // 2 stages
    uint64_t* tab = reinterpret_cast<uint64_t*>(smem + 2 * kStageBytes);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * kStageBytes + kTabBytes);
    uint32_t* s1 = reinterpret_cast<uint32_t*>(smem + 2 * kStageBytes + kTabBytes + 128);
    __shared__ int s_abort;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    for (int i = tid; i < 256 * 16; i += kFastThreads) {
        int c = i >> 4;
        tab[i] = c_sbox[(c & 0x80) ? 0 : c];
    }
    for (uint32_t i = tid; i < a.stage1_nwords; i += kFastThreads) s1[i] = a.stage1_words[i];
    const uint32_t bar0 = smem_u32(bars), bar1 = bar0 + 8;
    if (tid == 0) {
        s_abort = 0;
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const Geom g = a.g;
    const uint32_t R = a.rows;
    const uint32_t per_st = R + 1;  // halo load + R row loads
    uint32_t my_st = 0;
    if (blockIdx.x < a.n_supertiles) my_st = (a.n_supertiles - 1 - blockIdx.x) / gridDim.x + 1;
    const uint32_t total = my_st * per_st;
    const uint64_t* lane_tab = tab + (lane & 15);  // entry c of this lane's copy: lane_tab[c * 16]
    const uint32_t cmask = g.cache_mask;
    const uint32_t sh = a.stage1_shift;
    const uint32_t* s1w = s1;

    auto issue = [&](uint32_t k) {
        const uint32_t st = blockIdx.x + (k / per_st) * gridDim.x;
        const int r = (int)(k % per_st) - 1;
        const int y = r < 0 ? (int)R - 1 : r;
        const int z = (int)(st * kFastThreads) + (r < 0 ? -1 : 0);
        const uint32_t bar = (k & 1) ? bar1 : bar0;
        mbar_expect_tx(bar, kStageBytes);
        tma_load_3d(stage0 + (k & 1) * kStageBytes, &tmap, 0, y, z, bar);
    };

    if (tid == 0 && total > 0) issue(0);

    uint64_t h = 0;
    int lnp = -1000;               // last '\n' relative to the current row start
    long long first_nl = LLONG_MAX, last_nl = -1;
    uint32_t prev[8] = {0, 0, 0, 0, 0, 0, 0, 0};

    for (uint32_t k = 0; k < total; k++) {
        if (tid == 0 && k + 1 < total) issue(k + 1);
        const uint32_t bar = (k & 1) ? bar1 : bar0;
        const uint32_t parity = (k >> 1) & 1u;
        uint32_t it = 0;
        while (!mbar_try_wait(bar, parity)) {
            if (++it >= kWaitLimit) {
                atomicOr(a.counters + CNT_ERROR, 4u);
                s_abort = 1;
                break;
            }
        }
        if (s_abort) {
            // Give the load issued for k + 1 a bounded chance to land before this CTA's shared memory goes away.
            if (tid == 0 && k + 1 < total) {
                const uint32_t nb = ((k + 1) & 1) ? bar1 : bar0;
                for (uint32_t j = 0; j < kWaitLimit && !mbar_try_wait(nb, ((k + 1) >> 1) & 1u); j++) {
                }
            }
            break;
        }

        const uint32_t st = blockIdx.x + (k / per_st) * gridDim.x;
        const int r = (int)(k % per_st) - 1;
        const uint64_t z = (uint64_t)st * kFastThreads + tid;
        const bool active = z < a.n_streams;
        const uint8_t* row = smem + (k & 1) * kStageBytes + tid * kRowBytes;
        const int sw = tid & 7;

        if (r < 0) {
            // halo: the last 32 bytes before the stream (chunks 6 and 7 of the previous stream's last row)
            const uint4 c6 = *reinterpret_cast<const uint4*>(row + ((6 ^ sw) << 4));
            const uint4 c7 = *reinterpret_cast<const uint4*>(row + ((7 ^ sw) << 4));
            prev[0] = c6.x; prev[1] = c6.y; prev[2] = c6.z; prev[3] = c6.w;
            prev[4] = c7.x; prev[5] = c7.y; prev[6] = c7.z; prev[7] = c7.w;
            h = 0;
            lnp = -1000;
#pragma unroll
            for (int j = 0; j < 32; j++) {
                const uint32_t c = (prev[j >> 2] >> (8 * (j & 3))) & 0xFFu;
                h = rol64(h, 1) ^ lane_tab[c * 16];
                if (j >= L) {
                    const uint32_t co = (prev[(j - L) >> 2] >> (8 * ((j - L) & 3))) & 0xFFu;
                    h ^= rolL<L>(lane_tab[co * 16]);
                }
                if (c == 0x0Au) lnp = j - 32;
            }
            if (z == 0) lnp = -1;  // text start: nothing before offset 0
            first_nl = LLONG_MAX;
            last_nl = -1;
        } else {
            uint32_t w[32];
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const uint4 v = *reinterpret_cast<const uint4*>(row + ((c ^ sw) << 4));
                w[4 * c] = v.x; w[4 * c + 1] = v.y; w[4 * c + 2] = v.z; w[4 * c + 3] = v.w;
            }
            if (active) {
                const long long row_pos = (long long)(z * R + (uint32_t)r) * kRowBytes;
                const int lnp_in = lnp;
#pragma unroll
                for (int p = 0; p < kRowBytes; p++) {
                    const uint32_t c = byte_of(w, p);
                    uint32_t co;
                    if (p >= L) co = byte_of(w, p - L);
                    else co = (prev[(p - L + 32) >> 2] >> (8 * ((p - L + 32) & 3))) & 0xFFu;
                    h = rol64(h, 1) ^ lane_tab[c * 16] ^ rolL<L>(lane_tab[co * 16]);
                    if (c == 0x0Au) lnp = p;
                    if (p - lnp >= L) {
                        const uint32_t i0 = ((uint32_t)h & cmask) >> sh;
                        bool pass = (s1w[i0 >> 5] >> (i0 & 31)) & 1u;
                        if (pass && g.s > 1) {
                            const uint32_t i1 = ((uint32_t)(h >> 32) & cmask) >> sh;
                            pass = (s1w[i1 >> 5] >> (i1 & 31)) & 1u;
                        }
                        if (pass && full_check(g, a.main_words, h))
                            record_hit(g, a.ff_words, a.hits, a.hits_cap, a.counters, (uint64_t)(row_pos + p + 1 - L), h);
                    }
                }
                if (lnp != lnp_in) {
                    if (first_nl == LLONG_MAX) first_nl = row_pos + first_newline(w);
                    last_nl = row_pos + lnp;
                }
                lnp -= kRowBytes;
#pragma unroll
                for (int q = 0; q < 8; q++) prev[q] = w[24 + q];
            }
            if ((uint32_t)r == R - 1) {
                // per-16 KiB-tile newline summary: reduce over the lanes whose streams share the tile
                long long f = active ? first_nl : LLONG_MAX, l = active ? last_nl : -1;
                const int G = 1 << a.streams_per_tile_log2;
                for (int o = 1; o < G; o <<= 1) {
                    f = min(f, __shfl_xor_sync(0xffffffffu, f, o));
                    l = max(l, __shfl_xor_sync(0xffffffffu, l, o));
                }
                if (active && (lane & (G - 1)) == 0) {
                    const uint64_t tile = z >> a.streams_per_tile_log2;
                    a.tile_first_nl[tile] = f;
                    a.tile_last_nl[tile] = l;
                }
            }
        }
        __syncthreads();
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

template <int L>
cudaError_t launch_len(const CUtensorMap& map, const FastArgs& fa, int grid, size_t smem, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(k_scan_fast<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_scan_fast<L><<<grid, kFastThreads, smem, st>>>(map, fa);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace

bool fast_scan_supported(const Geom& g, uint64_t n) {
    switch (g.len) {
        case 16: case 19: case 20: case 24: case 32: break;
        default: return false;
    }
    if (g.s < 1) return false;
    if (n < (uint64_t)kScanTile) return false;
    return encoder() != nullptr;
}

uint32_t stage1_shift_for(const Geom& g) {
    uint32_t sh = 0;
    while (((uint64_t)g.cache_bits >> sh) > (uint64_t)kMaxCacheWords * 32) sh++;
    return sh;
}

cudaError_t scan_fast(const ScanArgs& a, const uint32_t* stage1_words, int num_sms, cudaStream_t st) {
    const uint64_t fast_tiles = a.n / kScanTile;  // whole 16 KiB tiles; the rest goes to the generic kernel
    // rows per stream: the largest power of two (<= 16) that still gives every SM several supertiles
    uint32_t rows = 16;
    while (rows > 4 && fast_tiles * kScanTile / ((uint64_t)rows * kRowBytes * kFastThreads) < 4ull * num_sms) rows >>= 1;
    const uint64_t slen = (uint64_t)rows * kRowBytes;
    const uint64_t n_streams = fast_tiles * kScanTile / slen;
    FastArgs fa{};
    fa.n_streams = n_streams;
    fa.rows = rows;
    fa.n_supertiles = (uint32_t)((n_streams + kFastThreads - 1) / kFastThreads);
    uint32_t spt = (uint32_t)(kScanTile / slen), lg = 0;
    while ((1u << lg) < spt) lg++;
    fa.streams_per_tile_log2 = lg;
    fa.g = a.g;
    fa.main_words = a.main_words;
    fa.ff_words = a.ff_words;
    fa.stage1_words = stage1_words;
    fa.stage1_shift = stage1_shift_for(a.g);
    fa.stage1_nwords = (uint32_t)(((uint64_t)a.g.cache_bits >> fa.stage1_shift) / 32);
    fa.hits = a.hits;
    fa.hits_cap = a.hits_cap;
    fa.counters = a.counters;
    fa.tile_first_nl = a.tile_first_nl;
    fa.tile_last_nl = a.tile_last_nl;

    if (n_streams > 0) {
        CUtensorMap map;
        cuuint64_t dims[3] = {(cuuint64_t)kRowBytes, (cuuint64_t)rows, (cuuint64_t)n_streams};
        cuuint64_t strides[2] = {(cuuint64_t)kRowBytes, (cuuint64_t)slen};
        cuuint32_t box[3] = {(cuuint32_t)kRowBytes, 1u, (cuuint32_t)kFastThreads};
        cuuint32_t estr[3] = {1u, 1u, 1u};
        CUresult cr = encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void*)a.text, dims, strides, box, estr,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
        const size_t smem = 1024 + 2 * kStageBytes + kTabBytes + 128 + 4 * (size_t)fa.stage1_nwords;
        const int grid = (int)(fa.n_supertiles < (uint32_t)num_sms ? fa.n_supertiles : (uint32_t)num_sms);
        cudaError_t e;
        switch (a.g.len) {
            case 16: e = launch_len<16>(map, fa, grid, smem, st); break;
            case 19: e = launch_len<19>(map, fa, grid, smem, st); break;
            case 20: e = launch_len<20>(map, fa, grid, smem, st); break;
            case 24: e = launch_len<24>(map, fa, grid, smem, st); break;
            case 32: e = launch_len<32>(map, fa, grid, smem, st); break;
            default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
    }
    // the partial last tile (and anything the streams did not cover) through the generic kernel
    const uint64_t ntiles = (a.n + kScanTile - 1) / kScanTile;
    if (fast_tiles < ntiles) {
        ScanArgs t = a;
        t.tile_begin = fast_tiles;
        t.cache_in_smem = a.g.cache_bits <= kSmemCacheMaxBits;
        const int grid = scan_generic_grid(a.g, t.cache_in_smem, ntiles - fast_tiles);
        if (grid <= 0) return cudaErrorInvalidConfiguration;
        return scan_generic(t, grid, st);
    }
    return cudaSuccess;
}

// Summary of the cache region for the stage-1 test: bit j = OR of cache bits [j << sh, (j + 1) << sh).
__global__ void k_stage1_summary(const uint32_t* main_words, uint32_t cache_bits, uint32_t sh, uint32_t* out,
                                 uint32_t nwords) {
    uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwords) return;
    uint32_t v = 0;
    for (uint32_t b = 0; b < 32; b++) {
        const uint64_t lo = ((uint64_t)(w * 32 + b)) << sh, hi = lo + (1ull << sh);
        bool any = false;
        for (uint64_t i = lo; i < hi && !any;) {
            if ((i & 31) == 0 && i + 32 <= hi) {
                any = main_words[i >> 5] != 0;
                i += 32;
            } else {
                any = (main_words[i >> 5] >> (i & 31)) & 1u;
                i++;
            }
        }
        v |= (uint32_t)any << b;
    }
    out[w] = v;
    (void)cache_bits;
}

cudaError_t build_stage1(const uint32_t* main_words, const Geom& g, uint32_t* out, cudaStream_t st) {
    const uint32_t sh = stage1_shift_for(g);
    const uint32_t nwords = (uint32_t)(((uint64_t)g.cache_bits >> sh) / 32);
    if (sh == 0) return cudaMemcpyAsync(out, main_words, 4ull * nwords, cudaMemcpyDeviceToDevice, st);
    k_stage1_summary<<<(nwords + 255) / 256, 256, 0, st>>>(main_words, g.cache_bits, sh, out, nwords);
    note_launches(1);
    return cudaGetLastError();
}

uint32_t stage1_words_for(const Geom& g) { return (uint32_t)(((uint64_t)g.cache_bits >> stage1_shift_for(g)) / 32); }

}  // namespace ffbf
