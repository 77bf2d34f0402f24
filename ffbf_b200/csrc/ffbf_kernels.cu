// ffbf_kernels.cu -- FFBF device kernels other than the tuned scan: pattern line table and prefix
// hashing (filter build), the generic scan, hit -> line resolution, feed-forward prune, ordered
// compaction, the exact-verification hash table and byte compare, the filter cache codec and the
// single-line test.
#include <atomic>
#include <climits>

#include "ffbf_kernels.cuh"

namespace ffbf {

static std::atomic<uint64_t> g_launches{0};
void note_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void unnote_launches(uint64_t n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
uint64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }

// ------------------------------------------------------------------------------------------------
// Block-wide exclusive scan (THREADS a multiple of 32, <= 1024). `sh` holds THREADS/32 values.
template <int THREADS, class T>
__device__ __forceinline__ T block_excl_scan(T v, T* sh, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < THREADS / 32 ? sh[lane] : T(0);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w += y;
        }
        if (lane < THREADS / 32) sh[lane] = w;
    }
    __syncthreads();
    T before = warp ? sh[warp - 1] : T(0);
    *total = sh[THREADS / 32 - 1];
    __syncthreads();
    return before + x - v;
}

// ------------------------------------------------------------------------------------------------
// Ordered compaction, three phases: per-chunk counts, one-block exclusive scan of the counts, and an
// ordered emit where every block writes the indices of its chunk in ascending order.
constexpr int kCompThreads = 256;
constexpr int kCompItems = 16;                                     // consecutive items per thread per round
constexpr uint64_t kCompChunk = (uint64_t)kCompThreads * kCompItems * 16;  // items per block

struct BytePred {
    const uint8_t* p;
    uint8_t b;
    __device__ bool operator()(uint64_t i) const { return p[i] == b; }
};
struct FlagPred {
    const uint8_t* p;
    __device__ bool operator()(uint64_t i) const { return p[i] != 0; }
};

template <class Pred>
__global__ void __launch_bounds__(kCompThreads) k_count(Pred pred, uint64_t n, uint64_t* counts) {
    __shared__ uint64_t sh[kCompThreads / 32];
    uint64_t lo = blockIdx.x * kCompChunk, hi = min(n, lo + kCompChunk);
    uint64_t c = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kCompThreads) c += pred(i) ? 1 : 0;
    uint64_t tot;
    block_excl_scan<kCompThreads>(c, sh, &tot);
    if (threadIdx.x == 0) counts[blockIdx.x] = tot;
}

// In place: counts[0..nb) -> exclusive prefix sums, counts[nb] = total. One block.
template <class T>
__global__ void __launch_bounds__(1024) k_scan_single(T* counts, uint64_t nb) {
    __shared__ T sh[32];
    T carry = 0;
    for (uint64_t base = 0; base < nb; base += 1024) {
        uint64_t i = base + threadIdx.x;
        T v = i < nb ? counts[i] : T(0);
        T tot;
        T ex = block_excl_scan<1024>(v, sh, &tot);
        if (i < nb) counts[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) counts[nb] = carry;
}

template <class Pred>
__global__ void __launch_bounds__(kCompThreads) k_emit(Pred pred, uint64_t n, const uint64_t* offsets, uint64_t* out) {
    __shared__ uint64_t sh[kCompThreads / 32];
    uint64_t lo = blockIdx.x * kCompChunk, hi = min(n, lo + kCompChunk);
    uint64_t base = offsets[blockIdx.x];
    for (uint64_t r = lo; r < hi; r += (uint64_t)kCompThreads * kCompItems) {
        uint64_t a = r + (uint64_t)threadIdx.x * kCompItems;
        uint64_t b = min(hi, a + kCompItems);
        uint64_t c = 0;
        for (uint64_t i = a; i < b; i++) c += pred(i) ? 1 : 0;
        uint64_t tot;
        uint64_t pos = base + block_excl_scan<kCompThreads>(c, sh, &tot);
        for (uint64_t i = a; i < b; i++)
            if (pred(i)) out[pos++] = i;
        base += tot;
    }
}

uint64_t compact_blocks(uint64_t n) { return (n + kCompChunk - 1) / kCompChunk; }

template <class Pred>
static cudaError_t compact_count(Pred pred, uint64_t n, uint64_t* d_tmp, cudaStream_t st) {
    uint64_t nb = compact_blocks(n);
    if (nb == 0) return cudaMemsetAsync(d_tmp, 0, sizeof(uint64_t), st);
    k_count<<<(unsigned)nb, kCompThreads, 0, st>>>(pred, n, d_tmp);
    note_launches(1);
    k_scan_single<uint64_t><<<1, 1024, 0, st>>>(d_tmp, nb);
    note_launches(1);
    return cudaGetLastError();
}

template <class Pred>
static cudaError_t compact_emit(Pred pred, uint64_t n, uint64_t* d_out, const uint64_t* d_tmp, cudaStream_t st) {
    uint64_t nb = compact_blocks(n);
    if (nb == 0) return cudaSuccess;
    k_emit<<<(unsigned)nb, kCompThreads, 0, st>>>(pred, n, d_tmp, d_out);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t count_bytes(const uint8_t* d_buf, uint64_t n, uint8_t byte, uint64_t* d_tmp, cudaStream_t st) {
    return compact_count(BytePred{d_buf, byte}, n, d_tmp, st);
}
cudaError_t emit_bytes(const uint8_t* d_buf, uint64_t n, uint8_t byte, uint64_t* d_pos, const uint64_t* d_tmp,
                       cudaStream_t st) {
    return compact_emit(BytePred{d_buf, byte}, n, d_pos, d_tmp, st);
}
cudaError_t count_flags(const uint8_t* d_flags, uint64_t n, uint64_t* d_tmp, cudaStream_t st) {
    return compact_count(FlagPred{d_flags}, n, d_tmp, st);
}
cudaError_t emit_flags(const uint8_t* d_flags, uint64_t n, uint64_t* d_out, const uint64_t* d_tmp, cudaStream_t st) {
    return compact_emit(FlagPred{d_flags}, n, d_out, d_tmp, st);
}

// Line table of a pattern file from its newline positions: line i ends at nl[i] (or at n for a final
// line without '\n') and starts one past the previous line's end.
__global__ void k_lines(const uint64_t* nl, uint64_t m, uint64_t n, int tail, uint64_t* start, uint64_t* end) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t cnt = m + (tail ? 1 : 0);
    if (i >= cnt) return;
    end[i] = i < m ? nl[i] : n;
    start[i] = i == 0 ? 0 : nl[i - 1] + 1;
}

cudaError_t lines_from_newlines(const uint64_t* d_nl, uint64_t m, uint64_t n, int tail, uint64_t* d_start,
                                uint64_t* d_end, cudaStream_t st) {
    uint64_t cnt = m + (tail ? 1 : 0);
    if (!cnt) return cudaSuccess;
    k_lines<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(d_nl, m, n, tail, d_start, d_end);
    note_launches(1);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// Filter build: one thread per pattern line. operator<< (ffbf.cpp:268-283) hashes the first LEN bytes
// of a line at least LEN long and sets K bits in getHashValue order. The prefix hash is kept for the
// feed-forward prune and for verification.
__global__ void k_hash_patterns(const uint8_t* file, const uint64_t* start, const uint64_t* end, uint64_t npat,
                                Geom g, uint64_t* hash, uint32_t* main_words, int set_bits) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= npat) return;
    uint64_t s = start[i], e = end[i];
    if (e - s < g.len) {
        hash[i] = 0;
        return;
    }
    uint64_t h = window_hash(file + s, g.len);
    hash[i] = h;
    if (set_bits)
        for (uint32_t j = 0; j < g.k; j++) {
            uint32_t b = bit_index<1>(g, h, j);
            atomicOr(main_words + (b >> 5), 1u << (b & 31));
        }
}

cudaError_t hash_patterns(const uint8_t* d_file, const uint64_t* d_start, const uint64_t* d_end, uint64_t npat,
                          const Geom& g, uint64_t* d_hash, uint32_t* d_main, int set_bits, cudaStream_t st) {
    if (!npat) return cudaSuccess;
    k_hash_patterns<<<(unsigned)((npat + 255) / 256), 256, 0, st>>>(d_file, d_start, d_end, npat, g, d_hash, d_main,
                                                                       set_bits);
    note_launches(1);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// Generic scan (any LEN 1..63, K, S, geometry). processFile (ffbf.cpp:310-392) restated per window:
// the window ending at p is valid when its LEN bytes hold no '\n' (the reference resets the hash at
// '\n' and tests only once LEN bytes followed); a valid window hits when its K main bits are set, and
// then sets K feed-forward bits. Each CTA stages TILE bytes plus a 64-byte halo in shared memory; each
// thread owns SEG consecutive window ends and rolls the hash over them after a LEN-byte warm-up.
// The staged bytes are padded by 4 bytes after every 64 so that the threads' segments (64 bytes apart)
// fall in different banks.
__host__ __device__ __forceinline__ uint32_t pad_idx(uint32_t q) { return q + ((q >> 6) << 2); }

size_t scan_smem_bytes(int cache_in_smem, const Geom& g) {
    size_t text = pad_idx(kScanTile + kHalo) + 16;
    size_t b = 2048 + 16 + ((text + 15) & ~(size_t)15);
    if (cache_in_smem) b += g.cache_bits / 8;
    return b;
}

// One 16 KiB tile of the generic scan (window ends [tile*T, tile*T + T)). The caller provides the shared
// S-box copy, the tile newline accumulator, the padded staging buffer and the cache-region words to probe
// (shared-memory copy or the global filter).
__device__ __forceinline__ void generic_tile(const ScanArgs& a, uint64_t tile, const uint64_t* s_sbox, long long* s_nl,
                                             uint8_t* s_text, const uint32_t* cache_words) {
    const Geom g = a.g;
    const uint32_t L = g.len;
    const int tid = threadIdx.x;
    __syncthreads();
    const long long t0 = (long long)(tile * kScanTile);
    for (int q = tid; q < (kScanTile + kHalo) / 4; q += kScanThreads) {
        long long p = t0 - kHalo + 4LL * q;
        uint32_t v;
        if (p >= 0 && p + 4 <= (long long)a.n) {
            v = __ldg(reinterpret_cast<const uint32_t*>(a.text + p));
        } else {
            v = 0;
            for (int j = 0; j < 4; j++) {
                long long pj = p + j;
                uint32_t b = (pj < 0 || pj >= (long long)a.n) ? 0x0Au : a.text[pj];
                v |= b << (8 * j);
            }
        }
        *reinterpret_cast<uint32_t*>(s_text + pad_idx(4 * q)) = v;
    }
    if (tid == 0) {
        s_nl[0] = LLONG_MAX;
        s_nl[1] = -1;
    }
    __syncthreads();

    const long long seg0 = t0 + (long long)tid * kScanSeg;
    long long my_first = LLONG_MAX, my_last = -1;
    if (seg0 < (long long)a.n) {
        const long long seg1 = min(seg0 + kScanSeg, (long long)a.n);
        // staged byte of text position p: s_text[pad_idx(p - (t0 - kHalo))]
        const long long off = kHalo - t0;
        uint64_t h = 0;
        uint32_t run = 0;
        for (long long p = seg0 - L; p < seg0; p++) {
            uint32_t c = s_text[pad_idx((uint32_t)(p + off))];
            h = rol64(h, 1) ^ s_sbox[c];
            run = c == 0x0Au ? 0u : min(run + 1u, L);
        }
        for (long long p = seg0; p < seg1; p++) {
            uint32_t c = s_text[pad_idx((uint32_t)(p + off))];
            uint32_t co = s_text[pad_idx((uint32_t)(p - L + off))];
            h = rol64(h, 1) ^ s_sbox[c] ^ rol64(s_sbox[co], L);
            if (c == 0x0Au) {
                run = 0;
                if (my_first == LLONG_MAX) my_first = p;
                my_last = p;
                continue;
            }
            run = min(run + 1u, L);
            if (run < L) continue;
            bool hit = true;
            for (uint32_t i = 0; i < g.k && hit; i++) {
                uint32_t b = bit_index<1>(g, h, i);
                hit = test_bit(i < g.s ? cache_words : a.main_words, b);
            }
            if (hit) {
                set_all<2>(g, a.ff_words, h);
                uint32_t slot = atomicAdd(a.counters + CNT_HITS, 1u);
                if (slot < a.hits_cap) a.hits[slot] = HitRec{(uint64_t)(p + 1 - L), h};
            }
        }
    }
    if (my_first != LLONG_MAX) atomicMin(s_nl + 0, my_first);
    if (my_last >= 0) atomicMax(s_nl + 1, my_last);
    __syncthreads();
    if (tid == 0) {
        a.tile_first_nl[tile] = s_nl[0];
        a.tile_last_nl[tile] = s_nl[1];
    }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_generic(ScanArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint64_t* s_sbox = reinterpret_cast<uint64_t*>(smem);
    long long* s_nl = reinterpret_cast<long long*>(smem + 2048);
    uint8_t* s_text = smem + 2048 + 16;
    const uint32_t text_bytes = (pad_idx(kScanTile + kHalo) + 16 + 15) & ~15u;
    uint32_t* s_cache = reinterpret_cast<uint32_t*>(s_text + text_bytes);
    const int tid = threadIdx.x;
    for (int i = tid; i < 256; i += kScanThreads) s_sbox[i] = c_sbox[(i & 0x80) ? 0 : i];
    if (a.cache_in_smem)
        for (uint32_t w = tid; w < a.g.cache_bits / 32; w += kScanThreads) s_cache[w] = a.main_words[w];
    const uint32_t* cache_words = a.cache_in_smem ? s_cache : a.main_words;
    for (uint64_t tile = a.tile_begin + blockIdx.x; tile < a.ntiles; tile += gridDim.x)
        generic_tile(a, tile, s_sbox, s_nl, s_text, cache_words);
}

// Generic scan over tiles of many jobs: item i is tile items[i].y of job items[i].x. Probes the global filter.
__global__ void __launch_bounds__(kScanThreads) k_scan_generic_multi(const ScanArgs* jobs, const uint2* items,
                                                                     uint32_t n_items) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint64_t* s_sbox = reinterpret_cast<uint64_t*>(smem);
    long long* s_nl = reinterpret_cast<long long*>(smem + 2048);
    uint8_t* s_text = smem + 2048 + 16;
    for (int i = threadIdx.x; i < 256; i += kScanThreads) s_sbox[i] = c_sbox[(i & 0x80) ? 0 : i];
    for (uint32_t i = blockIdx.x; i < n_items; i += gridDim.x) {
        const uint2 it = items[i];
        const ScanArgs a = jobs[it.x];
        if (it.y >= a.ntiles) {  // self-check: skip a tile outside the job's text
            if (threadIdx.x == 0) atomicOr(a.counters + CNT_ERROR, 0x1000u);
            continue;
        }
        generic_tile(a, it.y, s_sbox, s_nl, s_text, a.main_words);
    }
}

cudaError_t scan_generic_multi(const ScanArgs* d_jobs, const uint2* d_items, uint32_t n_items, int num_sms,
                               cudaStream_t st) {
    if (!n_items) return cudaSuccess;
    const Geom none{};
    const size_t smem = scan_smem_bytes(0, none);
    cudaError_t e = cudaFuncSetAttribute(k_scan_generic_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint32_t grid = n_items < (uint32_t)(4 * num_sms) ? n_items : (uint32_t)(4 * num_sms);
    k_scan_generic_multi<<<grid, kScanThreads, smem, st>>>(d_jobs, d_items, n_items);
    note_launches(1);
    return cudaGetLastError();
}

// Zeroes the counters of every job of a batch.
__global__ void k_zero_counters(uint32_t* const* ptrs, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n * CNT_WORDS) ptrs[i / CNT_WORDS][i % CNT_WORDS] = 0;
}

cudaError_t zero_counters(uint32_t* const* d_ptrs, uint32_t n, cudaStream_t st) {
    if (!n) return cudaSuccess;
    k_zero_counters<<<(n * CNT_WORDS + 255) / 256, 256, 0, st>>>(d_ptrs, n);
    note_launches(1);
    return cudaGetLastError();
}

// Copies the counters of n jobs into one array (CNT_WORDS words per job), for one device-to-host copy.
__global__ void k_gather_counters(uint32_t* const* ptrs, uint32_t n, uint32_t* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n * CNT_WORDS) out[i] = ptrs[i / CNT_WORDS][i % CNT_WORDS];
}

cudaError_t gather_counters(uint32_t* const* d_ptrs, uint32_t n, uint32_t* d_out, cudaStream_t st) {
    if (!n) return cudaSuccess;
    k_gather_counters<<<(n * CNT_WORDS + 255) / 256, 256, 0, st>>>(d_ptrs, n, d_out);
    note_launches(1);
    return cudaGetLastError();
}

int scan_generic_grid(const Geom& g, int cache_in_smem, uint64_t ntiles) {
    size_t smem = scan_smem_bytes(cache_in_smem, g);
    if (cudaFuncSetAttribute(k_scan_generic, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_scan_generic, kScanThreads, smem) != cudaSuccess) return 0;
    uint64_t grid = (uint64_t)sms * (per > 0 ? per : 1);
    return (int)(grid < ntiles ? grid : (ntiles ? ntiles : 1));
}

cudaError_t scan_generic(const ScanArgs& a, int grid, cudaStream_t st) {
    size_t smem = scan_smem_bytes(a.cache_in_smem, a.g);
    cudaError_t e = cudaFuncSetAttribute(k_scan_generic, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (a.ntiles <= a.tile_begin) return cudaSuccess;
    k_scan_generic<<<grid, kScanThreads, smem, st>>>(a);
    note_launches(1);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// Hit -> line span. Tile summaries give, for every tile, the last '\n' before it and the first '\n'
// after it, so each hit searches at most one tile in each direction.
__global__ void __launch_bounds__(1024) k_tile_nl_scan(const long long* first, const long long* last,
                                                       long long* prev_nl, long long* next_nl, uint64_t nt) {
    // prev_nl[t] = max(last[0..t)), next_nl[t] = min(first(t..nt)). One block; per-thread ranges.
    __shared__ long long sh[1024];
    const uint64_t per = (nt + 1023) / 1024;
    const uint64_t lo = min(nt, threadIdx.x * per), hi = min(nt, lo + per);
    long long m = -1;
    for (uint64_t t = lo; t < hi; t++) m = max(m, last[t]);
    sh[threadIdx.x] = m;
    __syncthreads();
    long long before = -1;
    for (unsigned u = 0; u < threadIdx.x; u++) before = max(before, sh[u]);
    for (uint64_t t = lo; t < hi; t++) {
        prev_nl[t] = before;
        before = max(before, last[t]);
    }
    __syncthreads();
    long long f = LLONG_MAX;
    for (uint64_t t = lo; t < hi; t++) f = min(f, first[t]);
    sh[threadIdx.x] = f;
    __syncthreads();
    long long after = LLONG_MAX;
    for (unsigned u = threadIdx.x + 1; u < 1024; u++) after = min(after, sh[u]);
    for (uint64_t t = hi; t > lo; t--) {
        next_nl[t - 1] = after;
        after = min(after, first[t - 1]);
    }
}

// The same prefix max / suffix min in two passes over blocks of kTileAggBlock tiles (4 per thread):
// k_tile_agg reduces each block, k_tile_scan2 folds the other blocks' aggregates into a carry and scans its
// block with warp shuffles. Loads are coalesced and every SM takes part.
__global__ void __launch_bounds__(1024) k_tile_agg(const long long* first, const long long* last, uint64_t nt,
                                                   long long* agg_first, long long* agg_last) {
    __shared__ long long s_f[32], s_l[32];
    const uint64_t t0 = (uint64_t)blockIdx.x * kTileAggBlock;
    long long f = LLONG_MAX, l = -1;
    for (uint32_t k = threadIdx.x; k < kTileAggBlock; k += 1024) {
        const uint64_t t = t0 + k;
        if (t < nt) {
            f = min(f, first[t]);
            l = max(l, last[t]);
        }
    }
    for (int o = 16; o; o >>= 1) {
        f = min(f, __shfl_xor_sync(0xffffffffu, f, o));
        l = max(l, __shfl_xor_sync(0xffffffffu, l, o));
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_f[w] = f;
        s_l[w] = l;
    }
    __syncthreads();
    if (w == 0) {
        f = s_f[lane];
        l = s_l[lane];
        for (int o = 16; o; o >>= 1) {
            f = min(f, __shfl_xor_sync(0xffffffffu, f, o));
            l = max(l, __shfl_xor_sync(0xffffffffu, l, o));
        }
        if (lane == 0) {
            agg_first[blockIdx.x] = f;
            agg_last[blockIdx.x] = l;
        }
    }
}

__global__ void __launch_bounds__(1024) k_tile_scan2(const long long* first, const long long* last, uint64_t nt,
                                                     const long long* agg_first, const long long* agg_last,
                                                     uint32_t nb, long long* prev_nl, long long* next_nl) {
    __shared__ long long s_a[32], s_b[32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t b = blockIdx.x;
    // carries: the last '\n' of all earlier blocks, the first '\n' of all later ones
    long long cp = -1, cn = LLONG_MAX;
    for (uint32_t i = threadIdx.x; i < b; i += 1024) cp = max(cp, agg_last[i]);
    for (uint32_t i = b + 1 + threadIdx.x; i < nb; i += 1024) cn = min(cn, agg_first[i]);
    for (int o = 16; o; o >>= 1) {
        cp = max(cp, __shfl_xor_sync(0xffffffffu, cp, o));
        cn = min(cn, __shfl_xor_sync(0xffffffffu, cn, o));
    }
    if (lane == 0) {
        s_a[w] = cp;
        s_b[w] = cn;
    }
    __syncthreads();
    cp = s_a[lane];
    cn = s_b[lane];
    for (int o = 16; o; o >>= 1) {
        cp = max(cp, __shfl_xor_sync(0xffffffffu, cp, o));
        cn = min(cn, __shfl_xor_sync(0xffffffffu, cn, o));
    }
    __syncthreads();
    // this thread's 4 consecutive tiles
    const uint64_t t0 = (uint64_t)b * kTileAggBlock + 4u * threadIdx.x;
    long long L[4], F[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const bool in = t0 + k < nt;
        L[k] = in ? last[t0 + k] : -1;
        F[k] = in ? first[t0 + k] : LLONG_MAX;
    }
    const long long mx = max(max(L[0], L[1]), max(L[2], L[3]));
    const long long mn = min(min(F[0], F[1]), min(F[2], F[3]));
    // exclusive prefix max of mx and exclusive suffix min of mn over the block's threads
    long long pre = mx, suf = mn;
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, pre, o);
        const long long d = __shfl_down_sync(0xffffffffu, suf, o);
        if (lane >= o) pre = max(pre, u);
        if (lane + o < 32) suf = min(suf, d);
    }
    if (lane == 31) s_a[w] = pre;  // warp totals
    if (lane == 0) s_b[w] = suf;
    __syncthreads();
    long long wpre = -1, wsuf = LLONG_MAX;
    for (int u = 0; u < w; u++) wpre = max(wpre, s_a[u]);
    for (int u = w + 1; u < 32; u++) wsuf = min(wsuf, s_b[u]);
    long long ex_pre = __shfl_up_sync(0xffffffffu, pre, 1);
    long long ex_suf = __shfl_down_sync(0xffffffffu, suf, 1);
    if (lane == 0) ex_pre = -1;
    if (lane == 31) ex_suf = LLONG_MAX;
    long long run = max(cp, max(wpre, ex_pre));
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (t0 + k < nt) prev_nl[t0 + k] = run;
        run = max(run, L[k]);
    }
    run = min(cn, min(wsuf, ex_suf));
#pragma unroll
    for (int k = 3; k >= 0; k--) {
        if (t0 + k < nt) next_nl[t0 + k] = run;
        run = min(run, F[k]);
    }
}

// Byte masks of '\n' in a 32-bit word (0x80 in each byte that is '\n'; no false positives).
__device__ __forceinline__ uint32_t nl_bytes(uint32_t w) {
    const uint32_t t = w ^ 0x0A0A0A0Au;
    return ~(((t & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | t) & 0x80808080u;
}

// The aligned 16 bytes of `text` at c (c a multiple of 16, c < n). The last, partial chunk of a text whose
// length is not a multiple of 16 is read byte by byte, zero-filled past n, so nothing beyond the text is read.
__device__ __forceinline__ uint4 chunk16(const uint8_t* text, long long c, long long n) {
    if (c + 16 <= n) return __ldg(reinterpret_cast<const uint4*>(text + c));
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    for (int i = 0; i < 16 && c + i < n; i++) w[i >> 2] |= (uint32_t)__ldg(text + c + i) << (8 * (i & 3));
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// Last '\n' in [lo, p] (lo <= p < n), or -1: aligned 16-byte chunks from p down to lo.
__device__ __forceinline__ long long last_nl_back(const uint8_t* text, long long n, long long lo, long long p) {
    while (p >= lo) {
        const long long c = p & ~15LL;
        const uint4 v = chunk16(text, c, n);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
        // bytes of the chunk at offsets max(lo - c, 0) .. p - c
        const int hi = (int)(p - c), low = (int)max(lo - c, 0LL);
        for (int q = hi >> 2; q >= (low >> 2); q--) {
            uint32_t m = nl_bytes(w[q]);
            // keep byte positions 4q + b with low <= 4q + b <= hi
            const int b_hi = min(hi - 4 * q, 3), b_lo = max(low - 4 * q, 0);
            m &= (0xFFFFFFFFu >> (8 * (3 - b_hi))) & (0xFFFFFFFFu << (8 * b_lo));
            if (m) return c + 4 * q + (31 - __clz(m)) / 8;
        }
        p = c - 1;
    }
    return -1;
}

// First '\n' in [q, hi) (q < hi <= n), or -1: aligned 16-byte chunks from q up to hi.
__device__ __forceinline__ long long first_nl_fwd(const uint8_t* text, long long n, long long q, long long hi) {
    while (q < hi) {
        const long long c = q & ~15LL;
        const uint4 v = chunk16(text, c, n);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
        const int low = (int)(q - c), top = (int)min(hi - c, 16LL) - 1;  // offsets low .. top
        for (int k = low >> 2; k <= (top >> 2); k++) {
            uint32_t m = nl_bytes(w[k]);
            const int b_lo = max(low - 4 * k, 0), b_hi = min(top - 4 * k, 3);
            m &= (0xFFFFFFFFu << (8 * b_lo)) & (0xFFFFFFFFu >> (8 * (3 - b_hi)));
            if (m) return c + 4 * k + (__ffs(m) - 1) / 8;
        }
        q = c + 16;
    }
    return -1;
}

__global__ void k_resolve(const uint8_t* text, uint64_t n, uint32_t len, const HitRec* hits, uint32_t nhits,
                          const long long* prev_nl, const long long* next_nl, HitLine* out) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nhits) return;
    const uint64_t w = hits[j].off;
    // line start: the last '\n' before the window in its tile, else the tile summaries' prefix
    uint64_t s = 0;
    if (w > 0) {
        const uint64_t tb = (w - 1) / kScanTile;
        const long long p = last_nl_back(text, (long long)n, (long long)(tb * kScanTile), (long long)w - 1);
        s = p >= 0 ? (uint64_t)p + 1 : (uint64_t)(prev_nl[tb] + 1);
    }
    // line end: the first '\n' after the window in its tile, else the suffix summary, else the text's end
    uint64_t e = n;
    const uint64_t q = w + len;
    if (q < n) {
        const uint64_t te = q / kScanTile;
        const uint64_t hi = min(n, (te + 1) * (uint64_t)kScanTile);
        const long long f = first_nl_fwd(text, (long long)n, (long long)q, (long long)hi);
        if (f >= 0) e = (uint64_t)f;
        else e = next_nl[te] == LLONG_MAX ? n : (uint64_t)next_nl[te];
    }
    out[j] = HitLine{s, e};
}

cudaError_t resolve_lines(const uint8_t* text, uint64_t n, uint32_t len, const HitRec* hits, uint32_t nhits,
                          const long long* tile_first, const long long* tile_last, long long* prev_nl,
                          long long* next_nl, uint64_t ntiles, HitLine* out, cudaStream_t st, long long* agg) {
    if (ntiles && agg) {
        const uint32_t nb = (uint32_t)((ntiles + kTileAggBlock - 1) / kTileAggBlock);
        k_tile_agg<<<nb, 1024, 0, st>>>(tile_first, tile_last, ntiles, agg, agg + nb);
        k_tile_scan2<<<nb, 1024, 0, st>>>(tile_first, tile_last, ntiles, agg, agg + nb, nb, prev_nl, next_nl);
        note_launches(2);
    } else if (ntiles) {
        k_tile_nl_scan<<<1, 1024, 0, st>>>(tile_first, tile_last, prev_nl, next_nl, ntiles);
        note_launches(1);
    }
    if (nhits) {
        k_resolve<<<(nhits + 255) / 256, 256, 0, st>>>(text, n, len, hits, nhits, prev_nl, next_nl, out);
        note_launches(1);
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// Feed-forward prune (filterPhrases, ffbf.cpp:394-485): a line survives when it is >= LEN bytes and its
// prefix window's K feed-forward bits (getHashValue_2 order) are set.
__global__ void k_prune(const uint64_t* start, const uint64_t* end, const uint64_t* hash, uint64_t npat, Geom g,
                        const uint32_t* ff, uint8_t* flags) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= npat) return;
    flags[i] = (end[i] - start[i] >= g.len) && check_all<2>(g, ff, hash[i]);
}

cudaError_t prune_flags(const uint64_t* d_start, const uint64_t* d_end, const uint64_t* d_hash, uint64_t npat,
                        const Geom& g, const uint32_t* d_ff, uint8_t* d_flags, cudaStream_t st) {
    if (!npat) return cudaSuccess;
    k_prune<<<(unsigned)((npat + 255) / 256), 256, 0, st>>>(d_start, d_end, d_hash, npat, g, d_ff, d_flags);
    note_launches(1);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// Exact verification. Open-addressing multimap keyed by the pruned patterns' 64-bit prefix hash; every
// pattern gets its own slot (several patterns may share a prefix). Slots are claimed with atomicCAS on
// the value array (empty = 0xffffffff); lookups run in a later kernel.
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    return x ^ (x >> 33);
}

__global__ void k_table_build(const uint64_t* ids, uint64_t nids, const uint64_t* hash, uint64_t* keys,
                              uint32_t* vals, uint64_t mask, uint32_t* counters) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= nids) return;
    uint32_t id = (uint32_t)ids[i];
    uint64_t key = hash[id];
    uint64_t slot = mix64(key) & mask;
    for (uint64_t probe = 0; probe <= mask; probe++) {
        uint32_t old = atomicCAS(vals + slot, 0xffffffffu, id);
        if (old == 0xffffffffu) {
            keys[slot] = key;
            return;
        }
        slot = (slot + 1) & mask;
    }
    atomicOr(counters + CNT_ERROR, 1u);  // table full: cannot happen with size >= 2 * nids
}

cudaError_t table_build(const uint64_t* d_ids, uint64_t nids, const uint64_t* d_hash, uint64_t* d_keys,
                        uint32_t* d_vals, uint64_t mask, uint32_t* d_counters, cudaStream_t st) {
    if (!nids) return cudaSuccess;
    k_table_build<<<(unsigned)((nids + 255) / 256), 256, 0, st>>>(d_ids, nids, d_hash, d_keys, d_vals, mask,
                                                                    d_counters);
    note_launches(1);
    return cudaGetLastError();
}

// One thread per hit window: look its hash up, byte-compare every candidate pattern at the window start.
// The 16 bytes at p (any alignment), of which the first `need` (1..16) are used, read as aligned 16-byte
// loads: the chunk holding p, and the next one only when the bytes reach into it. An aligned chunk that holds a
// needed byte never crosses a page, so no load leaves the buffer's pages.
__device__ __forceinline__ uint4 load16_unaligned(const uint8_t* p, uint32_t need) {
    const uintptr_t a = (uintptr_t)p;
    const uint4* base = reinterpret_cast<const uint4*>(a & ~(uintptr_t)15);
    const uint32_t off = (uint32_t)(a & 15);
    const uint4 x0 = __ldg(base);
    const uint4 x1 = off + need > 16 ? __ldg(base + 1) : make_uint4(0, 0, 0, 0);
    const uint32_t ws = off >> 2, bs = (off & 3) * 8;
    // words ws .. ws + 4 of x0:x1, selected without a runtime-indexed array
    uint32_t w0, w1, w2, w3, w4;
    if (ws == 0) { w0 = x0.x; w1 = x0.y; w2 = x0.z; w3 = x0.w; w4 = x1.x; }
    else if (ws == 1) { w0 = x0.y; w1 = x0.z; w2 = x0.w; w3 = x1.x; w4 = x1.y; }
    else if (ws == 2) { w0 = x0.z; w1 = x0.w; w2 = x1.x; w3 = x1.y; w4 = x1.z; }
    else { w0 = x0.w; w1 = x1.x; w2 = x1.y; w3 = x1.z; w4 = x1.w; }
    return make_uint4(__funnelshift_r(w0, w1, bs), __funnelshift_r(w1, w2, bs), __funnelshift_r(w2, w3, bs),
                      __funnelshift_r(w3, w4, bs));
}

// mask of the bytes of 32-bit word i that fall within the first `need` bytes of a 16-byte block
__device__ __forceinline__ uint32_t word_mask(uint32_t need, uint32_t i) {
    const uint32_t v = need > 4 * i ? min(need - 4 * i, 4u) : 0u;
    return v >= 4 ? 0xffffffffu : (1u << (8 * v)) - 1u;
}

__global__ void k_verify(const HitRec* hits, uint32_t nhits, const uint8_t* text, uint64_t n, const uint64_t* keys,
                         const uint32_t* vals, uint64_t mask, const uint8_t* pat, const uint64_t* pstart,
                         const uint64_t* pend, uint64_t* m_off, uint32_t* m_pid, uint32_t cap, uint32_t* counters) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nhits) return;
    const uint64_t w = hits[j].off, h = hits[j].h;
    uint64_t slot = mix64(h) & mask;
    for (uint64_t probe = 0; probe <= mask; probe++) {
        uint32_t id = vals[slot];
        if (id == 0xffffffffu) break;
        if (keys[slot] == h) {
            uint64_t ps = pstart[id], pl = pend[id] - ps;
            if (w + pl <= n) {
                const uint8_t* t = text + w;
                const uint8_t* q = pat + ps;
                // byte compare, 16 bytes per step from aligned 16-byte loads of both sides
                bool same = true;
                for (uint64_t k = 0; k < pl && same; k += 16) {
                    const uint32_t need = pl - k < 16 ? (uint32_t)(pl - k) : 16u;
                    const uint4 x = load16_unaligned(t + k, need), y = load16_unaligned(q + k, need);
                    same = (((x.x ^ y.x) & word_mask(need, 0)) | ((x.y ^ y.y) & word_mask(need, 1)) |
                            ((x.z ^ y.z) & word_mask(need, 2)) | ((x.w ^ y.w) & word_mask(need, 3))) == 0;
                }
                if (same) {
                    uint32_t o = atomicAdd(counters + CNT_MATCHES, 1u);
                    if (o < cap) {
                        m_off[o] = w;
                        m_pid[o] = id;
                    }
                }
            }
        }
        slot = (slot + 1) & mask;
    }
}

cudaError_t verify_hits(const HitRec* hits, uint32_t nhits, const uint8_t* text, uint64_t n, const uint64_t* d_keys,
                        const uint32_t* d_vals, uint64_t mask, const uint8_t* d_pat, const uint64_t* d_start,
                        const uint64_t* d_end, uint64_t* d_match_off, uint32_t* d_match_pid, uint32_t match_cap,
                        uint32_t* d_counters, cudaStream_t st) {
    if (!nhits) return cudaSuccess;
    k_verify<<<(nhits + 255) / 256, 256, 0, st>>>(hits, nhits, text, n, d_keys, d_vals, mask, d_pat, d_start, d_end,
                                                   d_match_off, d_match_pid, match_cap, d_counters);
    note_launches(1);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// Filter cache file codec. loadFilterFromFile (ffbf.cpp:487-506) accumulates uint32 deltas (wrapping)
// and sets each running sum; saveFilterToFile (ffbf.cpp:508-527) writes the gaps between set bits.
constexpr int kCodecThreads = 256;
constexpr uint64_t kCodecChunk = 65536;

__global__ void __launch_bounds__(kCodecThreads) k_delta_block_sums(const uint32_t* d, uint64_t nd, uint32_t* sums) {
    __shared__ uint32_t sh[kCodecThreads / 32];
    uint64_t lo = blockIdx.x * kCodecChunk, hi = min(nd, lo + kCodecChunk);
    uint32_t s = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kCodecThreads) s += d[i];
    uint32_t tot;
    block_excl_scan<kCodecThreads>(s, sh, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kCodecThreads) k_delta_apply(const uint32_t* d, uint64_t nd, const uint32_t* offs,
                                                                uint32_t nbits, uint32_t* idx, uint32_t* counters) {
    __shared__ uint32_t sh[kCodecThreads / 32];
    constexpr int items = 16;
    uint64_t lo = blockIdx.x * kCodecChunk, hi = min(nd, lo + kCodecChunk);
    uint32_t base = offs[blockIdx.x];
    for (uint64_t r = lo; r < hi; r += (uint64_t)kCodecThreads * items) {
        uint64_t a = r + (uint64_t)threadIdx.x * items, b = min(hi, a + items);
        uint32_t s = 0;
        for (uint64_t i = a; i < b; i++) s += d[i];
        uint32_t tot;
        uint32_t run = base + block_excl_scan<kCodecThreads>(s, sh, &tot);
        for (uint64_t i = a; i < b; i++) {
            run += d[i];
            idx[i] = run;
            if (run >= nbits) atomicOr(counters + CNT_ERROR, 2u);
        }
        base += tot;
    }
}

cudaError_t filter_decode(const uint32_t* d_deltas, uint64_t nd, uint32_t nbits, uint32_t* d_idx, uint64_t* d_tmp,
                          uint32_t* d_counters, cudaStream_t st) {
    if (!nd) return cudaSuccess;
    uint64_t nb = (nd + kCodecChunk - 1) / kCodecChunk;
    uint32_t* sums = reinterpret_cast<uint32_t*>(d_tmp);
    k_delta_block_sums<<<(unsigned)nb, kCodecThreads, 0, st>>>(d_deltas, nd, sums);
    note_launches(1);
    k_scan_single<uint32_t><<<1, 1024, 0, st>>>(sums, nb);
    note_launches(1);
    k_delta_apply<<<(unsigned)nb, kCodecThreads, 0, st>>>(d_deltas, nd, sums, nbits, d_idx, d_counters);
    note_launches(1);
    return cudaGetLastError();
}

__global__ void k_set_indices(const uint32_t* idx, uint64_t nd, uint32_t* words) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= nd) return;
    uint32_t b = idx[i];
    atomicOr(words + (b >> 5), 1u << (b & 31));
}

cudaError_t filter_set_indices(const uint32_t* d_idx, uint64_t nd, uint32_t* d_main, cudaStream_t st) {
    if (!nd) return cudaSuccess;
    k_set_indices<<<(unsigned)((nd + 255) / 256), 256, 0, st>>>(d_idx, nd, d_main);
    note_launches(1);
    return cudaGetLastError();
}

// Encode: popcount per word chunk, scan, then emit ascending set-bit indices as deltas.
constexpr uint64_t kEncChunkWords = 16384;

__global__ void __launch_bounds__(kCodecThreads) k_popc_blocks(const uint32_t* w, uint32_t nwords, uint64_t* sums) {
    __shared__ uint64_t sh[kCodecThreads / 32];
    uint64_t lo = blockIdx.x * kEncChunkWords, hi = min((uint64_t)nwords, lo + kEncChunkWords);
    uint64_t s = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kCodecThreads) s += __popc(w[i]);
    uint64_t tot;
    block_excl_scan<kCodecThreads>(s, sh, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kCodecThreads) k_emit_bits(const uint32_t* w, uint32_t nwords, const uint64_t* offs,
                                                              uint32_t* out) {
    __shared__ uint64_t sh[kCodecThreads / 32];
    uint64_t lo = blockIdx.x * kEncChunkWords, hi = min((uint64_t)nwords, lo + kEncChunkWords);
    uint64_t base = offs[blockIdx.x];
    for (uint64_t r = lo; r < hi; r += kCodecThreads) {
        uint64_t i = r + threadIdx.x;
        uint32_t v = i < hi ? w[i] : 0u;
        uint64_t tot;
        uint64_t pos = base + block_excl_scan<kCodecThreads>((uint64_t)__popc(v), sh, &tot);
        while (v) {
            uint32_t b = __ffs(v) - 1;
            v &= v - 1;
            out[pos++] = (uint32_t)(i * 32 + b);
        }
        base += tot;
    }
}

__global__ void k_to_deltas(const uint32_t* idx, uint64_t n, uint32_t* out) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = idx[i] - (i ? idx[i - 1] : 0u);
}

uint64_t enc_blocks(uint32_t nwords) { return (nwords + kEncChunkWords - 1) / kEncChunkWords; }
uint64_t decode_blocks(uint64_t nd) { return (nd + kCodecChunk - 1) / kCodecChunk; }

cudaError_t filter_count(const uint32_t* d_main, uint32_t nwords, uint64_t* d_tmp, cudaStream_t st) {
    uint64_t nb = enc_blocks(nwords);
    k_popc_blocks<<<(unsigned)nb, kCodecThreads, 0, st>>>(d_main, nwords, d_tmp);
    note_launches(1);
    k_scan_single<uint64_t><<<1, 1024, 0, st>>>(d_tmp, nb);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t filter_encode(const uint32_t* d_main, uint32_t nwords, const uint64_t* d_tmp, uint32_t* d_idx,
                          cudaStream_t st) {
    uint64_t nb = enc_blocks(nwords);
    k_emit_bits<<<(unsigned)nb, kCodecThreads, 0, st>>>(d_main, nwords, d_tmp, d_idx);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t filter_deltas(const uint32_t* d_idx, uint64_t n, uint32_t* d_out, cudaStream_t st) {
    if (!n) return cudaSuccess;
    k_to_deltas<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_idx, n, d_out);
    note_launches(1);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// operator[] (ffbf.cpp:285-308): one string, no newline handling, first hitting window wins.
__global__ void k_test_line(const uint8_t* s, uint64_t n, Geom g, const uint32_t* main_words, uint32_t* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t res = 0;
    if (n >= g.len) {
        uint64_t h = 0;
        for (uint64_t p = 0; p < n && !res; p++) {
            h = rol64(h, 1) ^ sbox_of(s[p]);
            if (p >= g.len) h ^= rol64(sbox_of(s[p - g.len]), g.len);
            if (p + 1 >= g.len && check_all<1>(g, main_words, h)) res = 1;
        }
    }
    *out = res;
}

cudaError_t test_line(const uint8_t* d_line, uint64_t n, const Geom& g, const uint32_t* d_main, uint32_t* d_out,
                      cudaStream_t st) {
    k_test_line<<<1, 32, 0, st>>>(d_line, n, g, d_main, d_out);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace ffbf
