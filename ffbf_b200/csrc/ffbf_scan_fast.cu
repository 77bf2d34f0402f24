// ffbf_scan_fast.cu -- the tuned sm_100a scan of processFile (src/rabin-karp/ffbf.cpp:310-392).
//
// Work decomposition. The text is cut into streams of SLEN = rows * 128 bytes. A CTA of THREADS threads
// owns THREADS consecutive streams (a "supertile") at a time, one stream per thread, and walks them row by
// row. Each thread rolls the hash over its stream without restarting, so the LEN-byte warm-up is paid once
// per stream (from a 32-byte halo) instead of once per tile.
//
// Staging. Row r of the CTA's streams is loaded by TMA as 3-D boxes {128 bytes, 1 row, <=256 streams}
// (cp.async.bulk.tensor, 128B swizzle, one CTA per load) into a double-buffered shared-memory stage completed on
// an mbarrier. The 128B swizzle puts chunk c of thread t's row at chunk c ^ (t & 7), so the 16-byte reads
// of a quarter-warp hit eight different bank groups.
//
// Hash. h <- rol64(h,1) ^ S[in] ^ rol64(S[out], LEN) (hash_rot_sbox_pre_2.h:42-51 with the ring folded into
// the outgoing byte, still in registers), on two 32-bit halves. S sits in shared memory as 16 interleaved
// copies of 8-byte entries, so the 16 lanes of each half-warp read disjoint banks whatever their bytes. Bytes
// with the high bit set index entries that hold S[0] (ffbf.cpp:127-130).
//
// Probes. Stage 1 tests the first index function, h1 & (C-1), against a shared-memory table: the cache
// region itself when it fits, else its OR-summary (bit j = OR of cache bits [j<<sh, (j+1)<<sh)), which only
// rejects windows the full test rejects. A window that passes (and holds no '\n') is appended to its warp's
// candidate queue in shared memory; full queues and row ends are flushed by the whole warp, each lane taking
// queued candidates and running the full K-bit test on the global filter in the reference order
// (checkInFilter, ffbf.cpp:214-239). The queue keeps the per-byte path free of branches that wait on L2.
//
// Validity. A window is tested only when its LEN bytes hold no '\n' (processFile resets the hash at '\n').
// The last '\n' is tracked per thread; each stream's first and last '\n' feed the per-16 KiB-tile newline
// summaries the line resolver reads.
//
// Every mbarrier wait is bounded; on timeout the CTA records an error flag and stops.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "ffbf_scan_fast.cuh"

namespace ffbf {

namespace {

constexpr int kRowBytes = 128;
constexpr int kTabBytes = 256 * 16 * 8;  // 16 copies of the 256-entry S-box
constexpr int kQueueCap = 64;            // candidates per warp queue
constexpr int kQueueBytes = kQueueCap * 16;
constexpr uint32_t kWaitLimit = 1u << 24;
constexpr size_t kSmemLimit = 232448;    // opt-in shared memory per block on sm_100

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Waits for the phase of the given parity, at most kWaitLimit polls; false when it gave up.
__device__ __noinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity);

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

__device__ __noinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// The same load with an L2 cache policy (createpolicy): the text streams through L2 once.
__device__ __forceinline__ void tma_load_3d_hint(uint32_t dst, const CUtensorMap* map, int x, int y, int z,
                                                 uint32_t bar, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint "
        "[%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar), "l"(policy)
        : "memory");
}

__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Shared-memory loads of the read-only tables, which the compiler may schedule freely (a table is
// rewritten only between block barriers, at a change of job).
__device__ __forceinline__ uint2 lds64(uint32_t addr) {
    uint2 v;
    asm("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(addr));
    return v;
}
__device__ __forceinline__ uint32_t lds32(uint32_t addr) {
    uint32_t v;
    asm("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}

// Global load of one filter word when `pred` holds (0 otherwise); read-only path.
__device__ __forceinline__ uint32_t ldg_if(const uint32_t* p, bool pred) {
    uint32_t v;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\tmov.u32 %0, 0;\n\t@q ld.global.nc.u32 %0, [%1];\n\t}"
        : "=r"(v)
        : "l"(p), "r"((uint32_t)pred));
    return v;
}

// byte i (0..3) of w, zero-extended
__device__ __forceinline__ uint32_t byte_at(uint32_t w, int i) { return __byte_perm(w, 0u, 0x4440u + (uint32_t)i); }

// rol64 of (hi:lo) by N, 0 < N < 64, on 32-bit halves
template <int N>
__device__ __forceinline__ void rol_pair(uint32_t lo, uint32_t hi, uint32_t& rlo, uint32_t& rhi) {
    if constexpr (N == 32) {
        rlo = hi;
        rhi = lo;
    } else if constexpr (N < 32) {
        rlo = __funnelshift_l(hi, lo, N);
        rhi = __funnelshift_l(lo, hi, N);
    } else {
        rlo = __funnelshift_l(lo, hi, N - 32);
        rhi = __funnelshift_l(hi, lo, N - 32);
    }
}

// rol32 by a compile-time amount (0: identity)
template <int N>
__device__ __forceinline__ uint32_t rot_const(uint32_t x) {
    if constexpr (N == 0) return x;
    else return __funnelshift_l(x, x, N);
}

// Full test from probe FROM on (reference order, early exit); probes before FROM are known to be set.
__device__ __forceinline__ bool full_check_from(const Geom& g, const uint32_t* __restrict__ words, uint64_t h,
                                                uint32_t from) {
    for (uint32_t i = from; i < g.k; i++) {
        uint32_t b = bit_index<1>(g, h, i);
        if (!((__ldg(words + (b >> 5)) >> (b & 31)) & 1u)) return false;
    }
    return true;
}

// The whole warp drains its candidate queue: lane i takes entries i, i+32, ... (PER_LANE at most). An entry
// is {position | lane << 8, h1, h2, first}: probes before `first` are known to be set. Every lane issues the
// probe `first` of all its entries before testing any, so its L2 round trips overlap; survivors finish the
// test one by one.
template <int PER_LANE>
__device__ __noinline__ void flush_queue(const FastJob* J, uint32_t qaddr, int qn, uint64_t warp_row_pos0,
                                         uint64_t row_stride, int lane) {
    // the job's fields are read here rather than passed: the caller's loop keeps only its hot values live
    const Geom g = J->g;
    const uint32_t* __restrict__ main_words = J->main_words;
    uint32_t* ff_words = J->ff_words;
    HitRec* hits = J->hits;
    const uint32_t hits_cap = J->hits_cap;
    uint32_t* counters = J->counters;
    uint4 e[PER_LANE];
    uint32_t v[PER_LANE], bi[PER_LANE];
#pragma unroll
    for (int t = 0; t < PER_LANE; t++) {
        const int i = lane + 32 * t;
        e[t] = make_uint4(0, 0, 0, 0);
        v[t] = 0xffffffffu;
        bi[t] = 0;
        if (i < qn) {
            asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                         : "=r"(e[t].x), "=r"(e[t].y), "=r"(e[t].z), "=r"(e[t].w)
                         : "r"(qaddr + 16u * (uint32_t)i));
            if (e[t].w < g.k) {
                const uint64_t h = ((uint64_t)e[t].z << 32) | e[t].y;
                bi[t] = bit_index<1>(g, h, e[t].w);
                v[t] = __ldg(main_words + (bi[t] >> 5));
            }
        }
    }
#pragma unroll
    for (int t = 0; t < PER_LANE; t++) {
        const int i = lane + 32 * t;
        if (i >= qn) continue;
        const uint64_t h = ((uint64_t)e[t].z << 32) | e[t].y;
        if (!((v[t] >> (bi[t] & 31)) & 1u)) continue;
        if (!full_check_from(g, main_words, h, e[t].w + 1)) continue;
        // p = window end + 128 relative to the owner's current row (the dense rings carry the previous row's
        // last windows into the next row)
        const uint32_t owner = e[t].x >> 8, p = e[t].x & 0xFFu;
        if (owner >= 32) {
            atomicOr(counters + CNT_ERROR, 0x400u);
            continue;
        }
        const uint64_t start = warp_row_pos0 + owner * row_stride + p + 1 - g.len - kRowBytes;
        set_all<2>(g, ff_words, h);
        const uint32_t slot = atomicAdd(counters + CNT_HITS, 1u);
        if (slot < hits_cap) hits[slot] = HitRec{start, h};
    }
    __syncwarp();
}

// Work items. Job j owns items [item_begin_j, item_begin_{j+1}), one per supertile of THREADS streams; CTA b
// takes items b, b + gridDim.x, ... Each item is one TMA load of the streams' halo rows followed by `rows`
// row loads. Thread 0 issues load k+1 while the CTA consumes load k and records in meta[] which job, item
// and row each buffer holds.
//
// MODE 0 (sparse filters): stage 1 in shared memory, candidates queued per byte.
// MODE 1 (dense filters, where a shared-memory table would pass most windows): the exact probes of the
// first two index functions are global loads issued per valid window and consumed kRing bytes later from
// register rings, so L2 latency overlaps the hashing of the next windows; only windows whose two probed bits
// are set go to the queue.
// MODE 2: MODE 1 with the pipelined probes on index functions f2 = rot16(h1) and f3 = rot16(h2) (the
// external region for S <= 2, usually much sparser than the cache region, so fewer windows need a second
// probe); queued windows then run the whole K-bit test.
// MODE 3: MODE 1 with a shared-memory prefilter: the f0 load is issued only for windows whose bit in the
// folded cache region (the stage-1 table, sized for the room this kernel leaves) is set, so filters whose
// fold still rejects many windows issue that many fewer L2 probes.
// MODE 4 (sparse filters, deferred): MODE 0's two shared-memory probes, but the byte loop only shifts each
// window's pass bit into a 32-bit register mask; it carries no newline test and no warp vote, so a 32-byte
// block is one branch-free stretch of code. After the block, the block's newline mask (SWAR) gives each
// window's validity, and only when a lane of the warp holds a valid passing window is the hash of its 8-byte
// segment recomputed from a checkpoint, this time queueing the candidates as MODE 0 does. It pays where the
// stage-1 table rejects nearly every window (a large table: fewer threads per CTA).
template <int N>
__device__ __forceinline__ void shl64_or(uint32_t& lo, uint32_t& hi) {
    // (hi:lo) |= (hi:lo) << N, 0 < N < 32
    hi |= __funnelshift_l(lo, hi, N);
    lo |= lo << N;
}

// Bit j set when the window of L bytes ending at byte j of a 32-byte block holds a '\n'. `prev` and `cur`
// are the newline masks (bit i = byte i is '\n') of the previous block and of this one.
template <int L>
__device__ __forceinline__ uint32_t window_has_newline(uint32_t prev, uint32_t cur) {
    static_assert(L >= 1 && L <= 32, "windows reach back at most one block");
    // OR of (cur:prev) << k for k in [0, L), high word: (cur:prev) << k covers [0, w) after the doubling
    // steps below; the set bits of L add shifted copies of it
    uint32_t lo = prev, hi = cur;
    uint32_t rhi = 0;
    int covered = 0;
#pragma unroll
    for (int m = 0; m < 6; m++) {
        const int w = 1 << m;
        if (L & w) {
            if (covered == 0) rhi |= hi;
            else if (covered < 32) rhi |= __funnelshift_l(lo, hi, covered);
            else rhi |= lo << (covered - 32);
            covered += w;
        }
        if (2 * w <= L) {
            switch (w) {
                case 1: shl64_or<1>(lo, hi); break;
                case 2: shl64_or<2>(lo, hi); break;
                case 4: shl64_or<4>(lo, hi); break;
                case 8: shl64_or<8>(lo, hi); break;
                case 16: shl64_or<16>(lo, hi); break;
                default: break;
            }
        }
    }
    return rhi;
}

// Newline mask of 4 text bytes: bit k set when byte k of w is '\n' (exact per byte).
__device__ __forceinline__ uint32_t newline_bits4(uint32_t w) {
    const uint32_t t = w ^ 0x0A0A0A0Au;
    const uint32_t zb = ~(((t & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | t) & 0x80808080u;
    return (zb * 0x00204081u) >> 28;  // bits 7, 15, 23, 31 -> 28..31, without carries
}

__device__ __forceinline__ uint32_t newline_mask32(const uint32_t (&w)[8]) {
    uint32_t m = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) m |= newline_bits4(w[q]) << (4 * q);
    return m;
}

// CTAs per SM: the dense modes at 192 threads run two CTAs per SM (12 warps, as one 384-thread CTA, but two
// independent pipelines and barriers of 6 warps each); every other configuration runs one.
__host__ __device__ constexpr int ctas_per_sm(int threads, int mode) { return threads == 192 && mode >= 1 && mode <= 3 ? 2 : 1; }
// MODE 5 is MODE 0 whose warps meet through per-stage barriers instead of a block barrier per stage
__host__ __device__ constexpr bool sparse_mode(int mode) { return mode == 0 || mode == 5; }

template <int L, int THREADS, int MODE>
__global__ void __launch_bounds__(THREADS, ctas_per_sm(THREADS, MODE)) k_scan_fast(const FastJob* __restrict__ jobs, uint32_t n_jobs,
                                                          uint32_t n_items, uint32_t max_s1_words,
                                                          uint32_t* __restrict__ ctl) {
    // ctl[0]: error flags; ctl[1]: the work queue, the count of items handed out past the first wave
    uint32_t* const error_flag = ctl;
    constexpr int kStageBytes = THREADS * kRowBytes;
    constexpr int kQCap = (sparse_mode(MODE) || MODE == 4) ? kQueueCap : 2 * kQueueCap;
    constexpr int kQBytes = kQCap * 16;
    // dense mode: ring depth per stage (divides 32); 384-thread CTAs trade depth for warps (more L2 probes
    // in flight per SM within the register file)
    constexpr int kRing = THREADS >= 384 || ctas_per_sm(THREADS, MODE) == 2 ? 4 : 8;
    constexpr int kBox = THREADS > 256 ? THREADS / 2 : THREADS;  // streams per TMA box (<= 256)
    constexpr bool kTable = sparse_mode(MODE) || MODE == 3 || MODE == 4;  // reads the stage-1 table
    constexpr bool kSparse = sparse_mode(MODE);
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* smem = smem_raw + (base - raw);
    // layout: [stage 0][stage 1][S tables][mbarriers, meta (128 B)][warp queues][stage-1 table]
    const uint32_t stage0 = base;
    const uint32_t tab = base + 2 * kStageBytes;
    const uint32_t bar0 = tab + kTabBytes, bar1 = bar0 + 8;
    // Stage k & 1's "full" barrier completes when load k lands. With kStageBarriers (MODE 5) its "empty"
    // barrier completes when every warp is done reading it, load k + 2 reuses the stage only after that, and
    // warps otherwise run apart by up to a stage. It pays where few windows pass the shared-memory stage
    // (plain workload: 596 -> 630 GB/s); where many do, warps that wait for the stage of a warp busy with
    // its queue cost more than a block barrier (a 2^22-bit batched class: 370 -> 306), and in the dense
    // modes too (325 -> 308). The other modes keep one block barrier per stage.
    constexpr bool kStageBarriers = MODE == 5;
    auto ebar = [&](uint32_t k) { return bar0 + 48u + 8u * (k & 1u); };
    int* meta = reinterpret_cast<int*>(smem + 2 * kStageBytes + kTabBytes + 16);  // [buf][4]: job, item, row, valid
    const uint32_t queues = bar0 + 128;
    const uint32_t s1 = queues + (THREADS / 32) * kQBytes;
    uint32_t* s1p = reinterpret_cast<uint32_t*>(smem + (s1 - base));
    // Per-CTA state kept in shared memory rather than registers, which the dense mode's rings need:
    // the load sequencer (thread 0 only), each warp's first text position of its current row, each
    // thread's first and last '\n' so far in its stream.
    __shared__ int s_abort;
    __shared__ uint32_t s_ni, s_nj;
    __shared__ int s_nr;
    __shared__ uint64_t s_wpos[THREADS / 32];
    __shared__ long long s_fnl[THREADS], s_lnl[THREADS];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        uint64_t* tp = reinterpret_cast<uint64_t*>(smem + 2 * kStageBytes);
        for (int i = tid; i < 256 * 16; i += THREADS) {
            const int c = i >> 4;
            tp[i] = c_sbox[(c & 0x80) ? 0 : c];
        }
    }
    // load sequencer, run by thread 0: the next load is row nr (-1: halo) of item ni, which belongs to job nj.
    // Load k waits (bounded) until every warp has released load k - 2's stage; with no item left it completes
    // the stage's full barrier without a load and marks the end in meta. Returns false when the wait gave up.
    auto issue = [&](uint32_t k) -> bool {
        if constexpr (kStageBarriers) {
            if (k >= 2 && !mbar_wait_bounded(ebar(k), ((k - 2) >> 1) & 1u)) {
                atomicOr(error_flag, 4u);
                return false;
            }
        }
        int* m = meta + 4 * (k & 1);
        uint32_t ni = s_ni, nj = s_nj;
        int nr = s_nr;
        if (ni >= n_items) {
            m[3] = 0;
            if constexpr (kStageBarriers) mbar_arrive((k & 1) ? bar1 : bar0);
            return true;
        }
        while (nj + 1 < n_jobs && __ldg(&jobs[nj + 1].item_begin) <= ni) nj++;
        const FastJob* J = jobs + nj;
        const uint32_t R = __ldg(&J->rows);
        const uint32_t st = ni - __ldg(&J->item_begin);
        const int y = nr < 0 ? (int)R - 1 : nr;
        const int z = (int)(st * THREADS) + (nr < 0 ? -1 : 0);
        const uint32_t bar = (k & 1) ? bar1 : bar0;
        const uint32_t dst = stage0 + (k & 1) * kStageBytes;
        m[0] = (int)nj;
        m[1] = (int)st;
        m[2] = nr;
        m[3] = 1;
        mbar_expect_tx(bar, kStageBytes);
        if (__ldg(&J->text_evict_first)) {
            const uint64_t pol = l2_evict_first_policy();
            for (int b = 0; b < THREADS / kBox; b++)
                tma_load_3d_hint(dst + b * kBox * kRowBytes, &J->tmap, 0, y, z + b * kBox, bar, pol);
        } else {
            for (int b = 0; b < THREADS / kBox; b++)
                tma_load_3d(dst + b * kBox * kRowBytes, &J->tmap, 0, y, z + b * kBox, bar);
        }
        if (++nr == (int)R) {
            nr = -1;
            ni = gridDim.x + atomicAdd(ctl + 1, 1u);  // next item from the queue
        }
        s_ni = ni;
        s_nj = nj;
        s_nr = nr;
        return true;
    };
    if (tid == 0) {
        s_abort = 0;
        s_ni = blockIdx.x;
        s_nj = 0;
        s_nr = -1;
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        if constexpr (kStageBarriers) {
            mbar_init(ebar(0), THREADS / 32);
            mbar_init(ebar(1), THREADS / 32);
        }
        *reinterpret_cast<uint32_t*>(smem + (bar0 - base) + 64) = 0xFFFFFFFFu;  // the S = 1 second-probe word
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        // publication gate: a bounded poll, and no load in flight if it gives up
        bool open = true;
        if (const uint32_t* rw = jobs[0].ready) {
            const uint32_t spins = jobs[0].ready_spins;
            for (uint32_t i = 0;; i++) {
                if (*reinterpret_cast<const volatile uint32_t*>(rw) != 0u) break;
                if (i >= spins) {
                    atomicOr(error_flag, 4u);
                    open = false;
                    break;
                }
                __nanosleep(1000);
            }
        }
        if (open) {
            issue(0);
        } else {
            meta[3] = 0;
            if constexpr (kStageBarriers) mbar_arrive(bar0);
        }
    }
    __syncthreads();

    const uint32_t lane_tab = tab + (uint32_t)(lane & 15) * 8u;  // entry c of this lane's copy: + c * 128
    const uint32_t qaddr = queues + (uint32_t)warp * kQBytes;
    const unsigned lt_mask = (1u << lane) - 1u;

    // the current job's parameters (reloaded when the job changes)
    int cur_job = -1;
    uint32_t R = 0, s1_bmask = 0, s1_first = 0, spt_log2 = 0;
    uint32_t a_mask = 0, a_add = 0, b_mask = 0, b_add = 0;  // dense mode: regions of the two pipelined probes
    bool two = false;
    auto job_desc = [&]() { return jobs + cur_job; };
    // The filter pointer is held in a register: the loop's global stores would otherwise make the compiler
    // reload it from the descriptor before every probe. Fields used once per row or per queue flush are
    // read from the descriptor where they are used, so they hold no registers across the byte loop.
    const uint32_t* main_words = nullptr;
    bool s1_fits = true;

    int qn = 0;  // warp-uniform queue fill
    // Appends the lanes with `pass` to the warp queue; flushes when fewer than 32 slots remain.
    auto enqueue = [&](bool pass, uint32_t pos, uint32_t ql, uint32_t qh, uint32_t first) {
        const unsigned m = __ballot_sync(0xffffffffu, pass);
        if (m) {
            if (pass) {
                // qn <= kQCap - 32 holds on entry (the queue flushes above that), so slot < kQCap
                const uint32_t slot = (uint32_t)qn + __popc(m & lt_mask);
                asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(qaddr + 16u * slot),
                             "r"(pos | ((uint32_t)lane << 8)), "r"(ql), "r"(qh), "r"(first)
                             : "memory");
            }
            qn += __popc(m);
            if (qn > kQCap - 32) {
                __syncwarp();
                flush_queue<kQCap / 32>(job_desc(), qaddr, qn, s_wpos[warp], (uint64_t)R * kRowBytes, lane);
                qn = 0;
            }
        }
    };
    // dense-mode rings. Stage A: the first probe's word (0 when the window was not valid, so its test fails),
    // h1, h2. Stage B: the second probe's word (0 when stage A failed), h1, h2.
    constexpr int kR = (MODE == 1 || MODE == 2 || MODE == 3) ? kRing : 1;
    // dense mode: rotation of h1/h2 giving the pipelined probes' index functions, and the first probe a
    // queued window still needs in the reference order (MODE 1 knows f0 and f1; MODE 2 retests all)
    constexpr int kRot = MODE == 2 ? 16 : 0;
    constexpr uint32_t kFirstB = MODE == 2 ? 0u : 2u, kFirstA = MODE == 2 ? 0u : 1u;
    uint32_t ring_v[kR], ring_l[kR], ring_h[kR], ring2_v[kR], ring2_l[kR], ring2_h[kR];
#pragma unroll
    for (int q = 0; q < kR; q++) ring_v[q] = ring_l[q] = ring_h[q] = ring2_v[q] = ring2_l[q] = ring2_h[q] = 0;

    uint32_t hl = 0, hh = 0;
    int lnp = -1000;  // last '\n' relative to the current row start
    uint32_t prev[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // MODE 4: newline mask of the previous block (bit 31 forced at the text's start, where nothing precedes
    // offset 0). MODE 0 and 4: the second probe's table (the stage-1 table, or with S = 1 a word of ones)
    uint32_t nl_prev = 0;
    uint32_t s2 = s1, s2_bmask = 0;

    for (uint32_t k = 0;; k++) {
        const uint32_t bar = (k & 1) ? bar1 : bar0;
        const uint32_t parity = (k >> 1) & 1u;
        int job, r;
        uint32_t st;
        if constexpr (kStageBarriers) {
            // Warps meet only through the stages' barriers: a warp may start stage k + 1 while others still
            // read stage k, and thread 0 refills a stage once every warp has released it.
            uint32_t it = 0;
            while (!mbar_try_wait(bar, parity)) {
                if (++it >= kWaitLimit) {
                    atomicOr(error_flag, 4u);
                    s_abort = 1;
                    break;
                }
            }
            if (s_abort) {
                // Give a load still in flight a bounded chance to land before the shared memory goes away.
                if (tid == 0 && meta[4 * (k & 1) + 3])
                    for (uint32_t j = 0; j < kWaitLimit && !mbar_try_wait(bar, parity); j++) {
                    }
                break;
            }
            // the stage's meta is written before its full barrier completes, so it is read after the wait
            const int* m = meta + 4 * (k & 1);
            if (!m[3]) break;
            job = m[0];
            st = (uint32_t)m[1];
            r = m[2];
            if (tid == 0 && !issue(k + 1)) s_abort = 1;
        } else {
            // meta of stage k was written before the previous stage's block barrier
            const int* m = meta + 4 * (k & 1);
            if (!m[3]) break;
            job = m[0];
            st = (uint32_t)m[1];
            r = m[2];
            if (tid == 0) issue(k + 1);
            uint32_t it = 0;
            while (!mbar_try_wait(bar, parity)) {
                if (++it >= kWaitLimit) {
                    atomicOr(error_flag, 4u);
                    s_abort = 1;
                    break;
                }
            }
            if (s_abort) {
                // Give the load issued for k + 1 a bounded chance to land before the shared memory goes away.
                if (tid == 0 && meta[4 * ((k + 1) & 1) + 3]) {
                    const uint32_t nb = ((k + 1) & 1) ? bar1 : bar0;
                    for (uint32_t j = 0; j < kWaitLimit && !mbar_try_wait(nb, ((k + 1) >> 1) & 1u); j++) {
                    }
                }
                break;
            }
        }
        if (job != cur_job) {
            cur_job = job;
            const FastJob* J = job_desc();
            const Geom g = J->g;
            R = J->rows;
            spt_log2 = J->streams_per_tile_log2;
            main_words = J->main_words;
            s1_fits = !kTable || J->stage1_nwords <= max_s1_words;
            const uint32_t cmask = g.cache_mask;
            two = g.s > 1;
            // stage-1 table of T = C >> shift bits, folded modulo T: the byte offset of bit (h & (T-1))'s
            // word is (h >> 3) & s1_bmask
            s1_bmask = (((cmask >> J->stage1_shift) >> 3) & ~3u);
            a_mask = J->a_mask;
            a_add = J->a_add;
            b_mask = J->b_mask;
            b_add = J->b_add;
            // sparse mode: the stage-1 probes are exact when the table is the cache region itself
            s1_first = J->stage1_shift == 0 ? (two ? 2u : 1u) : 0u;
            s2 = two ? s1 : bar0 + 64;
            s2_bmask = two ? s1_bmask : 0u;
            if constexpr (kTable) {
                // every warp is done with the previous job's table before it is overwritten (all warps change
                // job at the same stage)
                if constexpr (kStageBarriers) __syncthreads();
                const uint32_t nw = s1_fits ? J->stage1_nwords : 0u;
                const uint32_t* src = J->stage1_words;
                for (uint32_t i = tid; i < nw; i += THREADS) s1p[i] = src[i];
                __syncthreads();
            }
        }

        // self-checks: a bad descriptor or sequencing records a code and skips the work
        if ((uint32_t)job >= n_jobs || st >= job_desc()->n_supertiles || r < -1 || r >= (int)R || !s1_fits) {
            if (tid == 0) atomicOr(error_flag, 0x100u);
            if constexpr (kStageBarriers) {
                __syncwarp();
                if (lane == 0) mbar_arrive(ebar(k));
            } else {
                __syncthreads();
            }
            continue;
        }
        const uint64_t z = (uint64_t)st * THREADS + tid;
        const bool active = z < job_desc()->n_streams;
        const uint8_t* row = smem + (k & 1) * kStageBytes + tid * kRowBytes;
        const int sw = tid & 7;

        if (r < 0) {
            // halo: the last 32 bytes before the stream (chunks 6 and 7 of the previous stream's last row)
            const uint4 c6 = *reinterpret_cast<const uint4*>(row + ((6 ^ sw) << 4));
            const uint4 c7 = *reinterpret_cast<const uint4*>(row + ((7 ^ sw) << 4));
            prev[0] = c6.x; prev[1] = c6.y; prev[2] = c6.z; prev[3] = c6.w;
            prev[4] = c7.x; prev[5] = c7.y; prev[6] = c7.z; prev[7] = c7.w;
            hl = 0;
            hh = 0;
            lnp = -1000;
#pragma unroll
            for (int j = 0; j < 32; j++) {
                const uint32_t c = byte_at(prev[j >> 2], j & 3);
                const uint2 sv = lds64(lane_tab + c * 128u);
                uint32_t nl = __funnelshift_l(hh, hl, 1), nh = __funnelshift_l(hl, hh, 1);
                nl ^= sv.x;
                nh ^= sv.y;
                if (j >= L) {
                    const uint32_t co = byte_at(prev[(j - L) >> 2], (j - L) & 3);
                    const uint2 o = lds64(lane_tab + co * 128u);
                    uint32_t rl, rh;
                    rol_pair<L>(o.x, o.y, rl, rh);
                    nl ^= rl;
                    nh ^= rh;
                }
                hl = nl;
                hh = nh;
                if (c == 0x0Au) lnp = j - 32;
            }
            if (z == 0) lnp = -1;  // text start: nothing before offset 0
            if constexpr (MODE == 4) nl_prev = newline_mask32(prev) | (z == 0 ? 0x80000000u : 0u);
            s_fnl[tid] = LLONG_MAX;
            s_lnl[tid] = -1;
        } else {
            // A stream past the job's end reads zero-filled rows (no '\n'): a last newline far ahead keeps all
            // its windows invalid, so the byte loop needs no separate `active` test.
            if (!active) lnp = 1 << 29;
            const int lnp_in = lnp;
            qn = 0;
            if (lane == 0)
                s_wpos[warp] = ((uint64_t)st * THREADS + (uint64_t)warp * 32) * R * kRowBytes + (uint64_t)r * kRowBytes;
            const bool need_first = s_fnl[tid] == LLONG_MAX;
            int row_first = -1;  // first '\n' of this row, found once per stream
#pragma unroll 1
            for (int b = 0; b < kRowBytes / 32; b++) {
                uint32_t cur[8];
                {
                    const uint4 v0 = *reinterpret_cast<const uint4*>(row + (((2 * b) ^ sw) << 4));
                    const uint4 v1 = *reinterpret_cast<const uint4*>(row + (((2 * b + 1) ^ sw) << 4));
                    cur[0] = v0.x; cur[1] = v0.y; cur[2] = v0.z; cur[3] = v0.w;
                    cur[4] = v1.x; cur[5] = v1.y; cur[6] = v1.z; cur[7] = v1.w;
                }
                const int lnp_blk = lnp;
                if constexpr (MODE == 4) {
                    // pass bits of the block's windows (bit j: the window ending at byte j passed both table
                    // probes), and the hash before each 8-byte segment
                    uint32_t pass = 0, ckl[4], ckh[4];
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        if ((j & 7) == 0) {
                            ckl[j >> 3] = hl;
                            ckh[j >> 3] = hh;
                        }
                        const uint32_t c = byte_at(cur[j >> 2], j & 3);
                        uint32_t co;
                        if (j >= L) co = byte_at(cur[(j - L) >> 2], (j - L) & 3);
                        else co = byte_at(prev[(j - L + 32) >> 2], (j - L + 32) & 3);
                        const uint2 sv = lds64(lane_tab + c * 128u);
                        const uint2 o = lds64(lane_tab + co * 128u);
                        uint32_t rl, rh;
                        rol_pair<L>(o.x, o.y, rl, rh);
                        const uint32_t nl = __funnelshift_l(hh, hl, 1), nh = __funnelshift_l(hl, hh, 1);
                        hl = nl ^ sv.x ^ rl;
                        hh = nh ^ sv.y ^ rh;
                        const uint32_t w0 = lds32(s1 + ((hl >> 3) & s1_bmask));
                        const uint32_t w1 = lds32(s2 + ((hh >> 3) & s2_bmask));
                        const uint32_t t = __funnelshift_r(w0, w0, hl) & __funnelshift_r(w1, w1, hh);
                        pass = __funnelshift_r(pass, t, 1);  // t's bit 0 enters at bit 31
                    }
                    const uint32_t nlm = newline_mask32(cur);
                    if (__any_sync(0xffffffffu, pass != 0u)) {
                        // valid windows hold no '\n' (processFile resets the hash there); a stream past the
                        // job's end has none
                        const uint32_t cand = active ? pass & ~window_has_newline<L>(nl_prev, nlm) : 0u;
#pragma unroll
                        for (int sg = 0; sg < 4; sg++) {
                            if (__any_sync(0xffffffffu, ((cand >> (8 * sg)) & 0xFFu) != 0u)) {
                                uint32_t ql = ckl[sg], qh = ckh[sg];
#pragma unroll
                                for (int jj = 0; jj < 8; jj++) {
                                    const int j = 8 * sg + jj;
                                    const uint32_t c = byte_at(cur[j >> 2], j & 3);
                                    uint32_t co;
                                    if (j >= L) co = byte_at(cur[(j - L) >> 2], (j - L) & 3);
                                    else co = byte_at(prev[(j - L + 32) >> 2], (j - L + 32) & 3);
                                    const uint2 sv = lds64(lane_tab + c * 128u);
                                    const uint2 o = lds64(lane_tab + co * 128u);
                                    uint32_t rl, rh;
                                    rol_pair<L>(o.x, o.y, rl, rh);
                                    const uint32_t nl = __funnelshift_l(qh, ql, 1), nh = __funnelshift_l(ql, qh, 1);
                                    ql = nl ^ sv.x ^ rl;
                                    qh = nh ^ sv.y ^ rh;
                                    enqueue(((cand >> j) & 1u) != 0u, (uint32_t)(kRowBytes + 32 * b + j), ql, qh,
                                            s1_first);
                                }
                            }
                        }
                    }
                    nl_prev = nlm;
                    if (nlm) {
                        lnp = 31 - __clz(nlm);
                        if (row_first < 0 && need_first) row_first = 32 * b + __ffs(nlm) - 1;
                    }
                } else {
                    // MODE 0 tests each window one byte late: the table words of byte j are loaded, then byte
                    // j - 1's (loaded a byte earlier) are tested and queued, so the shared-memory latency of a
                    // byte's probes overlaps the next byte's hash instead of stalling before its warp vote
                    uint32_t pw0 = 0, pw1 = 0, pl = 0, ph = 0;
                    bool pv = false;
                    // S-box entries of byte j's incoming and outgoing bytes; MODE 0 loads them a byte ahead
                    auto sbox_in = [&](int j) { return lds64(lane_tab + byte_at(cur[j >> 2], j & 3) * 128u); };
                    auto sbox_out = [&](int j) {
                        const uint32_t co = j >= L ? byte_at(cur[(j - L) >> 2], (j - L) & 3)
                                                   : byte_at(prev[(j - L + 32) >> 2], (j - L + 32) & 3);
                        return lds64(lane_tab + co * 128u);
                    };
                    uint2 nsv = make_uint2(0, 0), no = make_uint2(0, 0);
                    if constexpr (kSparse) {
                        nsv = sbox_in(0);
                        no = sbox_out(0);
                    }
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        const uint32_t c = byte_at(cur[j >> 2], j & 3);
                        uint2 sv, o;
                        if constexpr (kSparse) {
                            sv = nsv;
                            o = no;
                            if (j + 1 < 32) {
                                nsv = sbox_in(j + 1);
                                no = sbox_out(j + 1);
                            }
                        } else {
                            sv = sbox_in(j);
                            o = sbox_out(j);
                        }
                        uint32_t rl, rh;
                        rol_pair<L>(o.x, o.y, rl, rh);
                        const uint32_t nl = __funnelshift_l(hh, hl, 1), nh = __funnelshift_l(hl, hh, 1);
                        hl = nl ^ sv.x ^ rl;
                        hh = nh ^ sv.y ^ rh;
                        if (c == 0x0Au) lnp = j;
                        if constexpr (kSparse) {
                            // with S = 1 the second probe reads a word of ones
                            const uint32_t w0 = lds32(s1 + ((hl >> 3) & s1_bmask));
                            const uint32_t w1 = lds32(s2 + ((hh >> 3) & s2_bmask));
                            const bool valid = j - lnp >= L;
                            if (j > 0) {
                                const uint32_t t = __funnelshift_r(pw0, pw0, pl) & __funnelshift_r(pw1, pw1, ph);
                                enqueue(pv && (t & 1u) != 0, (uint32_t)(kRowBytes + 32 * b + j - 1), pl, ph, s1_first);
                            }
                            pw0 = w0;
                            pw1 = w1;
                            pl = hl;
                            ph = hh;
                            pv = valid;
                        } else {
                            const int slot = j % kRing;
                            // stage B: the window that entered stage A 2*kRing bytes ago (a probe's bit sits at
                            // f & 31 in its word: region offsets are multiples of 32)
                            const uint32_t fb_old = rot_const<kRot>(ring2_h[slot]);
                            const bool pass2 = (__funnelshift_r(ring2_v[slot], ring2_v[slot], fb_old) & 1u) != 0;
                            enqueue(pass2, (uint32_t)(kRowBytes + 32 * b + j - 2 * kRing), ring2_l[slot], ring2_h[slot],
                                    kFirstB);
                            // stage A: the window issued kRing bytes ago; its word has arrived by now
                            const uint32_t fa_old = rot_const<kRot>(ring_l[slot]);
                            const bool pass1 = (__funnelshift_r(ring_v[slot], ring_v[slot], fa_old) & 1u) != 0;
                            ring2_l[slot] = ring_l[slot];
                            ring2_h[slot] = ring_h[slot];
                            const uint32_t fb = rot_const<kRot>(ring_h[slot]);
                            ring2_v[slot] = ldg_if(main_words + (((fb & b_mask) + b_add) >> 5), pass1);
                            bool issue = j - lnp >= L;
                            if constexpr (MODE == 3) {
                                // the folded table's bit: clear means the cache bit of f0 is clear too
                                const uint32_t w = lds32(s1 + ((hl >> 3) & s1_bmask));
                                issue = issue && (__funnelshift_r(w, w, hl) & 1u) != 0;
                            }
                            ring_l[slot] = hl;
                            ring_h[slot] = hh;
                            const uint32_t fa = rot_const<kRot>(hl);
                            if constexpr (MODE != 2)  // f0 is in the cache region (S >= 1): no offset
                                ring_v[slot] = ldg_if(main_words + ((fa & a_mask) >> 5), issue);
                            else
                                ring_v[slot] = ldg_if(main_words + (((fa & a_mask) + a_add) >> 5), issue);
                        }
                    }
                    if constexpr (kSparse) {  // the block's last window
                        const uint32_t t = __funnelshift_r(pw0, pw0, pl) & __funnelshift_r(pw1, pw1, ph);
                        enqueue(pv && (t & 1u) != 0, (uint32_t)(kRowBytes + 32 * b + 31), pl, ph, s1_first);
                    }
                }
                if (MODE != 4 && lnp != lnp_blk && row_first < 0 && need_first) {
                    for (int q = 0; q < 8 && row_first < 0; q++) {
                        const uint32_t t = cur[q] ^ 0x0A0A0A0Au;
                        const uint32_t zb = ~(((t & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | t) & 0x80808080u;
                        if (zb) row_first = 32 * b + 4 * q + (__ffs(zb) - 1) / 8;
                    }
                }
                lnp -= 32;
#pragma unroll
                for (int q = 0; q < 8; q++) prev[q] = cur[q];
            }
            if constexpr (MODE == 1 || MODE == 2 || MODE == 3) {
                // The rings carry over into the stream's next row (whose bytes follow this row's); at the
                // stream's end they drain: stage-B slot q holds the window ending at 128 - 2*kRing + q,
                // stage-A slot q the one at 128 - kRing + q; stage-A survivors go to the queue with only
                // their first probe known.
                if ((uint32_t)r == R - 1) {
#pragma unroll
                    for (int q = 0; q < kRing; q++) {
                        const uint32_t fb = rot_const<kRot>(ring2_h[q]);
                        const bool pass2 = (__funnelshift_r(ring2_v[q], ring2_v[q], fb) & 1u) != 0;
                        enqueue(pass2, (uint32_t)(2 * kRowBytes - 2 * kRing + q), ring2_l[q], ring2_h[q], kFirstB);
                        const uint32_t fa = rot_const<kRot>(ring_l[q]);
                        const bool pass1 = (__funnelshift_r(ring_v[q], ring_v[q], fa) & 1u) != 0;
                        enqueue(pass1, (uint32_t)(2 * kRowBytes - kRing + q), ring_l[q], ring_h[q], kFirstA);
                        ring_v[q] = 0;
                        ring2_v[q] = 0;
                    }
                }
            }
            if (qn) {
                __syncwarp();
                flush_queue<kQCap / 32>(job_desc(), qaddr, qn, s_wpos[warp], (uint64_t)R * kRowBytes, lane);
                qn = 0;
            }
            // lnp is now relative to the next row's start; lnp + 128 is its position in this row
            if (active && lnp + kRowBytes != lnp_in) {
                const long long row_pos = (long long)(z * R + (uint32_t)r) * kRowBytes;
                if (need_first) s_fnl[tid] = row_pos + row_first;
                s_lnl[tid] = row_pos + lnp + kRowBytes;
            }
            if ((uint32_t)r == R - 1) {
                // per-16 KiB-tile newline summary: reduce over the lanes whose streams share the tile
                long long f = active ? s_fnl[tid] : LLONG_MAX, l = active ? s_lnl[tid] : -1;
                const int G = 1 << spt_log2;
                for (int o = 1; o < G; o <<= 1) {
                    f = min(f, __shfl_xor_sync(0xffffffffu, f, o));
                    l = max(l, __shfl_xor_sync(0xffffffffu, l, o));
                }
                if (active && (lane & (G - 1)) == 0) {
                    const uint64_t tile = z >> spt_log2;
                    const FastJob* J = job_desc();
                    if (tile < J->n_tiles) {
                        J->tile_first_nl[tile] = f;
                        J->tile_last_nl[tile] = l;
                    } else {
                        atomicOr(error_flag, 0x200u);
                    }
                }
            }
        }
        if constexpr (kStageBarriers) {
            // this warp is done reading the stage
            __syncwarp();
            if (lane == 0) mbar_arrive(ebar(k));
        } else {
            __syncthreads();
        }
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

// static shared memory of k_scan_fast<., THREADS, .> (sequencer, row positions, per-thread newline state)
constexpr size_t static_smem(int threads) { return 16 * (size_t)threads + 8 * (size_t)(threads / 32) + 64; }

template <int THREADS, int MODE>
constexpr size_t fixed_smem() {
    return 1024 + 2 * (size_t)THREADS * kRowBytes + kTabBytes + 128 +
           (THREADS / 32) * (size_t)(sparse_mode(MODE) || MODE == 4 ? kQueueBytes : 2 * kQueueBytes);
}

template <int L, int THREADS, int MODE>
cudaError_t launch_cfg(const FastJob* d_jobs, uint32_t n_jobs, uint32_t n_items, uint32_t max_s1_words,
                       uint32_t* d_ctl, int num_sms, cudaStream_t st) {
    const size_t smem =
        fixed_smem<THREADS, MODE>() + (sparse_mode(MODE) || MODE == 3 || MODE == 4 ? 4 * (size_t)max_s1_words : 0);
    cudaError_t e =
        cudaFuncSetAttribute(k_scan_fast<L, THREADS, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint32_t slots = (uint32_t)num_sms * (uint32_t)ctas_per_sm(THREADS, MODE);
    const int grid = (int)(n_items < slots ? n_items : slots);
    if (grid == 0) return cudaSuccess;
    k_scan_fast<L, THREADS, MODE><<<grid, THREADS, smem, st>>>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl);
    note_launches(1);
    return cudaGetLastError();
}

template <int L>
cudaError_t launch_len(const FastConfig& cfg, const FastJob* d_jobs, uint32_t n_jobs, uint32_t n_items,
                       uint32_t max_s1_words, uint32_t* d_ctl, int num_sms, cudaStream_t st) {
    if (cfg.mode == 1) {  // dense: 384 threads (ring depth 4), 256 (depth 8) or 2 x 192 (depth 4); 512 would spill
        if (cfg.threads == 192 && cfg.order != 2)
            return cfg.order == 1 ? launch_cfg<L, 192, 2>(d_jobs, n_jobs, n_items, 0, d_ctl, num_sms, st)
                                  : launch_cfg<L, 192, 1>(d_jobs, n_jobs, n_items, 0, d_ctl, num_sms, st);
        if (cfg.order == 1)
            return cfg.threads == 256 ? launch_cfg<L, 256, 2>(d_jobs, n_jobs, n_items, 0, d_ctl, num_sms, st)
                                      : launch_cfg<L, 384, 2>(d_jobs, n_jobs, n_items, 0, d_ctl, num_sms, st);
        if (cfg.order == 2)
            return cfg.threads == 256
                       ? launch_cfg<L, 256, 3>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st)
                       : launch_cfg<L, 384, 3>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
        return cfg.threads == 256 ? launch_cfg<L, 256, 1>(d_jobs, n_jobs, n_items, 0, d_ctl, num_sms, st)
                                  : launch_cfg<L, 384, 1>(d_jobs, n_jobs, n_items, 0, d_ctl, num_sms, st);
    }
    if (cfg.mode == 3)  // sparse with per-stage barriers: 512 threads
        return launch_cfg<L, 512, 5>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
    if (cfg.mode == 2) {  // sparse, deferred candidates: 192, 256 or 384 threads (larger stage-1 tables)
        switch (cfg.threads) {
            case 192: return launch_cfg<L, 192, 4>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
            case 384: return launch_cfg<L, 384, 4>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
            default: return launch_cfg<L, 256, 4>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
        }
    }
    switch (cfg.threads) {
        case 256: return launch_cfg<L, 256, 0>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
        case 384: return launch_cfg<L, 384, 0>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
        default: return launch_cfg<L, 512, 0>(d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
    }
}

size_t fixed_smem_for(int threads, bool dense) {
    if (dense) return threads == 256 ? fixed_smem<256, 1>() : threads == 192 ? fixed_smem<192, 1>() : fixed_smem<384, 1>();
    switch (threads) {
        case 192: return fixed_smem<192, 0>();
        case 256: return fixed_smem<256, 0>();
        case 384: return fixed_smem<384, 0>();
        default: return fixed_smem<512, 0>();
    }
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

// Largest power-of-two stage-1 table (in bits, <= C) that fits beside the fixed shared-memory layout.
uint32_t stage1_shift_for(const Geom& g, int threads, bool dense) {
    const size_t room = kSmemLimit - fixed_smem_for(threads, dense) - static_smem(threads) - 64;
    uint32_t sh = 0;
    while (((uint64_t)g.cache_bits >> sh) / 8 > room) sh++;
    return sh;
}

uint32_t stage1_words_for(const Geom& g, int threads, bool dense) {
    return (uint32_t)(((uint64_t)g.cache_bits >> stage1_shift_for(g, threads, dense)) / 32);
}

int dense_probe_order(const Geom& g, double cache_fill, double ext_fill) {
    // Cost of a plan per valid window, in L2 probes: the first probe always, the second when the first
    // passes, and a queued window's full test (about three probes' worth of issue and flush work) when both
    // pass. A probe of a region that the L1 left beside the shared memory can largely hold (about 64 KiB)
    // mostly hits there.
    const double c_bytes = g.cache_bits / 8.0, e_bytes = (g.ext_mask + 1.0) / 8.0;
    auto fill = [&](uint32_t i) { return i < g.s ? cache_fill : ext_fill; };
    auto miss = [&](uint32_t i) { return 1.0 - std::min(1.0, 65536.0 / (i < g.s ? c_bytes : e_bytes)); };
    auto cost = [&](uint32_t a, uint32_t b) {
        return miss(a) + fill(a) * miss(b) + 3.0 * fill(a) * fill(b);
    };
    int best = 0;
    double best_cost = cost(0, 1);
    if (g.k >= 4 && cost(2, 3) < best_cost) {
        best = 1;
        best_cost = cost(2, 3);
    }
    // Order 2: f0's load only where the folded cache region (the table the 384-thread dense kernel has room
    // for) has its bit set, at about 0.15 probes' worth of shared-memory work per window. A table bit ORs
    // C/T cache bits, so it is set with probability 1 - (1 - fill)^(C/T).
    const double folds = (double)(1u << stage1_shift_for(g, 384, true));
    const double fold_fill = 1.0 - std::pow(1.0 - cache_fill, folds);
    const double c2 = 0.15 + fold_fill * miss(0) + fill(0) * miss(1) + 3.0 * fill(0) * fill(1);
    if (c2 < best_cost) best = 2;
    return best;
}

int config_threads(const FastConfig& cfg) {
    if (cfg.mode == 1) return cfg.threads == 256 ? 256 : cfg.threads == 192 && cfg.order != 2 ? 192 : 384;
    if (cfg.mode == 2) return cfg.threads == 192 || cfg.threads == 384 ? cfg.threads : 256;
    if (cfg.mode == 3) return 512;
    return cfg.threads == 384 || cfg.threads == 512 ? cfg.threads : 256;
}

int fast_ctas_per_sm(const FastConfig& cfg) { return cfg.mode == 1 && config_threads(cfg) == 192 ? 2 : 1; }

uint32_t fast_rows(uint64_t n, const FastConfig& cfg, int num_sms, bool batch) {
    const int threads = config_threads(cfg);
    const uint64_t tiles_bytes = n / kScanTile * kScanTile;
    if (batch) {
        // in a batch other jobs fill the GPU: the largest tile this job still fills four times over
        uint32_t rows = 16;
        while (rows > 4 && tiles_bytes < 4ull * rows * kRowBytes * threads) rows >>= 1;
        return rows;
    }
    // alone: the scan lasts as many waves of equal items as the busiest CTA takes, and an item costs its
    // rows plus its halo, whose 32 hashed bytes are a quarter of a row's work (measured: 256 MiB of the
    // plain workload, 2 waves of 16 rows against 7 of 4, took 571 against 528 us). The row count with the
    // least work per CTA wins; ties go to the longer items.
    const uint64_t slots = (uint64_t)num_sms * (uint64_t)fast_ctas_per_sm(cfg);
    uint32_t best = 16;
    uint64_t best_cost = ~0ull;
    for (uint32_t rows = 16; rows >= 4; rows >>= 1) {
        const uint64_t items = (tiles_bytes / ((uint64_t)rows * kRowBytes) + threads - 1) / threads;
        const uint64_t cost = (items + slots - 1) / slots * (4 * rows + 1);  // in quarter rows
        if (cost < best_cost) {
            best_cost = cost;
            best = rows;
        }
    }
    return best;
}

uint64_t fill_fast_job(const ScanArgs& a, const uint32_t* stage1_words, const FastConfig& cfg, uint32_t rows,
                       FastJob* job, cudaError_t* err) {
    *err = cudaSuccess;
    const int threads = config_threads(cfg);
    const uint64_t fast_tiles = a.n / kScanTile;  // whole 16 KiB tiles; the rest goes to the generic kernel
    const uint64_t slen = (uint64_t)rows * kRowBytes;
    const uint64_t n_streams = fast_tiles * kScanTile / slen;
    memset(job, 0, sizeof *job);
    job->n_streams = n_streams;
    job->rows = rows;
    job->n_supertiles = (uint32_t)((n_streams + threads - 1) / threads);
    uint32_t spt = (uint32_t)(kScanTile / slen), lg = 0;
    while ((1u << lg) < spt) lg++;
    job->streams_per_tile_log2 = lg;
    job->g = a.g;
    job->main_words = a.main_words;
    job->ff_words = a.ff_words;
    job->stage1_words = stage1_words;
    // the table the kernel reads: the sparse mode's, or the dense mode's prefilter (order 2)
    const bool reads_table = cfg.mode != 1 || cfg.order == 2;
    job->stage1_shift = reads_table ? stage1_shift_for(a.g, threads, cfg.mode == 1) : 0;
    job->stage1_nwords = reads_table ? (uint32_t)(((uint64_t)a.g.cache_bits >> job->stage1_shift) / 32) : 0;
    {
        // dense mode: regions of the pipelined probes, index functions f0/f1 (order 0) or f2/f3 (order 1,
        // which only K >= 4 filters set)
        if (cfg.mode < 0 || cfg.mode > 3 ||
            (cfg.mode == 1 && (a.g.k < 2 || (cfg.order == 1 && a.g.k < 4) || cfg.order < 0 || cfg.order > 2)))
            *err = cudaErrorInvalidValue;
        const uint32_t fa = cfg.order == 1 ? 2u : 0u, fb = fa + 1;
        job->a_mask = fa < a.g.s ? a.g.cache_mask : a.g.ext_mask;
        job->a_add = fa < a.g.s ? 0u : a.g.cache_bits;
        job->b_mask = fb < a.g.s ? a.g.cache_mask : a.g.ext_mask;
        job->b_add = fb < a.g.s ? 0u : a.g.cache_bits;
    }
    job->hits = a.hits;
    job->hits_cap = a.hits_cap;
    job->counters = a.counters;
    job->tile_first_nl = a.tile_first_nl;
    job->tile_last_nl = a.tile_last_nl;
    job->n_tiles = a.ntiles;
    // FFBF_TEXT_L2=normal keeps the default L2 policy for the text's loads (for comparisons)
    static const bool evict_first = [] {
        const char* v = getenv("FFBF_TEXT_L2");
        return !(v && strcmp(v, "normal") == 0);
    }();
    job->text_evict_first = evict_first ? 1u : 0u;
    if (n_streams > 0) {
        const uint32_t box_streams = threads > 256 ? (uint32_t)threads / 2 : (uint32_t)threads;
        cuuint64_t dims[3] = {(cuuint64_t)kRowBytes, (cuuint64_t)rows, (cuuint64_t)n_streams};
        cuuint64_t strides[2] = {(cuuint64_t)kRowBytes, (cuuint64_t)slen};
        cuuint32_t box[3] = {(cuuint32_t)kRowBytes, 1u, box_streams};
        cuuint32_t estr[3] = {1u, 1u, 1u};
        CUresult cr = encoder()(&job->tmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void*)a.text, dims, strides, box, estr,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (cr != CUDA_SUCCESS) *err = cudaErrorInvalidValue;
    }
    return fast_tiles * kScanTile;
}

cudaError_t launch_fast_jobs(uint32_t len, const FastConfig& cfg, const FastJob* d_jobs, uint32_t n_jobs,
                             uint32_t n_items, uint32_t max_s1_words, uint32_t* d_ctl, int num_sms,
                             cudaStream_t st) {
    switch (len) {
        case 16: return launch_len<16>(cfg, d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
        case 19: return launch_len<19>(cfg, d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
        case 20: return launch_len<20>(cfg, d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
        case 24: return launch_len<24>(cfg, d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
        case 32: return launch_len<32>(cfg, d_jobs, n_jobs, n_items, max_s1_words, d_ctl, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t scan_tail(const ScanArgs& a, uint64_t covered, cudaStream_t st) {
    const uint64_t ntiles = (a.n + kScanTile - 1) / kScanTile;
    const uint64_t first = covered / kScanTile;
    if (first >= ntiles) return cudaSuccess;
    ScanArgs t = a;
    t.tile_begin = first;
    t.cache_in_smem = a.g.cache_bits <= kSmemCacheMaxBits;
    const int grid = scan_generic_grid(a.g, t.cache_in_smem, ntiles - first);
    if (grid <= 0) return cudaErrorInvalidConfiguration;
    return scan_generic(t, grid, st);
}

cudaError_t scan_fast(const ScanArgs& a, const uint32_t* stage1_words, const FastConfig& cfg, int num_sms,
                      FastJob* h_job, FastJob* d_job, cudaStream_t st) {
    const int threads = config_threads(cfg);
    const uint32_t rows = cfg.rows ? cfg.rows : fast_rows(a.n, cfg, num_sms, false);
    cudaError_t e;
    const uint64_t covered = fill_fast_job(a, stage1_words, cfg, rows, h_job, &e);
    if (e != cudaSuccess) return e;
    if (h_job->n_supertiles) {
        e = cudaMemcpyAsync(d_job, h_job, sizeof(FastJob), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
        e = launch_fast_jobs(a.g.len, cfg, d_job, 1, h_job->n_supertiles, h_job->stage1_nwords,
                             a.counters + CNT_ERROR, num_sms, st);  // ctl = {CNT_ERROR, CNT_QUEUE}
        if (e != cudaSuccess) return e;
    }
    return scan_tail(a, covered, st);
}

// Stage-1 table of T = C >> sh bits for the sparse mode: bit j = OR of the cache bits i with i mod T == j
// (a fold, so the table index of a window is just h & (T-1)). A window passes the reference test only if
// its cache bit is set, which sets its table bit: the table rejects only windows the full test rejects.
__global__ void k_stage1_fold(const uint32_t* main_words, uint32_t sh, uint32_t* out, uint32_t nwords) {
    uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwords) return;
    uint32_t v = 0;
    const uint32_t folds = 1u << sh;
    for (uint32_t m = 0; m < folds; m++) v |= main_words[w + m * nwords];
    out[w] = v;
}

cudaError_t build_stage1(const uint32_t* main_words, const Geom& g, int threads, bool dense, uint32_t* out,
                         cudaStream_t st) {
    const uint32_t sh = stage1_shift_for(g, threads, dense);
    const uint32_t nwords = (uint32_t)(((uint64_t)g.cache_bits >> sh) / 32);
    if (sh == 0) return cudaMemcpyAsync(out, main_words, 4ull * nwords, cudaMemcpyDeviceToDevice, st);
    k_stage1_fold<<<(nwords + 255) / 256, 256, 0, st>>>(main_words, sh, out, nwords);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace ffbf

namespace ffbf {

__global__ void k_popcount(const uint32_t* w, uint32_t n, unsigned long long* out) {
    unsigned long long c = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c += __popc(w[i]);
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

cudaError_t popcount_words(const uint32_t* w, uint32_t n, unsigned long long* d_out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess || n == 0) return e;
    k_popcount<<<(n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024, 256, 0, st>>>(w, n, d_out);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace ffbf
