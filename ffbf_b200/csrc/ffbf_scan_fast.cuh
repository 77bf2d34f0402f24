// ffbf_scan_fast.cuh -- the tuned sm_100a scan (see ffbf_scan_fast.cu): job descriptors, configuration, launch.
#pragma once
#include <cuda.h>

#include "ffbf_kernels.cuh"

namespace ffbf {

// One scan job of the tuned kernel (a text, its filter, its outputs). Jobs live in device memory; a plain
// scan is a batch of one. The tensor map is the first member (64-byte alignment).
struct alignas(64) FastJob {
    CUtensorMap tmap;        // the text as {128 bytes, rows, n_streams}
    uint64_t n_streams;      // streams covered by the tensor map
    uint32_t rows;           // rows per stream (tile size: a supertile is THREADS * rows * 128 bytes)
    uint32_t n_supertiles;   // ceil(n_streams / THREADS)
    uint32_t item_begin;     // first work item of this job; the next job's item_begin ends it
    uint32_t streams_per_tile_log2;  // log2(16384 / (rows * 128))
    Geom g;
    const uint32_t* main_words;
    uint32_t* ff_words;
    const uint32_t* stage1_words;  // sparse mode: cache region copy or its fold (global), copied into smem
    uint32_t stage1_nwords;
    uint32_t stage1_shift;         // the table holds C >> shift bits (0: exact copy of the cache region)
    // dense mode: the regions of its two pipelined probes (bit = (f & mask) + add for index functions f0/f1,
    // or f2/f3 when the configuration's probe order is 1)
    uint32_t a_mask, a_add, b_mask, b_add;
    HitRec* hits;
    uint32_t hits_cap;
    uint32_t ready_spins;  // polls of *ready before the launch gives up (about 1 us each)
    uint32_t* counters;
    long long* tile_first_nl;
    long long* tile_last_nl;
    uint64_t n_tiles;  // 16 KiB tiles of the text (bounds the newline summary writes)
    // 1: the text's TMA loads carry an L2 evict-first policy (every text byte is read once, so its lines
    // should leave L2 before the filter's do); 0: the default policy
    uint32_t text_evict_first;
    // Optional publication gate of the launch (read from its first job): no load is issued until *ready is
    // non-zero; a gate still closed after ready_spins polls ends the launch with the timeout flag.
    const uint32_t* ready;
};

// How a job is scanned: CTA size (256/384/512), probe mode (0: sparse, shared-memory stage 1; 1: dense,
// pipelined L2 probes), rows per stream (0: chosen from the text size), and in the dense mode the probe order
// (0: the pipelined probes are index functions f0 = h1 and f1 = h2; 1: f2 = rot16(h1) and f3 = rot16(h2),
// the better pair when their region is sparser; 2: f0 and f1, with f0's load issued only when a folded copy
// of the cache region in shared memory has its bit set). The order only changes which bits are tested
// first: a window hits iff all K bits are set, in any order.
struct FastConfig {
    int threads;
    int mode;
    uint32_t rows;
    int order;
};

// Probe order for the dense mode from the fills (fraction of set bits) of the cache and external regions:
// the plan with the fewest expected L2 probes per window. Order 1 needs f2 and f3 among the K index
// functions (K >= 4).
int dense_probe_order(const Geom& g, double cache_fill, double ext_fill);

// True when the tuned kernel handles this geometry and text size; otherwise the generic scan runs.
bool fast_scan_supported(const Geom& g, uint64_t n);

int config_threads(const FastConfig& cfg);

// Stage-1 table for a CTA size: a copy of the cache region when it fits in the shared memory the kernel
// leaves over (the sparse kernel's, or with `dense` the dense kernel's, whose table prefilters f0 in probe
// order 2), otherwise its fold to C >> shift bits.
uint32_t stage1_shift_for(const Geom& g, int threads, bool dense = false);
uint32_t stage1_words_for(const Geom& g, int threads, bool dense = false);
cudaError_t build_stage1(const uint32_t* main_words, const Geom& g, int threads, bool dense, uint32_t* out,
                         cudaStream_t st);

// CTAs of the tuned kernel resident per SM for a configuration (two for the 192-thread dense kernel).
int fast_ctas_per_sm(const FastConfig& cfg);

// Rows per stream for a text of n bytes, alone on the GPU or in a batch.
uint32_t fast_rows(uint64_t n, const FastConfig& cfg, int num_sms, bool batch);

// Fills *job (host memory) for the whole 16 KiB tiles of a.text and returns the bytes it covers; the
// caller sets item_begin. scan_tail runs the generic kernel over the tiles from `covered` on.
uint64_t fill_fast_job(const ScanArgs& a, const uint32_t* stage1_words, const FastConfig& cfg, uint32_t rows,
                       FastJob* job, cudaError_t* err);
cudaError_t scan_tail(const ScanArgs& a, uint64_t covered, cudaStream_t st);

// One launch of the tuned kernel over n_jobs device-resident jobs sharing LEN and configuration.
// d_ctl[0] collects error flags; d_ctl[1] is the work-queue counter and must be zero at launch.
cudaError_t launch_fast_jobs(uint32_t len, const FastConfig& cfg, const FastJob* d_jobs, uint32_t n_jobs,
                             uint32_t n_items, uint32_t max_s1_words, uint32_t* d_ctl, int num_sms, cudaStream_t st);

// A plain scan: one job (h_job pinned host staging, d_job device copy) plus the generic tail.
cudaError_t scan_fast(const ScanArgs& a, const uint32_t* stage1_words, const FastConfig& cfg, int num_sms,
                      FastJob* h_job, FastJob* d_job, cudaStream_t st);

// Number of set bits in n words, written to *d_out (device).
cudaError_t popcount_words(const uint32_t* w, uint32_t n, unsigned long long* d_out, cudaStream_t st);

}  // namespace ffbf
