// ffbf_kernels.cuh -- launch interface of the FFBF device kernels (host-callable wrappers).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "ffbf_device.cuh"

namespace ffbf {

// Process-wide count of kernels launched by the library (reported through ffbf_kernel_launches).
void note_launches(uint64_t n);
// Takes back launches counted while a stream was being captured (they run when the graph does).
void unnote_launches(uint64_t n);
uint64_t launches_total();

// One hit window: start offset in the text and its 64-bit rolling hash.
struct HitRec {
    uint64_t off;
    uint64_t h;
};

// Line span of a hit, filled by the resolve kernel.
struct HitLine {
    uint64_t start;
    uint64_t end;
};

// Device counters shared by a scan: [0] hits found, [1] matches found, [2] error flags.
// Per-scan counters: hit windows, verified matches, error flags, and the tuned scan's next-item counter
// (its work queue); all four start at zero.
enum { CNT_HITS = 0, CNT_MATCHES = 1, CNT_ERROR = 2, CNT_QUEUE = 3, CNT_WORDS = 4 };

// Scan tile geometry of the generic kernel: each CTA stages TILE bytes (+ a 64-byte halo).
constexpr int kScanThreads = 256;
constexpr int kScanSeg = 64;
constexpr int kScanTile = kScanThreads * kScanSeg;  // 16 KiB
constexpr int kHalo = 64;                           // >= LEN-1 for LEN <= 63, and 16-byte aligned
constexpr uint32_t kSmemCacheMaxBits = 1u << 20;    // cache region copied to smem when C <= 2^20 bits

struct ScanArgs {
    const uint8_t* text;
    uint64_t n;
    Geom g;
    const uint32_t* main_words;
    uint32_t* ff_words;
    HitRec* hits;
    uint32_t hits_cap;
    uint32_t* counters;
    long long* tile_first_nl;  // per tile: first '\n' position in the tile, or LLONG_MAX
    long long* tile_last_nl;   // per tile: last '\n' position in the tile, or -1
    uint64_t ntiles;
    uint64_t tile_begin;  // first tile this launch handles (tiles before it belong to another kernel)
    int cache_in_smem;
};

// Ordered compaction in two steps. *_count leaves per-chunk offsets in d_tmp (compact_blocks(n) + 1
// words) and the total in d_tmp[compact_blocks(n)]; *_emit writes the ascending indices.
uint64_t compact_blocks(uint64_t n);
cudaError_t count_bytes(const uint8_t* d_buf, uint64_t n, uint8_t byte, uint64_t* d_tmp, cudaStream_t st);
cudaError_t emit_bytes(const uint8_t* d_buf, uint64_t n, uint8_t byte, uint64_t* d_pos, const uint64_t* d_tmp,
                       cudaStream_t st);
cudaError_t count_flags(const uint8_t* d_flags, uint64_t n, uint64_t* d_tmp, cudaStream_t st);
cudaError_t emit_flags(const uint8_t* d_flags, uint64_t n, uint64_t* d_out, const uint64_t* d_tmp, cudaStream_t st);
cudaError_t lines_from_newlines(const uint64_t* d_nl, uint64_t m, uint64_t n, int tail, uint64_t* d_start,
                                uint64_t* d_end, cudaStream_t st);
cudaError_t hash_patterns(const uint8_t* d_file, const uint64_t* d_start, const uint64_t* d_end, uint64_t npat,
                          const Geom& g, uint64_t* d_hash, uint32_t* d_main, int set_bits, cudaStream_t st);

size_t scan_smem_bytes(int cache_in_smem, const Geom& g);
int scan_generic_grid(const Geom& g, int cache_in_smem, uint64_t ntiles);
// Generic scan of tiles from many jobs (items: {job index, tile}); probes the global filters.
cudaError_t scan_generic_multi(const ScanArgs* d_jobs, const uint2* d_items, uint32_t n_items, int num_sms,
                               cudaStream_t st);
cudaError_t zero_counters(uint32_t* const* d_ptrs, uint32_t n, cudaStream_t st);
cudaError_t gather_counters(uint32_t* const* d_ptrs, uint32_t n, uint32_t* d_out, cudaStream_t st);
cudaError_t scan_generic(const ScanArgs& a, int grid, cudaStream_t st);
// Hit -> line span. `agg` (2 * tile_agg_words(ntiles) words, optional) lets the tile-newline scan run
// over all SMs; without it one block scans the tiles.
constexpr uint32_t kTileAggBlock = 4096;  // tiles per block of the two-pass tile-newline scan
inline uint64_t tile_agg_words(uint64_t ntiles) { return ntiles / kTileAggBlock + 1; }
cudaError_t resolve_lines(const uint8_t* text, uint64_t n, uint32_t len, const HitRec* hits, uint32_t nhits,
                          const long long* tile_first, const long long* tile_last, long long* prev_nl,
                          long long* next_nl, uint64_t ntiles, HitLine* out, cudaStream_t st,
                          long long* agg = nullptr);

cudaError_t prune_flags(const uint64_t* d_start, const uint64_t* d_end, const uint64_t* d_hash, uint64_t npat,
                        const Geom& g, const uint32_t* d_ff, uint8_t* d_flags, cudaStream_t st);

cudaError_t table_build(const uint64_t* d_ids, uint64_t nids, const uint64_t* d_hash, uint64_t* d_keys,
                        uint32_t* d_vals, uint64_t mask, uint32_t* d_counters, cudaStream_t st);
cudaError_t verify_hits(const HitRec* hits, uint32_t nhits, const uint8_t* text, uint64_t n, const uint64_t* d_keys,
                        const uint32_t* d_vals, uint64_t mask, const uint8_t* d_pat, const uint64_t* d_start,
                        const uint64_t* d_end, uint64_t* d_match_off, uint32_t* d_match_pid, uint32_t match_cap,
                        uint32_t* d_counters, cudaStream_t st);

// Filter cache file codec (delta-coded uint32 set-bit indices).
cudaError_t filter_decode(const uint32_t* d_deltas, uint64_t nd, uint32_t nbits, uint32_t* d_idx, uint64_t* d_tmp,
                          uint32_t* d_counters, cudaStream_t st);
cudaError_t filter_set_indices(const uint32_t* d_idx, uint64_t nd, uint32_t* d_main, cudaStream_t st);
cudaError_t filter_count(const uint32_t* d_main, uint32_t nwords, uint64_t* d_tmp, cudaStream_t st);
// filter_count leaves per-chunk offsets in d_tmp and the number of set bits in d_tmp[enc_blocks(nwords)].
uint64_t enc_blocks(uint32_t nwords);
cudaError_t filter_encode(const uint32_t* d_main, uint32_t nwords, const uint64_t* d_tmp, uint32_t* d_idx,
                          cudaStream_t st);
cudaError_t filter_deltas(const uint32_t* d_idx, uint64_t n, uint32_t* d_out, cudaStream_t st);
uint64_t decode_blocks(uint64_t nd);

cudaError_t test_line(const uint8_t* d_line, uint64_t n, const Geom& g, const uint32_t* d_main, uint32_t* d_out,
                      cudaStream_t st);

}  // namespace ffbf
