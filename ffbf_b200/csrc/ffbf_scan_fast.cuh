// ffbf_scan_fast.cuh -- the tuned sm_100a scan (see ffbf_scan_fast.cu).
#pragma once
#include "ffbf_kernels.cuh"

namespace ffbf {

// True when the tuned kernel handles this geometry and text size; otherwise the generic scan runs.
bool fast_scan_supported(const Geom& g, uint64_t n);

// Same contract as scan_generic over tiles [0, ntiles): sets feed-forward bits, appends hits, fills the
// per-tile newline summaries (kScanTile granularity) that resolve_lines reads. Whole 16 KiB tiles run in
// the tuned kernel, a partial last tile in the generic one. stage1_words is the device buffer filled by
// build_stage1 for the current main filter.
// mode 0: sparse filters (shared-memory stage 1); mode 1: dense filters (pipelined exact h1 probe in L2).
cudaError_t scan_fast(const ScanArgs& a, const uint32_t* stage1_words, int mode, int num_sms, cudaStream_t st);

// Number of set bits in n words, written to *d_out (device).
cudaError_t popcount_words(const uint32_t* w, uint32_t n, unsigned long long* d_out, cudaStream_t st);

// Stage-1 table of the tuned scan: a copy of the cache region when it fits in shared memory, otherwise
// its OR-summary. stage1_words_for gives its size in 32-bit words.
uint32_t stage1_words_for(const Geom& g);
uint32_t stage1_shift_for(const Geom& g);

// Threads per CTA of the tuned scan (256, 384 or 512); anything else restores the default.
int fast_scan_threads();
void set_fast_scan_threads(int threads);
cudaError_t build_stage1(const uint32_t* main_words, const Geom& g, uint32_t* out, cudaStream_t st);

}  // namespace ffbf
