// ffbf_scan_fast.cuh -- the tuned sm_100a scan (see ffbf_scan_fast.cu).
#pragma once
#include "ffbf_kernels.cuh"

namespace ffbf {

// True when the tuned kernel handles this geometry and text size; otherwise the generic scan runs.
bool fast_scan_supported(const Geom& g, uint64_t n);

// Same contract as scan_generic: sets feed-forward bits, appends hits, fills the per-tile newline
// summaries (kScanTile granularity) that resolve_lines reads.
cudaError_t scan_fast(const ScanArgs& a, int num_sms, cudaStream_t st);

}  // namespace ffbf
