// ffbf_scan_fast.cu -- tuned sm_100a scan (placeholder until the tuned kernel lands).
#include "ffbf_scan_fast.cuh"

namespace ffbf {

bool fast_scan_supported(const Geom&, uint64_t) { return false; }

cudaError_t scan_fast(const ScanArgs&, int, cudaStream_t) { return cudaErrorNotSupported; }

}  // namespace ffbf
