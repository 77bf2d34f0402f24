// ffbf_order.cuh -- device-side ordering of scan results.
//
// processFile (src/rabin-karp/ffbf.cpp:310-392) meets hit windows in text order and prints each flagged
// line once. The scan kernels append hit records in whatever order their warps flush, so the results are
// put in text order here, on the device: window starts sorted ascending, the lines of the sorted windows
// reduced to the distinct ones, and verified matches sorted by (offset, pattern id). The host then copies
// back arrays that are already in their final order.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "ffbf_kernels.cuh"

namespace ffbf {

// Bits that hold every value below n (at least 1): the radix sorts skip the always-zero high bits.
int key_bits_for(uint64_t n);

// Device scratch bytes order_hits needs for nh records (its outputs not included).
size_t order_hits_scratch(uint32_t nh, int key_bits);

// Sorts the window starts of nh hit records ascending into d_off (nh words), writes the distinct lines of
// the sorted windows in text order to d_lines_out (at most nh) and their count to *d_nlines. Window
// starts must be below 2^key_bits.
cudaError_t order_hits(const HitRec* d_hits, const HitLine* d_lines, uint32_t nh, int key_bits, void* d_scratch,
                       size_t scratch_bytes, uint64_t* d_off, HitLine* d_lines_out, uint64_t* d_nlines,
                       cudaStream_t st);

// Device scratch bytes order_matches needs for nm matches.
size_t order_matches_scratch(uint32_t nm, int off_bits);

// Sorts nm matches (d_off[i], d_pid[i]) by offset and then pattern id, in place. Offsets must be below
// 2^off_bits.
cudaError_t order_matches(uint64_t* d_off, uint32_t* d_pid, uint32_t nm, int off_bits, void* d_scratch,
                          size_t scratch_bytes, cudaStream_t st);

}  // namespace ffbf
