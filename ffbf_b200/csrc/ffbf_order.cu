// ffbf_order.cu -- device-side ordering of scan results (see ffbf_order.cuh).
//
// The sorts are CUB's stable LSD radix sorts over only the key bits that can be non-zero (the text
// length's bit width), so a 4 GiB text's window starts take 5 eight-bit passes instead of 8. The line
// reduction is a flag per sorted window (its line starts where the previous window's does not) and a
// flagged selection.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include "ffbf_order.cuh"

namespace ffbf {

namespace {

constexpr size_t kAlign = 256;

size_t up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

int grid_for(uint64_t n) {
    const uint64_t g = (n + 255) / 256;
    return (int)(g < 148 * 16 ? (g ? g : 1) : 148 * 16);
}

__global__ void k_hit_keys(const HitRec* __restrict__ hits, uint32_t nh, uint64_t* __restrict__ keys,
                           uint32_t* __restrict__ idx) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) {
        keys[i] = hits[i].off;
        idx[i] = i;
    }
}

// The lines of the sorted windows, and a flag on each window whose line is not the previous window's.
// Lines are disjoint and windows sorted by start, so equal lines are adjacent.
__global__ void k_sorted_lines(const HitLine* __restrict__ lines, const uint32_t* __restrict__ perm, uint32_t nh,
                               HitLine* __restrict__ out, uint8_t* __restrict__ flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) {
        const HitLine l = lines[perm[i]];
        out[i] = l;
        flags[i] = (i == 0 || lines[perm[i - 1]].start != l.start) ? 1 : 0;
    }
}

struct HitsLayout {
    size_t keys, vals_in, vals_out, lines, flags, temp, total;
};

HitsLayout hits_layout(uint32_t nh, int key_bits) {
    size_t sort_tmp = 0, sel_tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, nh, 0, key_bits);
    cub::DeviceSelect::Flagged(nullptr, sel_tmp, (const HitLine*)nullptr, (const uint8_t*)nullptr, (HitLine*)nullptr,
                               (uint64_t*)nullptr, (int64_t)nh);
    HitsLayout L;
    L.keys = 0;
    L.vals_in = L.keys + up(8ull * nh);
    L.vals_out = L.vals_in + up(4ull * nh);
    L.lines = L.vals_out + up(4ull * nh);
    L.flags = L.lines + up(sizeof(HitLine) * (size_t)nh);
    L.temp = L.flags + up(nh);
    L.total = L.temp + up(sort_tmp > sel_tmp ? sort_tmp : sel_tmp);
    return L;
}

struct MatchLayout {
    size_t pid, off, temp, temp_bytes, total;
};

MatchLayout match_layout(uint32_t nm, int off_bits) {
    size_t t1 = 0, t2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const uint64_t*)nullptr, (uint64_t*)nullptr, nm, 0, 32);
    cub::DeviceRadixSort::SortPairs(nullptr, t2, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, nm, 0, off_bits);
    MatchLayout L;
    L.pid = 0;
    L.off = L.pid + up(4ull * nm);
    L.temp = L.off + up(8ull * nm);
    L.temp_bytes = t1 > t2 ? t1 : t2;
    L.total = L.temp + up(L.temp_bytes);
    return L;
}

}  // namespace

int key_bits_for(uint64_t n) {
    int b = 1;
    while (b < 64 && (n >> b) != 0) b++;
    return b;
}

size_t order_hits_scratch(uint32_t nh, int key_bits) { return hits_layout(nh, key_bits).total; }

cudaError_t order_hits(const HitRec* d_hits, const HitLine* d_lines, uint32_t nh, int key_bits, void* d_scratch,
                       size_t scratch_bytes, uint64_t* d_off, HitLine* d_lines_out, uint64_t* d_nlines,
                       cudaStream_t st) {
    if (nh == 0) return cudaMemsetAsync(d_nlines, 0, sizeof(uint64_t), st);
    const HitsLayout L = hits_layout(nh, key_bits);
    if (scratch_bytes < L.total) return cudaErrorInvalidValue;
    uint8_t* s = static_cast<uint8_t*>(d_scratch);
    uint64_t* keys = reinterpret_cast<uint64_t*>(s + L.keys);
    uint32_t* vals_in = reinterpret_cast<uint32_t*>(s + L.vals_in);
    uint32_t* vals_out = reinterpret_cast<uint32_t*>(s + L.vals_out);
    HitLine* lines = reinterpret_cast<HitLine*>(s + L.lines);
    uint8_t* flags = s + L.flags;
    size_t temp_bytes = L.total - L.temp;

    k_hit_keys<<<grid_for(nh), 256, 0, st>>>(d_hits, nh, keys, vals_in);
    note_launches(1);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(s + L.temp, temp_bytes, keys, d_off, vals_in, vals_out, nh, 0,
                                                    key_bits, st);
    if (e != cudaSuccess) return e;
    k_sorted_lines<<<grid_for(nh), 256, 0, st>>>(d_lines, vals_out, nh, lines, flags);
    note_launches(1);
    temp_bytes = L.total - L.temp;
    return cub::DeviceSelect::Flagged(s + L.temp, temp_bytes, lines, flags, d_lines_out, d_nlines, (int64_t)nh, st);
}

size_t order_matches_scratch(uint32_t nm, int off_bits) { return match_layout(nm, off_bits).total; }

cudaError_t order_matches(uint64_t* d_off, uint32_t* d_pid, uint32_t nm, int off_bits, void* d_scratch,
                          size_t scratch_bytes, cudaStream_t st) {
    if (nm < 2) return cudaSuccess;
    const MatchLayout L = match_layout(nm, off_bits);
    if (scratch_bytes < L.total) return cudaErrorInvalidValue;
    uint8_t* s = static_cast<uint8_t*>(d_scratch);
    uint32_t* pid = reinterpret_cast<uint32_t*>(s + L.pid);
    uint64_t* off = reinterpret_cast<uint64_t*>(s + L.off);
    // least significant key first: by pattern id, then (stable) by offset
    size_t tb = L.temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(s + L.temp, tb, d_pid, pid, d_off, off, nm, 0, 32, st);
    if (e != cudaSuccess) return e;
    tb = L.temp_bytes;
    return cub::DeviceRadixSort::SortPairs(s + L.temp, tb, off, d_off, pid, d_pid, nm, 0, off_bits, st);
}

}  // namespace ffbf
