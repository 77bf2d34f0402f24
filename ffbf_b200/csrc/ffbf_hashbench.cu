// ffbf_hashbench.cu -- the reference's hash benchmark (src/hashes/hashbench.cc) for the scan's hash,
// hash_rot_sbox_pre_2<19>, on the device: `-l` prints every line's final hash, `-f` hashes the whole text.
//
// hashbench hashes raw bytes (it does not map bytes >= 0x80 to 0 as the filter does), so these kernels index
// the full 256-entry S-box. After a byte at position i the rolling hash is
//     h_i = XOR over j in [max(0, i - 18), i] of rol64(S[x_j], i - j),
// the closed form of hash_rot_sbox_pre_2::update (hash_rot_sbox_pre_2.h:42-51), so any position's hash needs
// only the 19 bytes ending there.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ffbf.h"
#include "ffbf_device.cuh"
#include "ffbf_kernels.cuh"

namespace {

constexpr int kHbLen = 19;            // HashTester<HASHFN<19>, 19> (hashbench.cc:183)
constexpr uint32_t kFgetsMax = 4094;  // fgets(buf, hashbufsize - 1, f) with hashbufsize 4096 (:65, :113)

__device__ __forceinline__ uint64_t rol(uint64_t w, int s) { return s ? (w << s) | (w >> (64 - s)) : w; }

// One thread per fgets piece: hash the piece's C string (up to its first NUL or '\n'); report hval() and the
// string's length.
__global__ void k_hash_pieces(const uint8_t* text, const uint64_t* start, const uint32_t* len, uint32_t n,
                              uint32_t* hval, uint32_t* slen) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t* p = text + start[i];
    uint32_t e = 0;
    while (e < len[i] && p[e] != 0 && p[e] != '\n') e++;
    uint64_t h = 0;
    const uint32_t b = e > (uint32_t)kHbLen ? e - kHbLen : 0;
    for (uint32_t j = b; j < e; j++) h ^= rol(ffbf::c_sbox[p[j]], (int)(e - 1 - j));
    hval[i] = (uint32_t)(h >> 32);
    slen[i] = e;
}

constexpr int kTile = 16384, kSeg = 64, kThreads = kTile / kSeg, kHalo = 32;

// The rolling hash after every byte of the text, XORed together (hash_file, hashbench.cc:60-99, which
// updates the hash for every byte and reports only the time). Tiles of 16 KiB are staged in shared memory
// with the 32 bytes before them; each thread rolls over 64 bytes after warming up on the 19 before them.
__global__ void __launch_bounds__(kThreads) k_hash_xor(const uint8_t* text, uint64_t n, unsigned long long* out) {
    __shared__ uint64_t s_sbox[256];
    __shared__ __align__(16) uint8_t s_text[kHalo + kTile];
    for (int i = threadIdx.x; i < 256; i += kThreads) s_sbox[i] = ffbf::c_sbox[i];
    uint64_t acc = 0;
    for (uint64_t t0 = (uint64_t)blockIdx.x * kTile; t0 < n; t0 += (uint64_t)gridDim.x * kTile) {
        __syncthreads();
        for (int q = threadIdx.x; q < (kHalo + kTile) / 4; q += kThreads) {
            const long long p = (long long)t0 - kHalo + 4LL * q;
            uint32_t v = 0;
            if (p >= 0 && p + 4 <= (long long)n) {
                v = __ldg(reinterpret_cast<const uint32_t*>(text + p));
            } else {
                for (int j = 0; j < 4; j++)
                    if (p + j >= 0 && p + j < (long long)n) v |= (uint32_t)text[p + j] << (8 * j);
            }
            *reinterpret_cast<uint32_t*>(s_text + 4 * q) = v;
        }
        __syncthreads();
        const uint64_t s = t0 + (uint64_t)threadIdx.x * kSeg;
        if (s >= n) continue;
        const uint64_t e = min(n, s + kSeg);
        // warm up on the (up to) 19 bytes before s: those positions' outgoing bytes are not subtracted, so
        // the state equals the closed form over the window ending at s - 1
        const uint64_t w0 = s >= (uint64_t)kHbLen ? s - kHbLen : 0;
        uint64_t h = 0;
        for (uint64_t i = w0; i < s; i++) h = rol(h, 1) ^ s_sbox[s_text[i - t0 + kHalo]];
        for (uint64_t i = s; i < e; i++) {
            h = rol(h, 1) ^ s_sbox[s_text[i - t0 + kHalo]];
            if (i >= (uint64_t)kHbLen) h ^= rol(s_sbox[s_text[i - kHbLen - t0 + kHalo]], kHbLen);
            acc ^= h;
        }
    }
    for (int o = 16; o; o >>= 1) acc ^= __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicXor(out, (unsigned long long)acc);
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" {

ffbf_status ffbf_hashbench_lines(int device, const uint8_t* text, size_t len, uint8_t** out, size_t* out_len) {
    if (!out || !out_len || (!text && len)) return FFBF_EINVAL;
    *out = nullptr;
    *out_len = 0;
    // the pieces fgets would return: a line through its '\n', or the next 4094 bytes of a longer line
    std::vector<uint64_t> start;
    std::vector<uint32_t> plen;
    for (size_t pos = 0; pos < len;) {
        size_t m = std::min<size_t>(kFgetsMax, len - pos);
        const void* nl = memchr(text + pos, '\n', m);
        if (nl) m = (size_t)((const uint8_t*)nl - (text + pos)) + 1;
        start.push_back(pos);
        plen.push_back((uint32_t)m);
        pos += m;
    }
    const uint32_t n = (uint32_t)start.size();
    std::vector<uint32_t> hv(n), sl(n);
    if (n) {
        if (cudaSetDevice(device) != cudaSuccess) {
            cudaGetLastError();
            return FFBF_ECUDA;
        }
        DevBuf dt, ds, dl, dh, de;
        if (cudaMalloc(&dt.p, len) != cudaSuccess || cudaMalloc(&ds.p, n * 8ull) != cudaSuccess ||
            cudaMalloc(&dl.p, n * 4ull) != cudaSuccess || cudaMalloc(&dh.p, n * 4ull) != cudaSuccess ||
            cudaMalloc(&de.p, n * 4ull) != cudaSuccess) {
            cudaGetLastError();
            return FFBF_ENOMEM_DEVICE;
        }
        cudaError_t e = cudaMemcpy(dt.p, text, len, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(ds.p, start.data(), n * 8ull, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dl.p, plen.data(), n * 4ull, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            k_hash_pieces<<<(n + 255) / 256, 256>>>((const uint8_t*)dt.p, (const uint64_t*)ds.p,
                                                    (const uint32_t*)dl.p, n, (uint32_t*)dh.p, (uint32_t*)de.p);
            ffbf::note_launches(1);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpy(hv.data(), dh.p, n * 4ull, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(sl.data(), de.p, n * 4ull, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return FFBF_ECUDA;
        }
    }
    // printf("%x %s\n", h.hval(), buf) per piece (hashbench.cc:125)
    size_t total = 0;
    for (uint32_t i = 0; i < n; i++) total += 10 + sl[i];
    uint8_t* o = (uint8_t*)malloc(total ? total : 1);
    if (!o) return FFBF_ENOMEM_HOST;
    size_t w = 0;
    for (uint32_t i = 0; i < n; i++) {
        w += (size_t)snprintf((char*)o + w, 10, "%x ", hv[i]);
        memcpy(o + w, text + start[i], sl[i]);
        w += sl[i];
        o[w++] = '\n';
    }
    *out = o;
    *out_len = w;
    return FFBF_OK;
}

ffbf_status ffbf_hashbench_file(int device, const uint8_t* text, size_t len, uint64_t* xor_of_hashes,
                                double* seconds) {
    if (!xor_of_hashes || (!text && len)) return FFBF_EINVAL;
    *xor_of_hashes = 0;
    if (seconds) *seconds = 0;
    if (!len) return FFBF_OK;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return FFBF_ECUDA;
    }
    DevBuf dt, dx;
    if (cudaMalloc(&dt.p, len) != cudaSuccess || cudaMalloc(&dx.p, 8) != cudaSuccess) {
        cudaGetLastError();
        return FFBF_ENOMEM_DEVICE;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const uint64_t tiles = (len + kTile - 1) / kTile;
    const int grid = (int)std::min<uint64_t>(tiles, (uint64_t)sms * 8);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaError_t e = cudaMemcpy(dt.p, text, len, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dx.p, 0, 8);
    if (e == cudaSuccess) {
        cudaEventRecord(e0);
        k_hash_xor<<<grid, kThreads>>>((const uint8_t*)dt.p, len, (unsigned long long*)dx.p);
        ffbf::note_launches(1);
        cudaEventRecord(e1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess) e = cudaMemcpy(xor_of_hashes, dx.p, 8, cudaMemcpyDeviceToHost);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return FFBF_ECUDA;
    }
    if (seconds) *seconds = ms * 1e-3;
    return FFBF_OK;
}

}  // extern "C"
