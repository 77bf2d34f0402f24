// ffbf_device.cuh -- device-side definitions shared by the FFBF kernels.
//
// The hash, the index functions and the bit layout are fixed by efficient/ffbf:
//  * rolling hash   src/hashes/hash_rot_sbox_pre_2.h:42-51 (rol64 at src/hashes/hash_common.h:13-16);
//    closed form for a window x[0..L): h = XOR_j rol64(S[x_j], L-1-j)
//  * byte mapping   src/rabin-karp/ffbf.cpp:127-130 (bytes with the high bit set hash as 0)
//  * index order    getHashValue ffbf.cpp:135-159 (main filter), getHashValue_2 ffbf.cpp:161-185 (FF filter)
//  * bit layout     setBit ffbf.cpp:187-193: bit i is byte i>>3, mask 1<<(i&7). On little-endian that is
//                   bit i&31 of 32-bit word i>>5, so 32-bit atomicOr gives the same bytes.
#pragma once
#include <stdint.h>

#include "ffbf_sbox.h"

namespace ffbf {

// Geometry as the kernels see it. N = cache_bits + ext_bits <= 2^31.
struct Geom {
    uint32_t len;         // LEN
    uint32_t k;           // K
    uint32_t s;           // S
    uint32_t cache_bits;  // C (added to external-region indices)
    uint32_t cache_mask;  // C - 1
    uint32_t ext_mask;    // E - 1
    uint32_t nbits;       // N
    uint32_t pad;
};

__device__ __forceinline__ uint64_t rol64(uint64_t w, uint32_t s) {
    // s in 1..63 at every call site
    return (w << s) | (w >> (64u - s));
}

// Index function f of getHashValue (ffbf.cpp:140-153); getHashValue_2 case i is f = kFF2Map[i].
__device__ __forceinline__ uint32_t index_fn(uint32_t h1, uint32_t h2, uint32_t f) {
    switch (f) {
        case 0: return h1;
        case 1: return h2;
        case 2: return (h1 << 16) | (h1 >> 16);
        case 3: return (h2 << 16) | (h2 >> 16);
        case 4: return h1 + h2;
        case 5: return h1 + (h2 << 1);
        case 6: return h1 + (h2 << 2);
        case 7: return h1 + 3u * h2;
        case 8: return h1 + 5u * h2;
        case 9: return h1 + 6u * h2;
        default: return h1 + 7u * h2;
    }
}

// getHashValue_2 case i == getHashValue formula (i + 5) mod 11 (ffbf.cpp:168-178 vs :142-152).
__device__ __forceinline__ uint32_t ff2_fn(uint32_t i) { return i < 6 ? i + 5 : i - 6; }

// Bit index of probe i (0 <= i < K), main order (ORDER 1) or feed-forward order (ORDER 2).
template <int ORDER>
__device__ __forceinline__ uint32_t bit_index(const Geom& g, uint64_t h, uint32_t i) {
    uint32_t h1 = (uint32_t)h, h2 = (uint32_t)(h >> 32);
    uint32_t x = index_fn(h1, h2, ORDER == 2 ? ff2_fn(i) : i);
    return i < g.s ? (x & g.cache_mask) : (x & g.ext_mask) + g.cache_bits;
}

__device__ __forceinline__ bool test_bit(const uint32_t* words, uint32_t i) {
    return (words[i >> 5] >> (i & 31)) & 1u;
}

__device__ __forceinline__ void set_bit_atomic(uint32_t* words, uint32_t i) {
    uint32_t m = 1u << (i & 31);
    // Skip the atomic when the bit is already visible as set: FF bits are set by every hit window.
    if (!(__ldcg(words + (i >> 5)) & m)) atomicOr(words + (i >> 5), m);
}

template <int ORDER>
__device__ __forceinline__ bool check_all(const Geom& g, const uint32_t* words, uint64_t h) {
    for (uint32_t i = 0; i < g.k; i++)
        if (!test_bit(words, bit_index<ORDER>(g, h, i))) return false;
    return true;
}

template <int ORDER>
__device__ __forceinline__ void set_all(const Geom& g, uint32_t* words, uint64_t h) {
    for (uint32_t i = 0; i < g.k; i++) set_bit_atomic(words, bit_index<ORDER>(g, h, i));
}

// Statically initialised in every translation unit that includes this header (2 KiB of constant memory).
static __constant__ uint64_t c_sbox[256] = {FFBF_SBOX_WORDS};

__device__ __forceinline__ uint64_t sbox_of(uint32_t byte) { return c_sbox[(byte & 0x80u) ? 0u : byte]; }

// Hash of one window read from global memory (patterns, test lines); bytes are mapped per ffbf.cpp:127-130.
__device__ __forceinline__ uint64_t window_hash(const uint8_t* p, uint32_t len) {
    uint64_t h = 0;
    for (uint32_t j = 0; j < len; j++) {
        h = rol64(h, 1) ^ sbox_of(p[j]);
    }
    // The rolling form adds rol(S, LEN) for the byte leaving the window; over exactly LEN updates from a
    // zero state nothing leaves, so the result equals XOR_j rol64(S[x_j], LEN-1-j).
    return h;
}

}  // namespace ffbf
