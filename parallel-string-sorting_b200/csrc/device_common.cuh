// device_common.cuh -- shared device helpers of the B200 string sample sort.
//
// Key model (the reference's get_char_uint64_simple, src/tools/stringset.hpp:
// 201-231): the 8 chars at s + depth packed big-endian into a u64, every byte
// from the first NUL on set to zero. lcpKeyType / lcpKeyDepth restate
// src/parallel/bingmann-parallel_sample_sort.hpp:225-237.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pssgpu {

// Error bits OR-ed into the device error word and mapped to status codes.
enum : uint32_t {
    ERR_OFFSET = 1u,     // a string offset lies outside the arena
    ERR_TIMEOUT = 2u,    // a bounded device-side wait gave up (grid barriers of k_wave)
    ERR_OVERFLOW = 4u,   // a work list exceeded its capacity
    ERR_INTERNAL = 8u,   // an internal invariant failed (index out of range)
    ERR_UNTERMINATED = 16u,  // the arena's last char is not NUL
};

struct Seg {
    uint32_t begin;  // first position in the permutation arrays
    uint32_t size;   // number of strings
    uint32_t depth;  // chars known to be shared (FINAL: the LCP inside)
    uint32_t meta;   // META_* bits
};
static_assert(sizeof(Seg) == 16, "Seg layout");

enum : uint32_t {
    META_BUF = 1u,    // which ping-pong buffer holds the segment
    META_VALID = 2u,  // keys at `depth` are cached in keys[buf]
    META_FINAL = 4u,  // all strings equal: copy out, LCP inside = depth
};

__device__ __forceinline__ uint64_t bswap64(uint64_t x)
{
    uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
    uint32_t a = __byte_perm(lo, 0, 0x0123);
    uint32_t b = __byte_perm(hi, 0, 0x0123);
    return ((uint64_t)a << 32) | b;
}

// Big-endian key of the 8 chars at byte position p of the arena; positions at
// or beyond nchars read as NUL. The arena is 8-byte aligned and readable for
// nchars + 16 bytes, so both aligned words are in bounds whenever p < nchars.
__device__ __forceinline__ uint64_t load_key(const uint8_t* __restrict__ chars,
                                             uint64_t nchars, uint64_t p)
{
    if (p >= nchars) return 0;
    const uint64_t* w = reinterpret_cast<const uint64_t*>(chars + (p & ~7ull));
    const unsigned sh = (unsigned)(p & 7) * 8u;
    uint64_t raw = __ldg(w) >> sh;
    if (sh) raw |= __ldg(w + 1) << (64u - sh);
    // lowest zero byte (little-endian order = string order)
    const uint64_t z = (raw - 0x0101010101010101ull) & ~raw & 0x8080808080808080ull;
    if (z) {
        const unsigned nb = (unsigned)(__ffsll((long long)z) - 1) >> 3;
        raw = nb ? (raw & (~0ull >> (64u - 8u * nb))) : 0ull;
    }
    return bswap64(raw);
}

// The raw little-endian 8-char windows at p, p + 8, ... (cnt <= NB of them)
// into raw[0, cnt); raw[cnt, NB) are left 0 and chars at or beyond nchars
// read as 0. The words come from 16-byte loads at the 16-byte boundary at or
// below chars + p (an absolute address, so the arena needs no more than its
// 8-byte alignment): every vector lies in a 16-byte block that holds a char
// of the arena or of its padding, and at most ceil((NB + 2) / 2) are read,
// where byte-wise 8-byte loads would take NB + 1 (a string's loads are one
// L1 request per lane each, which bounds the common-prefix pass). A window
// becomes load_key's value through finish_key.
template <int NB>
__device__ __forceinline__ void load_raw_chunks(const uint8_t* __restrict__ chars, uint64_t nchars,
                                                uint64_t p, uint32_t cnt, uint64_t* raw)
{
    constexpr int NV = (NB + 3) / 2;
    const uintptr_t ab = reinterpret_cast<uintptr_t>(chars + p);
    const uintptr_t a16 = ab & ~(uintptr_t)15;
    const unsigned off = (unsigned)(ab - a16);  // 0..15
    const unsigned sh = (off & 7u) * 8u;
    const bool upper = off >= 8;                // the first window starts in the upper word
    const unsigned need = 8u * ((off >> 3) + cnt + 1);  // bytes of words used, from a16
    const int64_t base = (int64_t)(a16 - reinterpret_cast<uintptr_t>(chars));
    uint64_t wd[2 * NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const int64_t r = base + 16 * i;  // arena position of the vector's first byte
        uint64_t x = 0, y = 0;
        if ((unsigned)(16 * i) < need && r < (int64_t)nchars) {
            const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(a16 + 16 * i));
            x = v.x;
            y = v.y;
            const int64_t left = (int64_t)nchars - r;  // its bytes inside the arena
            if (left < 16) {
                if (left <= 8) {
                    x &= ~0ull >> (64u - 8u * (unsigned)left);
                    y = 0;
                } else {
                    y &= ~0ull >> (64u - 8u * (unsigned)(left - 8));
                }
            }
        }
        wd[2 * i] = x;
        wd[2 * i + 1] = y;
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const uint64_t lo = upper ? wd[i + 1] : wd[i];
        const uint64_t hi = upper ? wd[i + 2] : wd[i + 1];
        raw[i] = (uint32_t)i < cnt ? (sh ? ((lo >> sh) | (hi << (64u - sh))) : lo) : 0ull;
    }
}

// Big-endian key of a raw window: chars after its first NUL read as NUL.
__device__ __forceinline__ uint64_t finish_key(uint64_t raw)
{
    const uint64_t z = (raw - 0x0101010101010101ull) & ~raw & 0x8080808080808080ull;
    if (z) {
        const unsigned nb = (unsigned)(__ffsll((long long)z) - 1) >> 3;
        raw = nb ? (raw & (~0ull >> (64u - 8u * nb))) : 0ull;
    }
    return bswap64(raw);
}

__device__ __forceinline__ uint64_t gather_key(const uint8_t* __restrict__ chars,
                                               uint64_t nchars,
                                               const uint64_t* __restrict__ offs,
                                               uint32_t id, uint32_t depth)
{
    return load_key(chars, nchars, __ldg(offs + id) + depth);
}

// chars shared by two keys (8 when equal)
__device__ __forceinline__ uint32_t lcp_key_type(uint64_t a, uint64_t b)
{
    const uint64_t x = a ^ b;
    return x ? (uint32_t)__clzll((long long)x) >> 3 : 8u;
}

// number of non-NUL chars in a key
__device__ __forceinline__ uint32_t lcp_key_depth(uint64_t a)
{
    return a ? 8u - ((uint32_t)(__ffsll((long long)a) - 1) >> 3) : 0u;
}

__device__ __forceinline__ bool key_terminated(uint64_t k) { return (k & 0xFFu) == 0; }

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    // splitmix64 finaliser: deterministic sample positions
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ void set_error(uint32_t* err, uint32_t bit)
{
    atomicOr(err, bit);
}

}  // namespace pssgpu
