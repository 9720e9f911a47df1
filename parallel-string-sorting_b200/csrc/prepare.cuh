// prepare.cuh -- device-side input preparation: a text buffer becomes an
// arena and its offset array in HBM, as psstest does it on the host when it
// loads a plain file (src/tools/input.hpp:255-297) and builds the string
// pointer array (src/psstest.cpp:479-518).
//
//   lines     every '\n' and NUL byte of text[0, size) ends a string and
//             becomes NUL; position 0 and every position behind such a byte
//             start a string (input.hpp:279-283, psstest.cpp:483-485), so
//             n = 1 + the separators in text[0, size - 1)
//   suffixes  every position starts a string, n = size (input.hpp:289,
//             psstest.cpp:503-505)
//
// Both force the last byte to NUL (input.hpp:292). Three launches for lines:
// separators per chunk of PREP_CHUNK bytes, a scan of the chunk counts, then
// per chunk the offsets in order and the newline rewrite (8-byte words, one
// thread each; only words that held a newline are written back).
#pragma once

#include "block_util.cuh"

namespace pssgpu {

constexpr int PREP_THREADS = 256;
constexpr uint32_t PREP_CHUNK = 64 * 1024;  // text bytes per block, a multiple of 8 * PREP_THREADS
static_assert(PREP_CHUNK % (8 * PREP_THREADS) == 0, "chunk layout");

// 0xFF in every byte of the little-endian word that is '\n' or NUL
__device__ __forceinline__ uint64_t separator_bytes(uint64_t wd)
{
    const uint32_t lo = (uint32_t)wd, hi = (uint32_t)(wd >> 32);
    const uint32_t ml = __vcmpeq4(lo, 0x0A0A0A0Au) | __vcmpeq4(lo, 0u);
    const uint32_t mh = __vcmpeq4(hi, 0x0A0A0A0Au) | __vcmpeq4(hi, 0u);
    return ((uint64_t)mh << 32) | ml;
}

// separator marks of the word at byte a, restricted to bytes below hi
__device__ __forceinline__ uint64_t separators_below(const uint8_t* text, uint64_t a, uint64_t hi)
{
    uint64_t m = separator_bytes(*reinterpret_cast<const uint64_t*>(text + a));
    if (a + 8 > hi) m &= ~0ull >> (64u - 8u * (unsigned)(hi - a));
    return m;
}

// Separators in chunk blockIdx.x of text[0, size - 1).
__global__ void __launch_bounds__(PREP_THREADS) k_text_count(const uint8_t* __restrict__ text,
                                                            uint64_t size, uint32_t* __restrict__ cnt)
{
    __shared__ uint32_t tmp[32];
    const uint64_t lo = (uint64_t)blockIdx.x * PREP_CHUNK;
    const uint64_t hi = min(size - 1, lo + PREP_CHUNK);
    uint32_t c = 0;
    for (uint64_t a = lo + 8ull * threadIdx.x; a < hi; a += 8ull * PREP_THREADS)
        c += (uint32_t)__popcll(separators_below(text, a, hi)) >> 3;
    uint32_t total;
    block_excl_sum<PREP_THREADS>(c, tmp, &total);
    if (threadIdx.x == 0) cnt[blockIdx.x] = total;
}

// Exclusive scan of the chunk counts (one block); total = all separators.
__global__ void __launch_bounds__(1024) k_text_scan(const uint32_t* __restrict__ cnt, uint32_t nchunk,
                                                   uint64_t* __restrict__ base, uint64_t* __restrict__ total)
{
    __shared__ uint32_t tmp[32];
    uint64_t run = 0;
    for (uint32_t b0 = 0; b0 < nchunk; b0 += 1024) {
        const uint32_t b = b0 + threadIdx.x;
        const uint32_t v = b < nchunk ? cnt[b] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_sum<1024>(v, tmp, &tot);
        if (b < nchunk) base[b] = run + ex;
        run += tot;
    }
    if (threadIdx.x == 0) *total = run;
}

// Offsets of the strings that start behind the separators of chunk
// blockIdx.x (string 0 starts at 0 and is written by the host), and the
// newline rewrite. offs holds at least 1 + all separators entries.
__global__ void __launch_bounds__(PREP_THREADS) k_text_lines(uint8_t* __restrict__ text, uint64_t size,
                                                            const uint64_t* __restrict__ base,
                                                            uint64_t* __restrict__ offs)
{
    __shared__ uint32_t tmp[32];
    const uint64_t lo = (uint64_t)blockIdx.x * PREP_CHUNK;
    const uint64_t hi = min(size - 1, lo + PREP_CHUNK);
    uint64_t run = 1 + base[blockIdx.x];  // index of the string behind the chunk's first separator
    for (uint64_t a0 = lo; a0 < hi; a0 += 8ull * PREP_THREADS) {
        const uint64_t a = a0 + 8ull * threadIdx.x;
        uint64_t wd = 0, m = 0;
        if (a < hi) {
            wd = *reinterpret_cast<const uint64_t*>(text + a);
            m = separator_bytes(wd);
            if (a + 8 > hi) m &= ~0ull >> (64u - 8u * (unsigned)(hi - a));
        }
        uint32_t total;
        const uint32_t r = block_excl_sum<PREP_THREADS>((uint32_t)__popcll(m) >> 3, tmp, &total);
        uint64_t k = run + r;
        for (uint64_t mm = m; mm; ++k) {
            const uint32_t byte = (uint32_t)(__ffsll((long long)mm) - 1) >> 3;
            offs[k] = a + byte + 1;
            mm &= ~(0xFFull << (8 * byte));
        }
        // newlines become NUL (NUL bytes stay); bytes at and beyond hi keep
        // their values
        if (wd & m) *reinterpret_cast<uint64_t*>(text + a) = wd & ~m;
        run += total;
    }
}

// Suffix offsets: every position.
__global__ void k_text_suffixes(uint64_t* __restrict__ offs, uint64_t size)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size;
         i += (uint64_t)gridDim.x * blockDim.x)
        offs[i] = i;
}

// Offsets rebuilt from gaps. A host offset array that never decreases
// crosses PCIe as its gaps g[0] = 0, g[i] = offs[i] - offs[i-1] in 1 or 2
// bytes each; offs[i] = offs[0] + g[0] + ... + g[i]. Per chunk of
// GAP_CHUNK gaps (GAP_THREADS threads, GAP_PER contiguous gaps each): the
// chunk sum (k_gap_sum), the scan of the chunk sums (k_text_scan), then the
// offsets of the chunk (k_gap_offsets). The gap buffer is zero-padded to a
// whole number of chunks.
constexpr int GAP_THREADS = 256;
constexpr int GAP_PER = 32;
constexpr uint32_t GAP_CHUNK = GAP_THREADS * GAP_PER;

template <class T>
__device__ __forceinline__ void load_gaps(const T* __restrict__ g, uint32_t (&v)[GAP_PER])
{
    static_assert(sizeof(T) * GAP_PER % 16 == 0, "whole 16-byte vectors");
    constexpr int NV = (int)(sizeof(T) * GAP_PER / 16);
    const uint4* p = reinterpret_cast<const uint4*>(g);
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        const uint4 x = __ldg(p + q);
        const uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (sizeof(T) == 1) {
#pragma unroll
                for (int b = 0; b < 4; ++b) v[16 * q + 4 * k + b] = (w[k] >> (8 * b)) & 0xFFu;
            } else {
                v[8 * q + 2 * k] = w[k] & 0xFFFFu;
                v[8 * q + 2 * k + 1] = w[k] >> 16;
            }
        }
    }
}

template <class T>
__global__ void __launch_bounds__(GAP_THREADS) k_gap_sum(const T* __restrict__ gaps, uint32_t* __restrict__ cnt)
{
    __shared__ uint32_t tmp[32];
    uint32_t v[GAP_PER];
    load_gaps<T>(gaps + (size_t)blockIdx.x * GAP_CHUNK + (size_t)threadIdx.x * GAP_PER, v);
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < GAP_PER; ++j) s += v[j];
    uint32_t total;
    block_excl_sum<GAP_THREADS>(s, tmp, &total);
    if (threadIdx.x == 0) cnt[blockIdx.x] = total;
}

template <class T>
__global__ void __launch_bounds__(GAP_THREADS) k_gap_offsets(const T* __restrict__ gaps, uint64_t n, uint64_t first,
                                                             const uint64_t* __restrict__ base,
                                                             uint64_t* __restrict__ offs)
{
    __shared__ uint32_t tmp[32];
    const uint64_t i0 = (uint64_t)blockIdx.x * GAP_CHUNK + (uint64_t)threadIdx.x * GAP_PER;
    uint32_t v[GAP_PER];
    load_gaps<T>(gaps + i0, v);
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < GAP_PER; ++j) s += v[j];
    uint64_t run = first + base[blockIdx.x] + block_excl_sum<GAP_THREADS>(s, tmp, nullptr);
    if (i0 + GAP_PER <= n) {
        ulonglong2* o = reinterpret_cast<ulonglong2*>(offs + i0);
#pragma unroll
        for (int j = 0; j < GAP_PER; j += 2) {
            const uint64_t a = run + v[j];
            run = a + v[j + 1];
            o[j / 2] = make_ulonglong2(a, run);
        }
    } else {
#pragma unroll
        for (int j = 0; j < GAP_PER; ++j) {
            run += v[j];
            if (i0 + j < n) offs[i0 + j] = run;
        }
    }
}

}  // namespace pssgpu
