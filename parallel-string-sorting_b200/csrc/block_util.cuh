// block_util.cuh -- block-wide scans used by the sort kernels.
#pragma once

#include <cstdint>

namespace pssgpu {

__device__ __forceinline__ uint32_t warp_incl_sum(uint32_t x)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

__device__ __forceinline__ uint32_t warp_incl_max(uint32_t x)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, y);
    }
    return x;
}

// Exclusive block sum of one value per thread. tmp holds >= 32 words. All
// threads of the block must call; tmp is reusable on return.
template <int THREADS>
__device__ __forceinline__ uint32_t block_excl_sum(uint32_t v, uint32_t* tmp, uint32_t* total)
{
    constexpr int NW = THREADS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t incl = warp_incl_sum(v);
    if (lane == 31) tmp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < NW ? tmp[lane] : 0u;
        t = warp_incl_sum(t);
        if (lane < NW) tmp[lane] = t;
    }
    __syncthreads();
    const uint32_t prefix = wid ? tmp[wid - 1] : 0u;
    if (total) *total = tmp[NW - 1];
    __syncthreads();
    return prefix + incl - v;
}

// Exclusive block max (identity 0) of one value per thread.
template <int THREADS>
__device__ __forceinline__ uint32_t block_excl_max(uint32_t v, uint32_t* tmp)
{
    constexpr int NW = THREADS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t incl = warp_incl_max(v);
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = 0;
    if (lane == 31) tmp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < NW ? tmp[lane] : 0u;
        t = warp_incl_max(t);
        if (lane < NW) tmp[lane] = t;
    }
    __syncthreads();
    const uint32_t prefix = wid ? tmp[wid - 1] : 0u;
    __syncthreads();
    return max(prefix, excl);
}

// In-place exclusive scan of a[0, N) in shared memory; returns the total.
// Every thread owns a contiguous chunk. Caller synchronises before the call.
template <int THREADS>
__device__ __forceinline__ uint32_t block_scan_array(uint32_t* a, int N, uint32_t* tmp)
{
    const int per = (N + THREADS - 1) / THREADS;
    const int lo = min((int)threadIdx.x * per, N), hi = min(lo + per, N);
    uint32_t s = 0;
    for (int i = lo; i < hi; ++i) s += a[i];
    uint32_t total;
    uint32_t run = block_excl_sum<THREADS>(s, tmp, &total);
    for (int i = lo; i < hi; ++i) {
        const uint32_t v = a[i];
        a[i] = run;
        run += v;
    }
    __syncthreads();
    return total;
}

// Compiler fence that pins the values of v in registers at this point: the
// loads that produced them are issued (all in flight at once) before any
// memory access that follows.
template <int N>
__device__ __forceinline__ void hold_loaded(uint32_t (&v)[N])
{
    static_assert(N % 8 == 0, "multiple of 8");
#pragma unroll
    for (int i = 0; i < N; i += 8)
        asm volatile("" : "+r"(v[i]), "+r"(v[i + 1]), "+r"(v[i + 2]), "+r"(v[i + 3]), "+r"(v[i + 4]),
                     "+r"(v[i + 5]), "+r"(v[i + 6]), "+r"(v[i + 7])::"memory");
}

template <int N>
__device__ __forceinline__ void hold_loaded64(uint64_t (&v)[N])
{
    static_assert(N % 4 == 0, "multiple of 4");
#pragma unroll
    for (int i = 0; i < N; i += 4)
        asm volatile("" : "+l"(v[i]), "+l"(v[i + 1]), "+l"(v[i + 2]), "+l"(v[i + 3])::"memory");
}

// Bitonic stages (kk, j) with j <= 32 for kk in [kk_from, kk_to], on every
// 64-key chunk of a[0, S) in registers: each warp takes whole chunks, two
// keys per lane (positions e0 = 64 c + 2 lane and e0 + 1), partners by
// shuffle. Directions follow the global positions, as in the full network.
__device__ __forceinline__ void bitonic_chunk_stages(uint64_t* a, uint32_t S, uint32_t kk_from,
                                                     uint32_t kk_to)
{
    const uint32_t lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (uint32_t c = threadIdx.x >> 5; c < S / 64; c += nw) {
        const uint32_t e0 = c * 64 + 2 * lane;
        uint64_t x0 = a[e0], x1 = a[e0 + 1];
        for (uint32_t kk = kk_from; kk <= kk_to; kk <<= 1) {
            const bool asc = (e0 & kk) == 0;  // e0 and e0 + 1 agree for kk >= 2
            for (uint32_t j = min(kk >> 1, 32u); j > 0; j >>= 1) {
                if (j == 1) {
                    const uint64_t lo = min(x0, x1), hi = max(x0, x1);
                    x0 = asc ? lo : hi;
                    x1 = asc ? hi : lo;
                } else {
                    const uint64_t y0 = __shfl_xor_sync(0xffffffffu, x0, j >> 1);
                    const uint64_t y1 = __shfl_xor_sync(0xffffffffu, x1, j >> 1);
                    const bool keep_min = ((e0 & j) == 0) == asc;
                    x0 = keep_min ? min(x0, y0) : max(x0, y0);
                    x1 = keep_min ? min(x1, y1) : max(x1, y1);
                }
            }
        }
        a[e0] = x0;
        a[e0 + 1] = x1;
    }
}

// In-place ascending bitonic sort of S (a power of two) keys in shared
// memory by the whole block (a multiple of 32 threads); synchronises before
// returning. Partner distances of 64 and more go through shared memory with
// a barrier per stage, shorter ones run in registers inside a warp.
__device__ __forceinline__ void bitonic_sort_block(uint64_t* a, uint32_t S)
{
    auto smem_stage = [&](uint32_t kk, uint32_t j) {
        for (uint32_t i = threadIdx.x; i < S / 2; i += blockDim.x) {
            const uint32_t x0 = 2 * i - (i & (j - 1));
            const uint32_t x1 = x0 + j;
            const bool asc = (x0 & kk) == 0;
            const uint64_t x = a[x0], y = a[x1];
            if ((x > y) == asc) { a[x0] = y; a[x1] = x; }
        }
        __syncthreads();
    };
    if (S < 64) {
        for (uint32_t kk = 2; kk <= S; kk <<= 1)
            for (uint32_t j = kk >> 1; j > 0; j >>= 1) smem_stage(kk, j);
        return;
    }
    bitonic_chunk_stages(a, S, 2, 64);
    __syncthreads();
    for (uint32_t kk = 128; kk <= S; kk <<= 1) {
        for (uint32_t j = kk >> 1; j >= 64; j >>= 1) smem_stage(kk, j);
        bitonic_chunk_stages(a, S, kk, kk);
        __syncthreads();
    }
}

// Ascending bitonic sort of a[0, S) (S a power of two, at least 64) by the
// whole block, where a[m, S) holds padding larger than every key (m >= 1).
// Every compare-exchange puts the smaller key at the lower position, and each
// merge of 2^k keys starts by comparing every position with its mirror in the
// merged block (the network without descending halves), so the padding never
// moves: pairs that reach into it are skipped, and so are the 64-key chunks
// that hold only padding. A group of m keys just above a power of two costs
// little more than the power of two below it. Synchronises before returning.
__device__ __forceinline__ void bitonic_sort_block_padded(uint64_t* a, uint32_t S, uint32_t m)
{
    const uint32_t lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const uint32_t nch = (m + 63) / 64;  // chunks holding keys
    // register stages of one chunk: merges of 2..min(64, kk_to) keys in full
    // (tail = false), or the steps of partner distance 32..1 (tail = true)
    auto chunks = [&](uint32_t kk_to, bool tail) {
        for (uint32_t c = threadIdx.x >> 5; c < nch; c += nw) {
            const uint32_t e0 = c * 64 + 2 * lane;
            uint64_t x0 = a[e0], x1 = a[e0 + 1];
            auto step = [&](uint32_t j) {  // partner distance j, ascending
                if (j == 1) {
                    const uint64_t lo = min(x0, x1), hi = max(x0, x1);
                    x0 = lo;
                    x1 = hi;
                } else {
                    const uint64_t y0 = __shfl_xor_sync(0xffffffffu, x0, j >> 1);
                    const uint64_t y1 = __shfl_xor_sync(0xffffffffu, x1, j >> 1);
                    const bool keep_min = (lane & (j >> 1)) == 0;
                    x0 = keep_min ? min(x0, y0) : max(x0, y0);
                    x1 = keep_min ? min(x1, y1) : max(x1, y1);
                }
            };
            if (tail) {
#pragma unroll
                for (uint32_t j = 32; j > 0; j >>= 1) step(j);
            } else {
                for (uint32_t kk = 2; kk <= min(64u, kk_to); kk <<= 1) {
                    if (kk == 2) {
                        step(1);
                        continue;
                    }
                    // mirror step: position e pairs with e ^ (kk - 1)
                    const uint32_t mm = (kk >> 1) - 1;
                    const uint64_t y0 = __shfl_xor_sync(0xffffffffu, x1, mm);
                    const uint64_t y1 = __shfl_xor_sync(0xffffffffu, x0, mm);
                    const bool lower = (lane & (kk >> 2)) == 0;
                    x0 = lower ? min(x0, y0) : max(x0, y0);
                    x1 = lower ? min(x1, y1) : max(x1, y1);
                    for (uint32_t j = kk >> 2; j > 0; j >>= 1) step(j);
                }
            }
            a[e0] = x0;
            a[e0 + 1] = x1;
        }
    };
    auto cas = [&](uint32_t x0, uint32_t x1) {
        if (x1 >= m) return;  // padding stays where it is
        const uint64_t x = a[x0], y = a[x1];
        if (x > y) {
            a[x0] = y;
            a[x1] = x;
        }
    };
    chunks(S, false);
    __syncthreads();
    for (uint32_t kk = 128; kk <= S; kk <<= 1) {
        const uint32_t half = kk >> 1;
        for (uint32_t i = threadIdx.x; i < S / 2; i += blockDim.x) {
            const uint32_t blk = i / half, off = i - blk * half;
            cas(blk * kk + off, blk * kk + kk - 1 - off);
        }
        __syncthreads();
        for (uint32_t j = kk >> 2; j >= 64; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < S / 2; i += blockDim.x) {
                const uint32_t x0 = 2 * i - (i & (j - 1));
                cas(x0, x0 + j);
            }
            __syncthreads();
        }
        chunks(0, true);
        __syncthreads();
    }
}

}  // namespace pssgpu
