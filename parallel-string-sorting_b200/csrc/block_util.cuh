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

// In-place ascending bitonic sort of S (a power of two) keys in shared
// memory by the whole block; synchronises before returning.
__device__ __forceinline__ void bitonic_sort_block(uint64_t* a, uint32_t S)
{
    for (uint32_t kk = 2; kk <= S; kk <<= 1) {
        for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < S / 2; i += blockDim.x) {
                const uint32_t x0 = 2 * i - (i & (j - 1));
                const uint32_t x1 = x0 + j;
                const bool asc = (x0 & kk) == 0;
                const uint64_t x = a[x0], y = a[x1];
                if ((x > y) == asc) { a[x0] = y; a[x1] = x; }
            }
            __syncthreads();
        }
    }
}

}  // namespace pssgpu
