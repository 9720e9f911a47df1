// merge.cuh -- merge of K sorted runs of one arena into one sorted run with
// its LCP array: the step after per-shard sorts that the reference takes in
// its top-level merge of per-NUMA-node pS5 outputs
// (src/parallel/eberle-ps5-parallel-toplevel-merge.hpp:56-175, the
// LCP-aware K-way merge of src/parallel/eberle-parallel-lcp-merge*.hpp over
// src/sequential/bingmann-lcp_losertree.hpp).
//
// Here the runs merge pairwise, ceil(log2 K) rounds, each a fixed number of
// launches: every string finds its place in the merged pair by a binary
// search of the partner run (its own rank plus the partner's strings that
// precede it: strictly smaller for the left run, smaller or equal for the
// right one, so equal strings keep the left run first), then every merged
// position takes its LCP from the input when its predecessor was its
// predecessor in the same input run, else from comparing the two strings.
#pragma once

#include "device_common.cuh"

namespace pssgpu {

// Order and LCP of strings a and b (arena offsets oa, ob), 8 chars a step.
__device__ __forceinline__ int compare_lcp(const uint8_t* chars, uint64_t nchars, uint64_t oa,
                                           uint64_t ob, uint32_t* lcp)
{
    uint32_t d = 0;
    while (true) {
        const uint64_t ka = load_key(chars, nchars, oa + d), kb = load_key(chars, nchars, ob + d);
        if (ka != kb) {
            *lcp = d + lcp_key_type(ka, kb);
            return ka < kb ? -1 : 1;
        }
        if (key_terminated(ka)) {
            *lcp = d + lcp_key_depth(ka);
            return 0;
        }
        d += 8;
    }
}

// run r of the K runs with boundaries runs[0..K] that holds position q: the
// last r with runs[r] <= q (runs[K] > q)
__device__ __forceinline__ uint32_t run_of(const uint64_t* runs, uint32_t K, uint64_t q)
{
    uint32_t lo = 0, hi = K;  // runs[lo] <= q < runs[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (runs[mid] <= q) lo = mid; else hi = mid;
    }
    return lo;
}

// One round: runs 2p and 2p + 1 of ids_in merge into [runs[2p], runs[2p+2])
// of ids_out; src[pos] = the input position of the string placed at pos. An
// unpaired last run is copied.
__global__ void k_merge_place(const uint8_t* __restrict__ chars, uint64_t nchars,
                              const uint64_t* __restrict__ offs, const uint64_t* __restrict__ runs,
                              uint32_t K, const uint32_t* __restrict__ ids_in,
                              uint32_t* __restrict__ ids_out, uint32_t* __restrict__ src, uint64_t n)
{
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = run_of(runs, K, q);
        const uint32_t x = ids_in[q];
        uint64_t pos = q;
        if ((r | 1u) < K) {  // the pair is complete
            const uint64_t a0 = runs[r & ~1u], a1 = runs[(r & ~1u) + 1], b1 = runs[(r & ~1u) + 2];
            const uint64_t ox = __ldg(offs + x);
            uint32_t l;
            if (!(r & 1u)) {
                // left run: right-run strings strictly smaller than x
                uint64_t lo = a1, hi = b1;
                while (lo < hi) {
                    const uint64_t mid = (lo + hi) >> 1;
                    if (compare_lcp(chars, nchars, __ldg(offs + ids_in[mid]), ox, &l) < 0) lo = mid + 1;
                    else hi = mid;
                }
                pos = q + (lo - a1);
            } else {
                // right run: left-run strings smaller than or equal to x
                uint64_t lo = a0, hi = a1;
                while (lo < hi) {
                    const uint64_t mid = (lo + hi) >> 1;
                    if (compare_lcp(chars, nchars, __ldg(offs + ids_in[mid]), ox, &l) <= 0) lo = mid + 1;
                    else hi = mid;
                }
                pos = a0 + (q - a1) + (lo - a0);
            }
        }
        ids_out[pos] = x;
        src[pos] = (uint32_t)q;
    }
}

// LCPs of a round's output: runs_out are the merged runs (no LCP at their
// first position), runs_in the runs merged.
__global__ void k_merge_lcp(const uint8_t* __restrict__ chars, uint64_t nchars,
                            const uint64_t* __restrict__ offs, const uint64_t* __restrict__ runs_in,
                            uint32_t K_in, const uint64_t* __restrict__ runs_out, uint32_t K_out,
                            const uint32_t* __restrict__ ids_out, const uint32_t* __restrict__ src,
                            const uint32_t* __restrict__ lcp_in, uint32_t* __restrict__ lcp_out,
                            uint64_t n)
{
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (uint64_t)gridDim.x * blockDim.x) {
        if (runs_out[run_of(runs_out, K_out, p)] == p) continue;  // first of a merged run
        const uint32_t s0 = src[p - 1], s1 = src[p];
        if (s1 == s0 + 1 && runs_in[run_of(runs_in, K_in, s1)] != s1) {
            lcp_out[p] = lcp_in[s1];  // neighbours in the same input run
        } else {
            uint32_t l;
            compare_lcp(chars, nchars, __ldg(offs + ids_out[p - 1]), __ldg(offs + ids_out[p]), &l);
            lcp_out[p] = l;
        }
    }
}

}  // namespace pssgpu
