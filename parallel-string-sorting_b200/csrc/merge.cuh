// merge.cuh -- merge of K sorted runs of one arena into one sorted run with
// its LCP array: the step after per-shard sorts that the reference takes in
// its top-level merge of per-NUMA-node pS5 outputs
// (src/parallel/eberle-ps5-parallel-toplevel-merge.hpp:56-175, the
// LCP-aware K-way merge of src/parallel/eberle-parallel-lcp-merge*.hpp over
// src/sequential/bingmann-lcp_losertree.hpp).
//
// Here the runs merge pairwise, ceil(log2 K) rounds of three launches: the
// merge-path split of every piece of MERGE_PIECE outputs, the sequential
// merge of each piece by one thread (equal strings keep the left run
// first), then every merged position takes its LCP from the input when its
// predecessor was its predecessor in the same input run, else from
// comparing the two strings.
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

// Merge-path form of a round. A pair is (a0, a1, b1): left run [a0, a1),
// right run [a1, b1) (empty for an unpaired last run), merged into [a0, b1).
// Its output is cut into pieces of MERGE_PIECE positions; task t of the
// round is piece t - first[pair] of its pair. k_merge_split finds for every
// piece how many left-run strings precede it (a binary search along the
// piece's diagonal), k_merge_seq merges each piece sequentially from there.
constexpr uint32_t MERGE_PIECE = 32;

struct MergePair {
    uint64_t a0, a1, b1;
};

__device__ __forceinline__ uint32_t pair_of(const uint64_t* first, uint32_t npair, uint64_t t)
{
    uint32_t lo = 0, hi = npair;  // first[lo] <= t < first[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (first[mid] <= t) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void k_merge_split(const uint8_t* __restrict__ chars, uint64_t nchars,
                              const uint64_t* __restrict__ offs, const MergePair* __restrict__ pairs,
                              const uint64_t* __restrict__ first, uint32_t npair,
                              const uint32_t* __restrict__ ids_in, uint64_t* __restrict__ split)
{
    const uint64_t ntask = first[npair];
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = pair_of(first, npair, t);
        const MergePair pr = pairs[p];
        const uint64_t na = pr.a1 - pr.a0, nb = pr.b1 - pr.a1;
        const uint64_t d = (t - first[p]) * MERGE_PIECE;
        // left-run strings among the first d outputs: the first i with
        // A[i] > B[d - i - 1] (ties go to the left run)
        uint64_t lo = d > nb ? d - nb : 0, hi = min(d, na);
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            uint32_t l;
            const int c = compare_lcp(chars, nchars, __ldg(offs + ids_in[pr.a0 + mid]),
                                      __ldg(offs + ids_in[pr.a1 + d - mid - 1]), &l);
            if (c <= 0) lo = mid + 1; else hi = mid;
        }
        split[t] = lo;
    }
}

__global__ void k_merge_seq(const uint8_t* __restrict__ chars, uint64_t nchars,
                            const uint64_t* __restrict__ offs, const MergePair* __restrict__ pairs,
                            const uint64_t* __restrict__ first, uint32_t npair,
                            const uint64_t* __restrict__ split, const uint32_t* __restrict__ ids_in,
                            uint32_t* __restrict__ ids_out, uint32_t* __restrict__ src)
{
    const uint64_t ntask = first[npair];
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = pair_of(first, npair, t);
        const MergePair pr = pairs[p];
        const uint64_t na = pr.a1 - pr.a0, nb = pr.b1 - pr.a1;
        const uint64_t d0 = (t - first[p]) * MERGE_PIECE;
        const uint64_t d1 = min(d0 + MERGE_PIECE, na + nb);
        const uint64_t i0 = split[t];
        const uint64_t i1 = t + 1 < first[p + 1] ? split[t + 1] : na;
        uint64_t i = i0, j = d0 - i0;
        const uint64_t j1 = d1 - i1;
        for (uint64_t d = d0; d < d1; ++d) {
            bool take_a;
            if (i >= i1) take_a = false;
            else if (j >= j1) take_a = true;
            else {
                uint32_t l;
                take_a = compare_lcp(chars, nchars, __ldg(offs + ids_in[pr.a0 + i]),
                                     __ldg(offs + ids_in[pr.a1 + j]), &l) <= 0;
            }
            const uint64_t q = take_a ? pr.a0 + i : pr.a1 + j;
            ids_out[pr.a0 + d] = ids_in[q];
            src[pr.a0 + d] = (uint32_t)q;
            if (take_a) ++i; else ++j;
        }
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
