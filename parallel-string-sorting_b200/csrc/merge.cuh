// merge.cuh -- merge of K sorted runs of one arena into one sorted run with
// its LCP array: the step after per-shard sorts that the reference takes in
// its top-level merge of per-NUMA-node pS5 outputs
// (src/parallel/eberle-ps5-parallel-toplevel-merge.hpp:56-175, the
// LCP-aware K-way merge of src/parallel/eberle-parallel-lcp-merge*.hpp over
// src/sequential/bingmann-lcp_losertree.hpp).
//
// Here the runs merge pairwise, ceil(log2 K) rounds of two launches: the
// merge-path split of every piece of MERGE_PIECE outputs, then the merge of
// each piece by one thread. With the runs' LCP arrays the piece merge is
// LCP-aware, as the reference's loser tree is
// (src/sequential/bingmann-lcp_losertree.hpp:61-110, 156-185): each head
// carries its LCP with the last output, the head with the larger one is the
// smaller string without reading a char, equal ones compare from that depth
// only, and every output's LCP falls out of the same step.
#pragma once

#include "device_common.cuh"

namespace pssgpu {

// Order and LCP of strings a and b (arena offsets oa, ob) that share at
// least d chars, 8 chars a step from d.
__device__ __forceinline__ int compare_from(const uint8_t* chars, uint64_t nchars, uint64_t oa,
                                            uint64_t ob, uint32_t d, uint32_t* lcp)
{
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

__device__ __forceinline__ int compare_lcp(const uint8_t* chars, uint64_t nchars, uint64_t oa,
                                           uint64_t ob, uint32_t* lcp)
{
    return compare_from(chars, nchars, oa, ob, 0, lcp);
}

// Merge-path form of a round. A pair is (a0, a1, b1): left run [a0, a1),
// right run [a1, b1) (empty for an unpaired last run), merged into [a0, b1).
// Its output is cut into pieces of `piece` positions (MERGE_PIECE by
// default); task t of the round is piece t - first[pair] of its pair. k_merge_split finds for every
// piece how many left-run strings precede it (a binary search along the
// piece's diagonal), k_merge_lcp_seq (or k_merge_seq without LCP arrays)
// merges each piece sequentially from there.
constexpr uint32_t MERGE_PIECE = 128;
constexpr uint32_t MERGE_PIECE_MAX = 4096;

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

// Splits in two launches: coarse = 1 searches every MERGE_SPLIT_COARSE-th
// piece of a pair over the whole diagonal; coarse = 0 searches the other
// pieces between the two coarse splits around them. The merge path is a
// monotone staircase, so for a diagonal d between coarse diagonals D0 < D1
// with splits i0, i1: i0 <= i(d) <= i1 and d - D1 + i1 <= i(d) <= d - D0 + i0,
// a window of at most MERGE_SPLIT_COARSE * piece positions.
constexpr uint32_t MERGE_SPLIT_COARSE = 32;

__global__ void k_merge_split(const uint8_t* __restrict__ chars, uint64_t nchars,
                              const uint64_t* __restrict__ offs, const MergePair* __restrict__ pairs,
                              const uint64_t* __restrict__ first, uint32_t npair,
                              const uint32_t* __restrict__ ids_in, uint64_t* __restrict__ split,
                              uint32_t piece, int coarse)
{
    const uint64_t ntask = first[npair];
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = pair_of(first, npair, t);
        const uint64_t k = t - first[p];
        if ((k % MERGE_SPLIT_COARSE == 0) != (coarse != 0)) continue;
        const MergePair pr = pairs[p];
        const uint64_t na = pr.a1 - pr.a0, nb = pr.b1 - pr.a1;
        const uint64_t d = k * piece;
        // left-run strings among the first d outputs: the first i with
        // A[i] > B[d - i - 1] (ties go to the left run)
        int64_t lo = d > nb ? (int64_t)(d - nb) : 0, hi = (int64_t)min(d, na);
        if (!coarse) {
            const uint64_t k0 = k - k % MERGE_SPLIT_COARSE, k1 = k0 + MERGE_SPLIT_COARSE;
            const uint64_t D0 = k0 * piece, i0 = split[first[p] + k0];
            const bool last = first[p] + k1 >= first[p + 1];
            const uint64_t D1 = last ? na + nb : k1 * piece, i1 = last ? na : split[first[p] + k1];
            lo = max(lo, max((int64_t)i0, (int64_t)d - (int64_t)D1 + (int64_t)i1));
            hi = min(hi, min((int64_t)i1, (int64_t)(d - D0 + i0)));
        }
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            uint32_t l;
            const int c = compare_lcp(chars, nchars, __ldg(offs + ids_in[pr.a0 + mid]),
                                      __ldg(offs + ids_in[pr.a1 + d - mid - 1]), &l);
            if (c <= 0) lo = mid + 1; else hi = mid;
        }
        split[t] = (uint64_t)lo;
    }
}

// Piece merge without LCP arrays: every pair compares from char 0.
__global__ void k_merge_seq(const uint8_t* __restrict__ chars, uint64_t nchars,
                            const uint64_t* __restrict__ offs, const MergePair* __restrict__ pairs,
                            const uint64_t* __restrict__ first, uint32_t npair,
                            const uint64_t* __restrict__ split, const uint32_t* __restrict__ ids_in,
                            uint32_t* __restrict__ ids_out, uint32_t piece)
{
    const uint64_t ntask = first[npair];
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = pair_of(first, npair, t);
        const MergePair pr = pairs[p];
        const uint64_t na = pr.a1 - pr.a0, nb = pr.b1 - pr.a1;
        const uint64_t d0 = (t - first[p]) * piece;
        const uint64_t d1 = min(d0 + piece, na + nb);
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
            ids_out[pr.a0 + d] = take_a ? ids_in[pr.a0 + i] : ids_in[pr.a1 + j];
            if (take_a) ++i; else ++j;
        }
    }
}

// Sequential reads of a u32 array 16 bytes at a time: a thread that walks
// its own stretch of ids or LCPs keeps the last aligned 4-word block in
// registers instead of fetching a sector per word (the threads' streams are
// too many for the caches to keep their lines). The array must be 16-byte
// aligned and readable up to the next multiple of 4 words past its end.
struct SeqRead4 {
    const uint32_t* base;
    uint64_t blk = ~0ull;
    uint4 v{};
    __device__ __forceinline__ uint32_t get(uint64_t i)
    {
        const uint64_t b = i >> 2;
        if (b != blk) {
            v = __ldg(reinterpret_cast<const uint4*>(base + (b << 2)));
            blk = b;
        }
        const uint32_t k = (uint32_t)(i & 3);
        return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w;
    }
};

// LCP-aware piece merge (the reference's LCP loser-tree rule for two runs).
// Runs A = ids_in[a0, a1) and B = ids_in[a1, b1) with their LCP arrays in
// lcp_in (entries at a run's first position are not read). ha / hb are the
// LCPs of the heads A[i] / B[j] with the last output. A piece that does not
// start the pair first finds its previous output (the larger of A[i0 - 1]
// and B[j0 - 1]; equal strings: B's, as A's comes first) and the heads' LCPs
// with it. lcp_out (may be null) receives the LCP of every output but the
// pair's first.
__global__ void k_merge_lcp_seq(const uint8_t* __restrict__ chars, uint64_t nchars,
                                const uint64_t* __restrict__ offs,
                                const MergePair* __restrict__ pairs,
                                const uint64_t* __restrict__ first, uint32_t npair,
                                const uint64_t* __restrict__ split,
                                const uint32_t* __restrict__ ids_in,
                                const uint32_t* __restrict__ lcp_in,
                                uint32_t* __restrict__ ids_out, uint32_t* __restrict__ lcp_out,
                                uint32_t piece)
{
    const uint64_t ntask = first[npair];
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = pair_of(first, npair, t);
        const MergePair pr = pairs[p];
        const uint64_t na = pr.a1 - pr.a0, nb = pr.b1 - pr.a1;
        const uint32_t* A = ids_in + pr.a0;
        const uint32_t* B = ids_in + pr.a1;
        const uint32_t* LA = lcp_in + pr.a0;
        const uint32_t* LB = lcp_in + pr.a1;
        const uint64_t d0 = (t - first[p]) * piece;
        const uint64_t d1 = min(d0 + piece, na + nb);
        const uint64_t i0 = split[t];
        const uint64_t i1 = t + 1 < first[p + 1] ? split[t + 1] : na;
        const uint64_t j0 = d0 - i0, j1 = d1 - i1;
        uint64_t i = i0, j = j0;
        uint32_t ha = 0, hb = 0;
        if (d0 > 0) {
            if (i0 == 0) {  // previous output B[j0 - 1]
                hb = j < nb ? LB[j] : 0u;
                if (i < na) compare_from(chars, nchars, __ldg(offs + A[i]), __ldg(offs + B[j - 1]), 0, &ha);
            } else if (j0 == 0) {  // previous output A[i0 - 1]
                ha = i < na ? LA[i] : 0u;
                if (j < nb) compare_from(chars, nchars, __ldg(offs + B[j]), __ldg(offs + A[i - 1]), 0, &hb);
            } else {
                uint32_t l;
                const int c = compare_from(chars, nchars, __ldg(offs + A[i - 1]),
                                           __ldg(offs + B[j - 1]), 0, &l);
                // LCP(x, z) >= min(LCP(x, y), LCP(y, z)): start from that depth
                if (c <= 0) {  // previous output B[j0 - 1]
                    hb = j < nb ? LB[j] : 0u;
                    if (i < na)
                        compare_from(chars, nchars, __ldg(offs + A[i]), __ldg(offs + B[j - 1]),
                                     min(LA[i], l), &ha);
                } else {       // previous output A[i0 - 1]
                    ha = i < na ? LA[i] : 0u;
                    if (j < nb)
                        compare_from(chars, nchars, __ldg(offs + B[j]), __ldg(offs + A[i - 1]),
                                     min(LB[j], l), &hb);
                }
            }
        }
        // the heads' ids and arena offsets stay in registers: one offset
        // load per output, and a compare reads chars only; the runs' ids and
        // LCPs are read 16 bytes at a time
        SeqRead4 ra{ids_in}, rb{ids_in}, la{lcp_in}, lb{lcp_in};
        uint32_t ida = i < i1 ? ra.get(pr.a0 + i) : 0u, idb = j < j1 ? rb.get(pr.a1 + j) : 0u;
        uint64_t oa = i < i1 ? __ldg(offs + ida) : 0ull, ob = j < j1 ? __ldg(offs + idb) : 0ull;
        for (uint64_t d = d0; d < d1; ++d) {
            bool take_a;
            if (i >= i1) take_a = false;
            else if (j >= j1) take_a = true;
            else if (ha != hb) take_a = ha > hb;
            else {
                uint32_t l;
                take_a = compare_from(chars, nchars, oa, ob, ha, &l) <= 0;
                if (take_a) hb = l; else ha = l;  // the loser's LCP with the new last output
            }
            ids_out[pr.a0 + d] = take_a ? ida : idb;
            if (lcp_out && d > 0) lcp_out[pr.a0 + d] = take_a ? ha : hb;
            if (take_a) {
                ++i;
                ha = i < na ? la.get(pr.a0 + i) : 0u;  // against its predecessor, the last output
                if (i < i1) {
                    ida = ra.get(pr.a0 + i);
                    oa = __ldg(offs + ida);
                }
            } else {
                ++j;
                hb = j < nb ? lb.get(pr.a1 + j) : 0u;
                if (j < j1) {
                    idb = rb.get(pr.a1 + j);
                    ob = __ldg(offs + idb);
                }
            }
        }
    }
}

// Every id's offset must lie inside the arena (offsets >= nchars: *err).
__global__ void k_merge_check(const uint64_t* __restrict__ offs, uint64_t nchars,
                              const uint32_t* __restrict__ ids, uint64_t n, uint32_t* err)
{
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (uint64_t)gridDim.x * blockDim.x)
        if (__ldg(offs + ids[q]) >= nchars) atomicOr(err, ERR_OFFSET);
}

}  // namespace pssgpu
