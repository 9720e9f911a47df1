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

// How a round reads its runs. MergeByIds: the entries are string ids and
// a string's arena offset is gathered through offs at each use.
// MergeByHandles: the entries are handles (id << hbits | offset), made once
// by k_merge_pack, so the offset comes with the entry a round reads in order
// and no round gathers offsets.
struct MergeByIds {
    using T = uint32_t;
    const uint64_t* offs;
    __device__ __forceinline__ uint64_t off(uint32_t v) const { return __ldg(offs + v); }
};
struct MergeByHandles {
    using T = uint64_t;
    uint64_t hmask;
    __device__ __forceinline__ uint64_t off(uint64_t v) const { return v & hmask; }
};

// Sequential reads of an array 16 bytes at a time: a thread that walks its
// own stretch of entries or LCPs keeps the last aligned 16-byte block in
// registers instead of fetching a sector per entry (the threads' streams are
// too many for the caches to keep their lines). The array must be 16-byte
// aligned and readable up to the next 16-byte boundary past its end.
template <class T>
struct SeqRead;
template <>
struct SeqRead<uint32_t> {
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
template <>
struct SeqRead<uint64_t> {
    const uint64_t* base;
    uint64_t blk = ~0ull;
    ulonglong2 v{};
    __device__ __forceinline__ uint64_t get(uint64_t i)
    {
        const uint64_t b = i >> 1;
        if (b != blk) {
            v = __ldg(reinterpret_cast<const ulonglong2*>(base + (b << 1)));
            blk = b;
        }
        return (i & 1) ? v.y : v.x;
    }
};
using SeqRead4 = SeqRead<uint32_t>;

// Splits in two launches: coarse = 1 searches every MERGE_SPLIT_COARSE-th
// piece of a pair over the whole diagonal; coarse = 0 searches the other
// pieces between the two coarse splits around them. The merge path is a
// monotone staircase, so for a diagonal d between coarse diagonals D0 < D1
// with splits i0, i1: i0 <= i(d) <= i1 and d - D1 + i1 <= i(d) <= d - D0 + i0,
// a window of at most MERGE_SPLIT_COARSE * piece positions.
constexpr uint32_t MERGE_SPLIT_COARSE = 32;

template <class V>
__global__ void k_merge_split(const uint8_t* __restrict__ chars, uint64_t nchars, V view,
                              const MergePair* __restrict__ pairs,
                              const uint64_t* __restrict__ first, uint32_t npair,
                              const typename V::T* __restrict__ in, uint64_t* __restrict__ split,
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
        uint32_t depth = 0;  // chars every compared pair shares
        if (!coarse) {
            const uint64_t k0 = k - k % MERGE_SPLIT_COARSE, k1 = k0 + MERGE_SPLIT_COARSE;
            const uint64_t D0 = k0 * piece, i0 = split[first[p] + k0];
            const bool last = first[p] + k1 >= first[p + 1];
            const uint64_t D1 = last ? na + nb : k1 * piece, i1 = last ? na : split[first[p] + k1];
            lo = max(lo, max((int64_t)i0, (int64_t)d - (int64_t)D1 + (int64_t)i1));
            hi = min(hi, min((int64_t)i1, (int64_t)(d - D0 + i0)));
            if (hi - lo > 2) {
                // the search compares A[x], x in [lo, hi), with B[y], y in
                // [d - hi, d - lo): a sorted run's extremes share no more
                // than anything between them, so every such pair shares
                // min(LCP(A[lo], A[hi - 1]), LCP(A[lo], B[d - hi]),
                // LCP(B[d - hi], B[d - lo - 1])) chars
                const uint64_t a_lo = view.off(in[pr.a0 + lo]), a_hi = view.off(in[pr.a0 + hi - 1]);
                const uint64_t b_lo = view.off(in[pr.a1 + d - hi]), b_hi = view.off(in[pr.a1 + d - lo - 1]);
                uint32_t l1, l2, l3;
                compare_from(chars, nchars, a_lo, a_hi, 0, &l1);
                compare_from(chars, nchars, b_lo, b_hi, 0, &l2);
                compare_from(chars, nchars, a_lo, b_lo, 0, &l3);
                depth = min(min(l1, l2), l3);
            }
        }
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            uint32_t l;
            const int c = compare_from(chars, nchars, view.off(in[pr.a0 + mid]),
                                       view.off(in[pr.a1 + d - mid - 1]), depth, &l);
            if (c <= 0) lo = mid + 1; else hi = mid;
        }
        split[t] = (uint64_t)lo;
    }
}

// Piece merge without LCP arrays: every pair compares from char 0.
template <class V>
__global__ void k_merge_seq(const uint8_t* __restrict__ chars, uint64_t nchars, V view,
                            const MergePair* __restrict__ pairs,
                            const uint64_t* __restrict__ first, uint32_t npair,
                            const uint64_t* __restrict__ split, const typename V::T* __restrict__ in,
                            typename V::T* __restrict__ out, uint32_t piece)
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
                take_a = compare_lcp(chars, nchars, view.off(in[pr.a0 + i]), view.off(in[pr.a1 + j]),
                                     &l) <= 0;
            }
            out[pr.a0 + d] = take_a ? in[pr.a0 + i] : in[pr.a1 + j];
            if (take_a) ++i; else ++j;
        }
    }
}

// LCP-aware piece merge (the reference's LCP loser-tree rule for two runs).
// Runs A = in[a0, a1) and B = in[a1, b1) with their LCP arrays in lcp_in
// (entries at a run's first position are not read). ha / hb are the LCPs of
// the heads A[i] / B[j] with the last output. A piece that does not start
// the pair first finds its previous output (the larger of A[i0 - 1] and
// B[j0 - 1]; equal strings: B's, as A's comes first) and the heads' LCPs
// with it. lcp_out (may be null) receives the LCP of every output but the
// pair's first.
template <class V>
__global__ void __launch_bounds__(256, 4) k_merge_lcp_seq(const uint8_t* __restrict__ chars, uint64_t nchars, V view,
                                const MergePair* __restrict__ pairs,
                                const uint64_t* __restrict__ first, uint32_t npair,
                                const uint64_t* __restrict__ split,
                                const typename V::T* __restrict__ in,
                                const uint32_t* __restrict__ lcp_in,
                                typename V::T* __restrict__ out, uint32_t* __restrict__ lcp_out,
                                uint32_t piece)
{
    using T = typename V::T;
    const uint64_t ntask = first[npair];
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = pair_of(first, npair, t);
        const MergePair pr = pairs[p];
        const uint64_t na = pr.a1 - pr.a0, nb = pr.b1 - pr.a1;
        const T* A = in + pr.a0;
        const T* B = in + pr.a1;
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
                if (i < na) compare_from(chars, nchars, view.off(A[i]), view.off(B[j - 1]), 0, &ha);
            } else if (j0 == 0) {  // previous output A[i0 - 1]
                ha = i < na ? LA[i] : 0u;
                if (j < nb) compare_from(chars, nchars, view.off(B[j]), view.off(A[i - 1]), 0, &hb);
            } else {
                uint32_t l;
                const int c = compare_from(chars, nchars, view.off(A[i - 1]), view.off(B[j - 1]), 0, &l);
                // LCP(x, z) >= min(LCP(x, y), LCP(y, z)): start from that depth
                if (c <= 0) {  // previous output B[j0 - 1]
                    hb = j < nb ? LB[j] : 0u;
                    if (i < na)
                        compare_from(chars, nchars, view.off(A[i]), view.off(B[j - 1]), min(LA[i], l), &ha);
                } else {       // previous output A[i0 - 1]
                    ha = i < na ? LA[i] : 0u;
                    if (j < nb)
                        compare_from(chars, nchars, view.off(B[j]), view.off(A[i - 1]), min(LB[j], l), &hb);
                }
            }
        }
        // the heads' entries and arena offsets stay in registers: a compare
        // reads chars only; the runs' entries and LCPs are read 16 bytes at
        // a time
        SeqRead<T> ra{in}, rb{in};
        SeqRead4 la{lcp_in}, lb{lcp_in};
        T va = i < i1 ? ra.get(pr.a0 + i) : T(0), vb = j < j1 ? rb.get(pr.a1 + j) : T(0);
        uint64_t oa = i < i1 ? view.off(va) : 0ull, ob = j < j1 ? view.off(vb) : 0ull;
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
            out[pr.a0 + d] = take_a ? va : vb;
            if (lcp_out && d > 0) lcp_out[pr.a0 + d] = take_a ? ha : hb;
            if (take_a) {
                ++i;
                ha = i < na ? la.get(pr.a0 + i) : 0u;  // against its predecessor, the last output
                if (i < i1) {
                    va = ra.get(pr.a0 + i);
                    oa = view.off(va);
                }
            } else {
                ++j;
                hb = j < nb ? lb.get(pr.a1 + j) : 0u;
                if (j < j1) {
                    vb = rb.get(pr.a1 + j);
                    ob = view.off(vb);
                }
            }
        }
    }
}

// Handles of the runs' strings (32-bit id << hbits | arena offset, offsets
// below 2^hbits <= 2^32), with the arena check of k_merge_check.
__global__ void k_merge_pack(const uint64_t* __restrict__ offs, uint64_t nchars,
                             const uint32_t* __restrict__ ids, uint64_t n, uint32_t hbits,
                             uint64_t* __restrict__ out, uint32_t* err)
{
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t id = ids[q];
        const uint64_t o = __ldg(offs + id);
        if (o >= nchars) atomicOr(err, ERR_OFFSET);
        out[q] = ((uint64_t)id << hbits) | (o < nchars ? o : 0ull);
    }
}

// The ids of merged handles.
__global__ void k_merge_unpack(const uint64_t* __restrict__ h, uint64_t n, uint32_t hbits,
                               uint32_t* __restrict__ ids)
{
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (uint64_t)gridDim.x * blockDim.x)
        ids[q] = (uint32_t)(h[q] >> hbits);
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
