// merge.cuh -- merge of K sorted runs of one arena into one sorted run with
// its LCP array: the step after per-shard sorts that the reference takes in
// its top-level merge of per-NUMA-node pS5 outputs
// (src/parallel/eberle-ps5-parallel-toplevel-merge.hpp:56-175, the
// LCP-aware K-way merge of src/parallel/eberle-parallel-lcp-merge*.hpp over
// src/sequential/bingmann-lcp_losertree.hpp).
//
// Here the runs merge pairwise, ceil(log2 K) rounds of three launches: the
// merge-path splits of every MERGE_SPLIT_COARSE-th piece of MERGE_PIECE
// outputs (a warp each), those of the other pieces (a thread each, inside
// the window the coarse ones leave), then the merge of each piece by one
// thread. With the runs' LCP arrays the piece merge is LCP-aware, as the
// reference's loser tree is (src/sequential/bingmann-lcp_losertree.hpp:61-110,
// 156-185): each head carries its LCP with the last output, the head with
// the larger one is the smaller string without reading a char, equal ones
// compare from that depth only, and every output's LCP falls out of the same
// step. Each head also carries the 7 chars that follow its LCP (a wider form
// of the char cache of the reference's LCP + cache sorts), so most equal
// LCPs are settled without reading the arena; a thread's runs are staged in
// shared memory a chunk ahead and its outputs written per 32-byte sector.
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

// compare_from that also returns the last 8-char windows it read (*wa, *wb,
// both from depth *wd; the LCP lies in [*wd, *wd + 7]).
__device__ __forceinline__ int compare_from_win(const uint8_t* chars, uint64_t nchars, uint64_t oa,
                                                uint64_t ob, uint32_t d, uint32_t* lcp, uint64_t* wa,
                                                uint64_t* wb, uint32_t* wd)
{
    while (true) {
        const uint64_t ka = load_key(chars, nchars, oa + d), kb = load_key(chars, nchars, ob + d);
        if (ka != kb || key_terminated(ka)) {
            *wa = ka;
            *wb = kb;
            *wd = d;
            if (ka != kb) {
                *lcp = d + lcp_key_type(ka, kb);
                return ka < kb ? -1 : 1;
            }
            *lcp = d + lcp_key_depth(ka);
            return 0;
        }
        d += 8;
    }
}

// Char cache of a run head (the reference's LCP + char-cache form, with
// more than one char): the chars of the string from depth h, its LCP with
// the last output, big-endian in bits 63..8 (7 chars, NUL past the string's
// end) and in bits 7..0 how many of them are known (1..7). A run's cache
// array holds, for every entry but its first, the chars at the depth of its
// LCP with its predecessor, so a head taken from the run brings them along.
__device__ __forceinline__ uint64_t cache_of_key(uint64_t key) { return (key & ~0xFFull) | 7u; }

// The cache of the same string j chars deeper (j < known).
__device__ __forceinline__ uint64_t cache_shift(uint64_t c, uint32_t j)
{
    return (((c & ~0xFFull) << (8u * j)) & ~0xFFull) | ((c & 0xFFu) - j);
}

// Order of heads a and b that both share h chars with the last output, from
// their caches first and from the arena past the chars both know. Returns
// whether a comes first (equal strings: a, the left run's); the loser's LCP
// with the winner, the new last output, replaces its h and its cache moves
// to that depth.
__device__ __forceinline__ bool cached_tie(const uint8_t* chars, uint64_t nchars, uint64_t oa,
                                           uint64_t ob, uint32_t& ha, uint64_t& ca, uint32_t& hb,
                                           uint64_t& cb)
{
    const uint32_t h = ha;
    const uint32_t m = min((uint32_t)(ca & 0xFFu), (uint32_t)(cb & 0xFFu));
    const uint64_t mask = ~0ull << (64u - 8u * m);
    const uint64_t ka = ca & mask, kb = cb & mask;
    uint32_t j;
    bool take_a;
    if (ka != kb) {  // differ within the known chars
        j = lcp_key_type(ka, kb);
        take_a = ka < kb;
    } else if ((j = lcp_key_depth(ka)) < m) {  // both end within them: equal
        take_a = true;
    } else {  // the arena past the known chars
        uint32_t l, wd;
        uint64_t wa, wb;
        take_a = compare_from_win(chars, nchars, oa, ob, h + m, &l, &wa, &wb, &wd) <= 0;
        const uint32_t sft = l - wd;  // 0..7
        const uint64_t nc = (((take_a ? wb : wa) << (8u * sft)) & ~0xFFull) | min(7u, 8u - sft);
        if (take_a) {
            hb = l;
            cb = nc;
        } else {
            ha = l;
            ca = nc;
        }
        return take_a;
    }
    if (take_a) {
        hb = h + j;
        cb = cache_shift(cb, j);
    } else {
        ha = h + j;
        ca = cache_shift(ca, j);
    }
    return take_a;
}

// Merge-path form of a round. A pair is (a0, a1, b1): left run [a0, a1),
// right run [a1, b1) (empty for an unpaired last run), merged into [a0, b1).
// Its output is cut into pieces of `piece` positions (unless the caller
// sets it: MERGE_PIECE_MIN..MERGE_PIECE, sized to fill whole waves of the
// GPU's resident piece-merge threads); task t of the round is piece
// t - first[pair] of its pair. The splits find for every piece how many
// left-run strings precede it (a search along the piece's diagonal),
// k_merge_lcp_seq (or k_merge_seq without LCP arrays) merges each piece
// sequentially from there.
constexpr uint32_t MERGE_PIECE = 256;
constexpr uint32_t MERGE_PIECE_MIN = 64;
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
// by k_merge_prep, so the offset comes with the entry a round reads in order
// and no round gathers offsets.
struct MergeByIds {
    using T = uint32_t;
    const uint64_t* offs;
    __device__ __forceinline__ uint64_t off(uint32_t v) const { return __ldg(offs + v); }
    __device__ __forceinline__ uint32_t id(uint32_t v) const { return v; }
};
struct MergeByHandles {
    using T = uint64_t;
    uint64_t hmask;
    uint32_t hbits;
    __device__ __forceinline__ uint64_t off(uint64_t v) const { return v & hmask; }
    __device__ __forceinline__ uint32_t id(uint64_t v) const { return (uint32_t)(v >> hbits); }
};


// Splits in two launches: k_merge_split_coarse searches every
// MERGE_SPLIT_COARSE-th piece of a pair over the whole diagonal;
// k_merge_split searches the other pieces between the two coarse splits
// around them. The merge path is a monotone staircase, so for a diagonal d
// between coarse diagonals D0 < D1 with splits i0, i1: i0 <= i(d) <= i1 and
// d - D1 + i1 <= i(d) <= d - D0 + i0, a window of at most
// MERGE_SPLIT_COARSE * piece positions. A split is the number of left-run
// strings among the first d outputs: the first i with A[i] > B[d - i - 1]
// (ties go to the left run).
constexpr uint32_t MERGE_SPLIT_COARSE = 32;

// One warp per coarse split (cfirst[p]: the pair's first coarse split; a
// pair of P pieces has ceil(P / MERGE_SPLIT_COARSE)): each step probes 32
// positions of the window at once, one per lane, and keeps the 33rd part
// between the last probe below the split and the first at or above it, so a
// diagonal of 2^22 positions takes 5 steps of parallel compares where a
// binary search takes 22 dependent ones. Blocks of whole warps.
template <class V>
__global__ void k_merge_split_coarse(const uint8_t* __restrict__ chars, uint64_t nchars, V view,
                                     const MergePair* __restrict__ pairs,
                                     const uint64_t* __restrict__ first,
                                     const uint64_t* __restrict__ cfirst, uint32_t npair,
                                     const typename V::T* __restrict__ in, uint64_t* __restrict__ split,
                                     uint32_t piece)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t ncoarse = cfirst[npair];
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < ncoarse; w += nwarps) {
        const uint32_t p = pair_of(cfirst, npair, w);
        const uint64_t k = (w - cfirst[p]) * MERGE_SPLIT_COARSE;
        const MergePair pr = pairs[p];
        const uint64_t na = pr.a1 - pr.a0, nb = pr.b1 - pr.a1;
        const int64_t d = (int64_t)(k * piece);
        // the split lies in [lo, hi]; positions >= hi count as above it
        int64_t lo = d > (int64_t)nb ? d - (int64_t)nb : 0, hi = min(d, (int64_t)na);
        auto above = [&](int64_t x) {
            uint32_t l;
            return compare_from(chars, nchars, view.off(in[pr.a0 + x]), view.off(in[pr.a1 + d - x - 1]), 0,
                                &l) > 0;
        };
        while (hi - lo > 32) {
            // probes x_i = lo + floor((i + 1) * len / 33), strictly
            // increasing inside [lo, hi) for len > 32
            const int64_t len = hi - lo;
            const int64_t x = lo + ((int64_t)(lane + 1) * len) / 33;
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, above(x));
            if (m == 0) {
                lo = lo + (32 * len) / 33 + 1;
            } else {
                const int f = __ffs(m) - 1;
                const int64_t xf = lo + ((int64_t)(f + 1) * len) / 33;
                lo = f ? lo + ((int64_t)f * len) / 33 + 1 : lo;
                hi = xf;
            }
        }
        const int64_t x = lo + lane;
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, x < hi ? above(x) : true);
        if (lane == 0) split[first[p] + k] = (uint64_t)(m ? min(lo + (int64_t)(__ffs(m) - 1), hi) : hi);
    }
}

template <class V>
__global__ void k_merge_split(const uint8_t* __restrict__ chars, uint64_t nchars, V view,
                              const MergePair* __restrict__ pairs,
                              const uint64_t* __restrict__ first, uint32_t npair,
                              const typename V::T* __restrict__ in, uint64_t* __restrict__ split,
                              uint32_t piece)
{
    const uint64_t ntask = first[npair];
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = pair_of(first, npair, t);
        const uint64_t k = t - first[p];
        if (k % MERGE_SPLIT_COARSE == 0) continue;
        const MergePair pr = pairs[p];
        const uint64_t na = pr.a1 - pr.a0, nb = pr.b1 - pr.a1;
        const uint64_t d = k * piece;
        int64_t lo = d > nb ? (int64_t)(d - nb) : 0, hi = (int64_t)min(d, na);
        uint32_t depth = 0;  // chars every compared pair shares
        const uint64_t k0 = k - k % MERGE_SPLIT_COARSE, k1 = k0 + MERGE_SPLIT_COARSE;
        const uint64_t D0 = k0 * piece, i0 = split[first[p] + k0];
        const bool last = first[p] + k1 >= first[p + 1];
        const uint64_t D1 = last ? na + nb : k1 * piece, i1 = last ? na : split[first[p] + k1];
        lo = max(lo, max((int64_t)i0, (int64_t)d - (int64_t)D1 + (int64_t)i1));
        hi = min(hi, min((int64_t)i1, (int64_t)(d - D0 + i0)));
        if (hi - lo > 2) {
            // the search compares A[x], x in [lo, hi), with B[y], y in
            // [d - hi, d - lo): a sorted run's extremes share no more than
            // anything between them, so every such pair shares
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

// Shared-memory staging of the LCP-aware piece merge. A thread's heads come
// from two runs it reads in order, and its outputs go to one stretch: per
// run and stream (entries, LCPs, caches) two chunks of MS_CH entries, the
// next one in flight (cp.async) while the current one is read, and per
// output stream the 32-byte sector being filled, written at once when full.
// Every byte a thread fetches is then one it uses, and no output sector is
// written in parts (a partial sector costs a fill read from DRAM).
constexpr uint32_t MS_THREADS = 128;
constexpr uint32_t MS_CH = 4;

template <class T>
struct alignas(32) MergeStage {
    T v[2][2][MS_THREADS][MS_CH];           // run, slot, thread, entry
    uint64_t ck[2][2][MS_THREADS][MS_CH];
    uint32_t lcp[2][2][MS_THREADS][MS_CH];
    T ov[MS_THREADS][32 / sizeof(T)];       // output sectors
    uint64_t ock[MS_THREADS][4];
    uint32_t olcp[MS_THREADS][8];
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// MS_CH entries of X (aligned to their size) in 16-byte copies, or one
// 8-byte copy
template <class X>
__device__ __forceinline__ void cp_async_chunk(X* smem, const X* gmem)
{
    if constexpr (MS_CH * sizeof(X) >= 16) {
#pragma unroll
        for (uint32_t k = 0; k < MS_CH; k += 16 / sizeof(X)) cp_async16(smem + k, gmem + k);
    } else {
        static_assert(MS_CH * sizeof(X) == 8, "chunks of 8 or a multiple of 16 bytes");
        cp_async8(smem, gmem);
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// One 32-byte sector from shared memory to an aligned global address.
__device__ __forceinline__ void store_sector(void* gdst, const void* ssrc)
{
    const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(ssrc);
    const ulonglong2 y = *(reinterpret_cast<const ulonglong2*>(ssrc) + 1);
    asm volatile("st.global.v4.u64 [%0], {%1, %2, %3, %4};\n" ::"l"(gdst), "l"(x.x), "l"(x.y), "l"(y.x),
                 "l"(y.y)
                 : "memory");
}

// Chunk c (entries [c * MS_CH, c * MS_CH + MS_CH) of the round's arrays) of
// run r into its slot, as one cp.async group. The arrays are 16-byte
// aligned and padded past their last chunk.
template <class T>
__device__ __forceinline__ void stage_chunk(MergeStage<T>& sm, uint32_t r, uint64_t c, const T* in,
                                            const uint32_t* lcp_in, const uint64_t* ck_in)
{
    const uint32_t tid = threadIdx.x, sl = (uint32_t)(c & 1);
    const uint64_t q = c * MS_CH;
    cp_async_chunk(&sm.v[r][sl][tid][0], in + q);
    cp_async_chunk(&sm.ck[r][sl][tid][0], ck_in + q);
    cp_async_chunk(&sm.lcp[r][sl][tid][0], lcp_in + q);
    cp_async_commit();
}

// Run R's head entered chunk c (its end: q1): wait for the chunk (it was
// staged one ahead; the other run's chunk in flight is not waited for when
// it went out later) and stage the next one into the slot just read. mine /
// other: whether run R's / the other run's chunk is in flight; last_b:
// whether run B staged the latest group.
template <uint32_t R, class T>
__device__ __forceinline__ void next_chunk(MergeStage<T>& sm, uint64_t c, uint64_t q1, const T* in,
                                           const uint32_t* lcp_in, const uint64_t* ck_in, bool& mine,
                                           bool& other, bool& last_b)
{
    const bool other_later = R == 0 ? last_b : !last_b;
    if (other && other_later) {
        cp_async_wait1();
    } else {
        cp_async_wait0();
        other = false;
    }
    mine = false;
    if ((c + 1) * MS_CH < q1) {
        stage_chunk(sm, R, c + 1, in, lcp_in, ck_in);
        mine = true;
        last_b = R == 1;
    }
}

// An output stream: entries written to base[o] for o in [lo, hi) in order,
// collected per 32-byte sector in shared memory (buf, E entries of U) and
// written per sector; a sector the stretch covers only in part is written
// entry by entry. s: the sector slot of the next entry.
template <class U>
struct SectorOut {
    static constexpr uint32_t E = 32 / sizeof(U);
    U* base;
    U* buf;
    uint64_t lo;
    uint32_t s;
    __device__ __forceinline__ void init(U* b, U* sbuf, uint64_t lo_)
    {
        base = b;
        buf = sbuf;
        lo = lo_;
        s = (uint32_t)((reinterpret_cast<uintptr_t>(b + lo_) / sizeof(U)) & (E - 1));
    }
    __device__ __forceinline__ void put(uint64_t o, U x)
    {
        buf[s] = x;
        if (s == E - 1) {
            if (o + 1 >= lo + E) {
                store_sector(base + (o + 1 - E), buf);
            } else {
                for (uint64_t k = lo; k <= o; ++k) base[k] = buf[(uint32_t)(k + E - 1 - o)];
            }
            s = 0;
        } else {
            ++s;
        }
    }
    // the entries of [lo, hi) after the last full sector (slots [0, s))
    __device__ __forceinline__ void finish(uint64_t hi)
    {
        if (s == 0 || hi <= lo) return;
        uint64_t k = hi - s;
        if (k < lo) k = lo;
        for (; k < hi; ++k) base[k] = buf[(uint32_t)(k + s - hi)];
    }
};

// LCP-aware piece merge (the reference's LCP loser-tree rule for two runs,
// with char caches). Runs A = in[a0, a1) and B = in[a1, b1) with their LCP
// arrays in lcp_in and char caches in ck_in (entries at a run's first
// position are not read). ha / hb are the LCPs of the heads A[i] / B[j] with
// the last output, ca / cb their chars from there: heads with different
// LCPs order by them, equal ones by their caches, and only chars neither
// cache holds are read from the arena. A piece that does not start the pair
// first finds its previous output (the larger of A[i0 - 1] and B[j0 - 1];
// equal strings: B's, as A's comes first) and the heads' LCPs with it, and
// reads its heads' chars from the arena. lcp_out (may be null) receives the
// LCP of every output but the pair's first, ck_out (may be null) every
// output's cache; with ids_out (the last round) the outputs' string ids go
// there instead of their entries to out. MS_THREADS threads per block, sizeof(MergeStage<T>) bytes
// of dynamic shared memory.
template <class V>
__global__ void __launch_bounds__(MS_THREADS)
    k_merge_lcp_seq(const uint8_t* __restrict__ chars, uint64_t nchars, V view,
                                const MergePair* __restrict__ pairs,
                                const uint64_t* __restrict__ first, uint32_t npair,
                                const uint64_t* __restrict__ split,
                                const typename V::T* __restrict__ in,
                                const uint32_t* __restrict__ lcp_in, const uint64_t* __restrict__ ck_in,
                                typename V::T* __restrict__ out, uint32_t* __restrict__ lcp_out,
                                uint64_t* __restrict__ ck_out, uint32_t* __restrict__ ids_out, uint32_t piece)
{
    using T = typename V::T;
    extern __shared__ __align__(32) unsigned char merge_smem[];
    MergeStage<T>& sm = *reinterpret_cast<MergeStage<T>*>(merge_smem);
    const uint32_t tid = threadIdx.x;
    const uint64_t ntask = first[npair];
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + tid; t < ntask;
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
        // absolute positions of the heads and their ends
        uint64_t qa = pr.a0 + i0, qb = pr.a1 + j0;
        const uint64_t qa1 = pr.a0 + i1, qb1 = pr.a1 + j1;
        // the first chunks of both runs in flight while the heads' LCPs
        // with the previous output are found
        bool pend_a = false, pend_b = false, last_b = false;
        if (qa < qa1) {
            stage_chunk(sm, 0, qa / MS_CH, in, lcp_in, ck_in);
            if ((qa / MS_CH + 1) * MS_CH < qa1) stage_chunk(sm, 0, qa / MS_CH + 1, in, lcp_in, ck_in);
        }
        if (qb < qb1) {
            stage_chunk(sm, 1, qb / MS_CH, in, lcp_in, ck_in);
            if ((qb / MS_CH + 1) * MS_CH < qb1) stage_chunk(sm, 1, qb / MS_CH + 1, in, lcp_in, ck_in);
        }
        uint32_t ha = 0, hb = 0;
        {
            const uint64_t i = i0, j = j0;
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
        }
        cp_async_wait0();
        T va = T(0), vb = T(0);
        uint64_t oa = 0, ob = 0, ca = 0, cb = 0;
        if (qa < qa1) {
            va = sm.v[0][(qa / MS_CH) & 1][tid][qa % MS_CH];
            oa = view.off(va);
            ca = cache_of_key(load_key(chars, nchars, oa + ha));
        }
        if (qb < qb1) {
            vb = sm.v[1][(qb / MS_CH) & 1][tid][qb % MS_CH];
            ob = view.off(vb);
            cb = cache_of_key(load_key(chars, nchars, ob + hb));
        }
        const uint64_t o0 = pr.a0 + d0, o1 = pr.a0 + d1;
        SectorOut<T> wv;
        SectorOut<uint32_t> wi, wl;
        SectorOut<uint64_t> wc;
        if (ids_out) wi.init(ids_out, reinterpret_cast<uint32_t*>(sm.ov[tid]), o0);
        else wv.init(out, sm.ov[tid], o0);
        if (lcp_out) wl.init(lcp_out, sm.olcp[tid], d0 == 0 ? o0 + 1 : o0);
        if (ck_out) wc.init(ck_out, sm.ock[tid], o0);
        // per run: heads left in the piece (the current one included), the
        // current chunk, its slot and the head's entry in it; the thread's
        // staging of each run
        uint32_t na_left = (uint32_t)(qa1 - qa), nb_left = (uint32_t)(qb1 - qb);
        uint64_t cha = qa / MS_CH, chb = qb / MS_CH;
        uint32_t sla = (uint32_t)(cha & 1), slb = (uint32_t)(chb & 1);
        uint32_t ea = (uint32_t)(qa % MS_CH), eb = (uint32_t)(qb % MS_CH);
        constexpr uint32_t SLOT = MS_THREADS * MS_CH;  // entries from one slot to the next
        const T* svA = &sm.v[0][0][tid][0];
        const T* svB = &sm.v[1][0][tid][0];
        const uint32_t* slA = &sm.lcp[0][0][tid][0];
        const uint32_t* slB = &sm.lcp[1][0][tid][0];
        const uint64_t* skA = &sm.ck[0][0][tid][0];
        const uint64_t* skB = &sm.ck[1][0][tid][0];
        const uint32_t plen = (uint32_t)(d1 - d0);
        for (uint32_t k = 0; k < plen; ++k) {
            const uint64_t o = o0 + k;
            bool take_a;
            if (!na_left) take_a = false;
            else if (!nb_left) take_a = true;
            else if (ha != hb) take_a = ha > hb;
            else take_a = cached_tie(chars, nchars, oa, ob, ha, ca, hb, cb);
            if (ids_out) wi.put(o, view.id(take_a ? va : vb));
            else wv.put(o, take_a ? va : vb);
            if (lcp_out && (k | d0)) wl.put(o, take_a ? ha : hb);
            if (ck_out) wc.put(o, take_a ? ca : cb);
            if (take_a) {
                if (--na_left) {  // against its predecessor, the last output
                    if (++ea == MS_CH) {
                        ea = 0;
                        sla ^= 1;
                        next_chunk<0>(sm, ++cha, qa1, in, lcp_in, ck_in, pend_a, pend_b, last_b);
                    }
                    const uint32_t at = sla * SLOT + ea;
                    va = svA[at];
                    ha = slA[at];
                    ca = skA[at];
                    oa = view.off(va);
                }
            } else {
                if (--nb_left) {
                    if (++eb == MS_CH) {
                        eb = 0;
                        slb ^= 1;
                        next_chunk<1>(sm, ++chb, qb1, in, lcp_in, ck_in, pend_b, pend_a, last_b);
                    }
                    const uint32_t at = slb * SLOT + eb;
                    vb = svB[at];
                    hb = slB[at];
                    cb = skB[at];
                    ob = view.off(vb);
                }
            }
        }
        if (ids_out) wi.finish(o1);
        else wv.finish(o1);
        if (lcp_out) wl.finish(o1);
        if (ck_out) wc.finish(o1);
        cp_async_wait0();  // nothing of this piece left in flight
    }
}

// Round 0's inputs in the library's own buffers (aligned, padded, so that
// the rounds stage them in 16-byte copies), with the arena check: every
// id's offset must lie inside the arena (else *err). PACK: handles (32-bit
// id << hbits | arena offset, offsets below 2^hbits <= 2^32) into out; else
// the ids as they are (out may be null: no copy). With the runs' LCP arrays
// (lcp not null) their copy into lcp_out.
template <bool PACK>
__global__ void k_merge_prep(const uint64_t* __restrict__ offs, uint64_t nchars,
                             const uint32_t* __restrict__ ids, const uint32_t* __restrict__ lcp, uint64_t n,
                             uint32_t hbits, void* out, uint32_t* __restrict__ lcp_out, uint32_t* err)
{
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t id = ids[q];
        const uint64_t o = __ldg(offs + id);
        const bool bad = o >= nchars;
        if (bad) atomicOr(err, ERR_OFFSET);
        if (PACK) static_cast<uint64_t*>(out)[q] = ((uint64_t)id << hbits) | (bad ? 0ull : o);
        else if (out) static_cast<uint32_t*>(out)[q] = id;
        if (lcp) lcp_out[q] = lcp[q];
    }
}

// Every entry's cache at the depth of its LCP (round 0's ck_in; a run's
// first LCP is any value, its cache is not read). Needed by round 0's piece
// merge only, so it runs beside round 0's splits.
template <class V>
__global__ void k_merge_caches(const uint8_t* __restrict__ chars, uint64_t nchars, V view,
                               const typename V::T* __restrict__ in, const uint32_t* __restrict__ lcp,
                               uint64_t n, uint64_t* __restrict__ ck_out)
{
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (uint64_t)gridDim.x * blockDim.x)
        ck_out[q] = cache_of_key(load_key(chars, nchars, view.off(in[q]) + lcp[q]));
}

// The ids of merged handles.
__global__ void k_merge_unpack(const uint64_t* __restrict__ h, uint64_t n, uint32_t hbits,
                               uint32_t* __restrict__ ids)
{
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (uint64_t)gridDim.x * blockDim.x)
        ids[q] = (uint32_t)(h[q] >> hbits);
}

}  // namespace pssgpu
