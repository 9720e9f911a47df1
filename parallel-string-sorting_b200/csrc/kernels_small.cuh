// kernels_small.cuh -- warp-level finishing of groups of at most 32 strings,
// including every deeper character round and the LCP array. This is the
// device counterpart of pS5's base cases: sort_mkqs_cache /
// insertion_sort_cache on 8-byte caches (src/parallel/
// bingmann-parallel_sample_sort.hpp:805-861, 1056-1178), inssort_generic
// (src/sequential/inssort.hpp:63-95) and lcp_insertion_sort
// (src/sequential/bingmann-lcp_inssort.hpp:38-189).
//
// Size classes (push_seg in kernels_big.cuh picks the list):
//   k_tiny            <= 32 strings (several segments share one warp window)
//   k_block<256,128>  <= 256 strings, one block (kernels_block.cuh)
//   k_block<1024,256> <= 1024 strings, one block (kernels_block.cuh)
//
// A warp window holds up to 32 strings from one or more independent groups.
// Each lane owns one output slot (a position of the permutation); groups
// never leave their lanes. Every round sorts (group, key) over the 32 lanes,
// splits runs of equal keys into groups one 8-byte round deeper; after two
// rounds in which no group split and no string finished, every group jumps to
// its common prefix with warp-wide 512-byte compares, so deep repeats cost
// O(LCP / 512) steps.
#pragma once

#include "block_util.cuh"
#include "work.cuh"

namespace pssgpu {

// Common-prefix extension (in 8-byte chunks from depth d) of the string
// behind handle `other` against the one behind `base`: the first chunk where
// they differ or base ends. The search stops at *limit, which other threads
// lower meanwhile (re-read every 4 chunks; the 4 chunks of both strings are
// loaded at once), so one long shared repeat does not hold up the block once
// another string has shown a shorter common prefix.
__device__ __forceinline__ uint32_t chunks_equal(const Work& w, uint64_t base, uint64_t other,
                                                 uint32_t d, const volatile uint32_t* limit)
{
    const uint64_t ob = h_off(w, base) + d, oo = h_off(w, other) + d;
    for (uint32_t c = 0;; c += 4) {
        if (c >= *limit) return c;
        uint64_t ra[4], rb[4];
        load_raw_chunks<4>(w.chars, w.nchars, ob + 8ull * c, 4, ra);
        load_raw_chunks<4>(w.chars, w.nchars, oo + 8ull * c, 4, rb);
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            // equal windows without a NUL continue; any other pair of windows
            // either differs before a NUL or ends base's string here
            const uint64_t z = (ra[q] - 0x0101010101010101ull) & ~ra[q] & 0x8080808080808080ull;
            if (ra[q] != rb[q] || z) return c + q;
        }
    }
}

// Finish a warp window. Per lane on entry: the string handle of the slot,
// mygrp = lane index where the slot's group starts (32 for an unused lane),
// mydep = chars the group shares, mypos = output position of the slot, and
// the key at mydep when has_key. Returns the handle that sorts into this
// lane's slot; LCPs inside groups are written to lcp[mypos]. scratch is 32
// words of shared memory private to the warp.
// With defer_hnd set (the block sorters), groups that stall on a long common
// prefix are not walked here: their handles go to defer_hnd[mypos] and the
// group to the deep-group list (segment meta defer_meta), and k_deep finishes
// them in the next pass, one warp per group, while this block moves on; the
// slots of such lanes are left to k_deep. jump_first starts with the jump.
__device__ __forceinline__ uint64_t warp_window(const Work& w, uint64_t myh, uint32_t mygrp,
                                                uint32_t mydep, uint32_t mypos, bool has_key,
                                                uint64_t key0, uint32_t* scratch,
                                                uint64_t* defer_hnd = nullptr,
                                                uint32_t defer_meta = 0, bool jump_first = false)
{
    const uint32_t lane = threadIdx.x & 31;
    uint32_t mystate = mygrp < 32 ? 0u : 1u;  // 0 active, 1 done
    uint64_t mykey = 0;
    uint32_t prev_active = __popc(__ballot_sync(0xffffffffu, mystate == 0));
    uint32_t gstarts = __ballot_sync(0xffffffffu, mystate == 0 && mygrp == lane);
    uint32_t prev_groups = __popc(gstarts);
    uint32_t stalled = jump_first ? 2u : 0u;  // rounds in a row without progress
    bool first = true;
    while (true) {
        uint32_t A = __ballot_sync(0xffffffffu, mystate == 0);
        if (A == 0) break;
        if (stalled >= 2) {
            // the last two rounds neither split a group nor finished a
            // string: defer the groups, or move every active group to its
            // common prefix, one group at a time, 64 chunks of 8 bytes per step
            stalled = 0;
            uint32_t todo = gstarts;
            if (defer_hnd) {
                const int nxt = w.cur ^ 1;
                const bool lead = mystate == 0 && mygrp == lane;
                const uint32_t same = __match_any_sync(0xffffffffu, mystate == 0 ? mygrp : 64u + lane);
                uint32_t at = 0xFFFFFFFFu;
                if (lead) {
                    at = atomicAdd(w.counters + C_DEEP + nxt, 1u);
                    if (at < w.deep_cap)
                        w.deep[nxt][at] = Seg{mypos, (uint32_t)__popc(same), mydep, defer_meta};
                }
                const uint32_t D = __ballot_sync(0xffffffffu, lead && at < w.deep_cap);
                if (mystate == 0 && ((D >> mygrp) & 1u)) {
                    defer_hnd[mypos] = myh;
                    mystate = 1;
                }
                todo &= ~D;  // groups the full list could not take are walked here
            }
            while (todo) {
                const int f = __ffs(todo) - 1;
                todo &= todo - 1;
                const uint64_t base = __shfl_sync(0xffffffffu, myh, f);
                const uint32_t dd = __shfl_sync(0xffffffffu, mydep, f);
                const bool member = mystate == 0 && mygrp == (uint32_t)f;
                uint32_t rest = __ballot_sync(0xffffffffu, member) & ~(1u << f);
                uint32_t best = 0xFFFFFFFFu;
                const uint64_t ob = h_off(w, base) + dd;
                while (rest) {
                    const int j = __ffs(rest) - 1;
                    rest &= rest - 1;
                    const uint64_t other = __shfl_sync(0xffffffffu, myh, j);
                    const uint64_t oo = h_off(w, other) + dd;
                    for (uint32_t t = 0; t * 64 < best; ++t) {
                        // lane l compares chunks 64 t + 2 l and 64 t + 2 l + 1:
                        // equal windows without a NUL continue
                        const uint32_t ch = t * 64 + 2 * lane;
                        uint64_t ra[2], rb[2];
                        load_raw_chunks<2>(w.chars, w.nchars, ob + 8ull * ch, 2, ra);
                        load_raw_chunks<2>(w.chars, w.nchars, oo + 8ull * ch, 2, rb);
                        const uint64_t z0 = (ra[0] - 0x0101010101010101ull) & ~ra[0] & 0x8080808080808080ull;
                        const uint64_t z1 = (ra[1] - 0x0101010101010101ull) & ~ra[1] & 0x8080808080808080ull;
                        const bool m0 = ra[0] != rb[0] || z0, m1 = ra[1] != rb[1] || z1;
                        const uint32_t bal = __ballot_sync(0xffffffffu, m0 || m1);
                        if (bal) {
                            const int fl = __ffs(bal) - 1;
                            const uint32_t first0 = __ballot_sync(0xffffffffu, m0) >> fl & 1u;
                            best = min(best, t * 64 + 2u * fl + (first0 ? 0u : 1u));
                            break;
                        }
                    }
                }
                if (member) mydep = dd + 8u * best;
            }
        }
        if (mystate == 0) mykey = (first && has_key) ? key0 : h_key(w, myh, mydep);
        first = false;
        // Groups are contiguous lane ranges; a group starts at the lane whose
        // mygrp is itself, and unused lanes end the window. Sort the active
        // groups by (key, lane): by rank inside the group when the largest
        // active group is small, else with a 32-lane bitonic network.
        const uint32_t GB = __ballot_sync(0xffffffffu, mygrp == lane || mygrp >= 32);
        const uint32_t above = lane == 31 ? 0u : (GB & (0xFFFFFFFFu << (lane + 1)));
        const uint32_t gend = above ? (uint32_t)(__ffs(above) - 1) : 32u;
        const uint32_t glen = mystate == 0 ? gend - mygrp : 0u;
        const uint32_t M = __reduce_max_sync(0xffffffffu, glen);
        if (M > 16) {
            uint32_t tag = (mygrp << 5) | lane;
            uint64_t k = mykey;
#pragma unroll
            for (uint32_t kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
                for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
                    const uint32_t ot = __shfl_xor_sync(0xffffffffu, tag, j);
                    const uint64_t ok = __shfl_xor_sync(0xffffffffu, k, j);
                    const bool lower = (lane & j) == 0;
                    const bool asc = (lane & kk) == 0;
                    bool other_less;
                    if ((ot >> 5) != (tag >> 5)) other_less = (ot >> 5) < (tag >> 5);
                    else if (ok != k) other_less = ok < k;
                    else other_less = (ot & 31u) < (tag & 31u);
                    // the lower lane of an ascending pair keeps the smaller
                    if ((lower == asc) ? other_less : !other_less) { tag = ot; k = ok; }
                }
            }
            const uint32_t src = tag & 31u;
            myh = __shfl_sync(0xffffffffu, myh, src);
            mydep = __shfl_sync(0xffffffffu, mydep, src);
            mystate = __shfl_sync(0xffffffffu, mystate, src);
            mygrp = tag >> 5;
            mykey = k;
        } else if (M > 1) {
            uint32_t rank = 0;
            for (uint32_t j = 0; j < M; ++j) {
                const uint32_t src = (mygrp + j) & 31u;
                const uint64_t kj = __shfl_sync(0xffffffffu, mykey, src);
                if (j < glen && (kj < mykey || (kj == mykey && mygrp + j < lane))) ++rank;
            }
            scratch[mystate == 0 ? mygrp + rank : lane] = lane;
            __syncwarp();
            const uint32_t src = scratch[lane];
            __syncwarp();
            myh = __shfl_sync(0xffffffffu, myh, src);
            mydep = __shfl_sync(0xffffffffu, mydep, src);
            mykey = __shfl_sync(0xffffffffu, mykey, src);
        }
        const uint32_t pg = __shfl_up_sync(0xffffffffu, mygrp, 1);
        const uint64_t pk = __shfl_up_sync(0xffffffffu, mykey, 1);
        const bool ns = lane == 0 || mygrp != pg || mykey != pk;
        const uint32_t NS = __ballot_sync(0xffffffffu, ns);
        const uint32_t le = NS & (0xFFFFFFFFu >> (31 - lane));
        const uint32_t rs = 31u - __clz(le);
        const uint32_t gtm = lane == 31 ? 0u : (NS & (0xFFFFFFFFu << (lane + 1)));
        const uint32_t nx = gtm ? (uint32_t)(__ffs(gtm) - 1) : 32u;
        const uint32_t len = nx - rs;
        if (mystate == 0) {
            if (lane >= 1 && pg == mygrp && w.lcp) {
                if (pk != mykey) w.lcp[mypos] = mydep + lcp_key_type(pk, mykey);
                else if (key_terminated(mykey)) w.lcp[mypos] = mydep + lcp_key_depth(mykey);
            }
            if (len == 1 || key_terminated(mykey)) mystate = 1;
            else mydep += 8;
            mygrp = rs;
        }
        const uint32_t A2 = __ballot_sync(0xffffffffu, mystate == 0);
        const uint32_t G2 = __ballot_sync(0xffffffffu, mystate == 0 && rs == lane);
        const uint32_t na = __popc(A2);
        stalled = (na == prev_active && __popc(G2) == prev_groups) ? stalled + 1 : 0;
        prev_active = na;
        prev_groups = __popc(G2);
        gstarts = G2;
    }
    return myh;
}

// Greedy packing of a short list of groups into warp windows of <= 32 lanes.
// Calls fn(window_first, window_count) for consecutive runs of groups; every
// lane of the warp takes part. sizes(j) gives the strings of group j.
template <typename SizeFn, typename WinFn>
__device__ __forceinline__ void for_each_window(uint32_t ngroups, SizeFn sizes, WinFn fn)
{
    uint32_t j = 0;
    while (j < ngroups) {
        uint32_t used = 0, e = j;
        while (e < ngroups && used + sizes(e) <= 32u) used += sizes(e++);
        fn(j, e - j);
        j = e;
    }
}

// A warp's list entries L[0, ng) (ng <= 32, every entry at most 32 strings)
// packed greedily into windows of at most 32 strings. The entries are loaded
// once, one per lane, and read through shuffles. fn(s, gq, gs, real) runs
// once per window on every lane: s is the lane's entry, gq its index inside
// the window, gs the entry's first lane, real whether the lane holds a string.
template <typename Fn>
__device__ __forceinline__ void warp_seg_windows(const Seg* __restrict__ L, uint32_t ng, Fn fn)
{
    const uint32_t lane = threadIdx.x & 31;
    Seg mine{};
    if (lane < ng) mine = L[lane];
    uint32_t j = 0;
    while (j < ng) {
        uint32_t used = 0, e = j;
        while (e < ng) {
            const uint32_t sz = __shfl_sync(0xffffffffu, mine.size, e);
            if (used + sz > 32u) break;
            used += sz;
            ++e;
        }
        if (e == j) ++e;  // no entry is larger than a window; never stall
        uint32_t off = 0, gs = 32, gq = 31;
        Seg sg{};
        for (uint32_t q = j; q < e; ++q) {
            const uint32_t b = __shfl_sync(0xffffffffu, mine.begin, q);
            const uint32_t sz = __shfl_sync(0xffffffffu, mine.size, q);
            const uint32_t d = __shfl_sync(0xffffffffu, mine.depth, q);
            const uint32_t m = __shfl_sync(0xffffffffu, mine.meta, q);
            if (lane >= off && lane < off + sz) {
                sg = Seg{b, sz, d, m};
                gs = off;
                gq = q - j;
            }
            off += sz;
        }
        fn(sg, gq, gs, gs < 32u && lane < 32u);
        j = e;
    }
}

// Segments of at most 32 strings: each warp takes TINY_PER_WARP consecutive
// list entries and packs them into warp windows.
constexpr int TINY_WARPS = 8;
constexpr int TINY_PER_WARP = 8;
__global__ void __launch_bounds__(32 * TINY_WARPS, 5) k_tiny(Work w, const Seg* list, uint32_t count)
{
    __shared__ uint32_t scratch[TINY_WARPS][32];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t g0 = (blockIdx.x * TINY_WARPS + (threadIdx.x >> 5)) * TINY_PER_WARP;
    if (g0 >= count) return;  // whole warp
    const uint32_t ng = min((uint32_t)TINY_PER_WARP, count - g0);
    warp_seg_windows(list + g0, ng, [&](const Seg& sg, uint32_t, uint32_t gs, bool real) {
        const uint32_t mygrp = real ? gs : 32u;
        const int buf = sg.meta & META_BUF;
        const uint32_t pos = sg.begin + (lane - gs);
        const uint64_t h = real ? w.hnd[buf][pos] : ~0ull;
        const bool hk = real && (sg.meta & META_VALID);
        const uint64_t k0 = hk ? w.keys[buf][pos] : 0ull;
        const uint64_t r = warp_window(w, h, mygrp, sg.depth, pos, hk, k0, scratch[threadIdx.x >> 5]);
        if (real) w.perm[pos] = h_id(w, r);
    });
}

// Deep groups handed over by the block sorters: one warp per group, which
// starts with the common-prefix jump and then sorts the group to the end.
__global__ void __launch_bounds__(32 * TINY_WARPS) k_deep(Work w, const Seg* list, uint32_t count)
{
    __shared__ uint32_t scratch[TINY_WARPS][32];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t g = blockIdx.x * TINY_WARPS + (threadIdx.x >> 5);
    if (g >= count) return;  // whole warp
    const Seg sg = list[g];
    const bool real = lane < sg.size;
    const uint32_t pos = sg.begin + lane;
    const uint64_t h = real ? w.hnd[sg.meta & META_BUF][pos] : ~0ull;
    const uint64_t r = warp_window(w, h, real ? 0u : 32u, sg.depth, pos, false, 0ull,
                                   scratch[threadIdx.x >> 5], nullptr, 0u, true);
    if (real) w.perm[pos] = h_id(w, r);
}

// the block-sorted size classes (kernels_block.cuh)
constexpr int SMALL_A = 256;
constexpr int SMALL_A_THREADS = 64;

}  // namespace pssgpu
