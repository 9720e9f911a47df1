// kernels_small.cuh -- finishes segments of at most SMALL_MAX strings,
// including every deeper character round and the LCP array. This is the
// device counterpart of pS5's base cases: sort_mkqs_cache /
// insertion_sort_cache on 8-byte caches (src/parallel/
// bingmann-parallel_sample_sort.hpp:805-861, 1056-1178), inssort_generic
// (src/sequential/inssort.hpp:63-95) and lcp_insertion_sort
// (src/sequential/bingmann-lcp_inssort.hpp:38-189).
//
// Size classes (push_seg in kernels_big.cuh picks the list):
//   k_tiny            <= 32 strings, one warp per segment, shuffles only
//   k_small<256,128>  <= 256 strings, one block
//   k_small<2048,256> <= 2048 strings, one block
// Block phase: sort (group, key, handle) with a shared-memory bitonic sort;
// runs of equal keys become groups one 8-byte round deeper; a group that
// stops splitting jumps to its common prefix. Groups of <= 32 strings are
// parked and finished by the warp phase (the k_tiny rounds), where a group
// that stops splitting jumps ahead with a warp-wide 256-byte compare, so deep
// repeats cost O(LCP / 256) rounds.
#pragma once

#include "block_util.cuh"
#include "work.cuh"

namespace pssgpu {

template <int MAXN>
struct SmallSmem {
    uint64_t key[MAXN];
    uint64_t hnd[MAXN];
    uint32_t gdep[MAXN];   // depth of the active group starting here
    uint32_t ndep[MAXN];   // next depth, staged
    uint16_t grp[MAXN];    // start index of the element's group
    uint16_t rs[MAXN];     // start index of the element's run
    uint16_t runlen[MAXN]; // run length, at the run start
    uint8_t state[MAXN];   // 0 active (block phase), 1 done, 2 parked
    uint16_t park_start[MAXN / 2];
    uint16_t park_len[MAXN / 2];
    uint32_t park_dep[MAXN / 2];
    uint32_t tmp[32];
    uint32_t npark;
    uint32_t nactive;
    uint32_t ngroups;
    uint32_t g0;
    uint32_t jump;
};

__device__ __forceinline__ bool tuple_less(uint32_t ga, uint64_t ka, uint64_t ha,
                                           uint32_t gb, uint64_t kb, uint64_t hb)
{
    if (ga != gb) return ga < gb;
    if (ka != kb) return ka < kb;
    return ha < hb;
}

// Common-prefix extension (in 8-byte chunks from depth d) of the string
// behind handle `other` against the one behind `base`: the first chunk where
// they differ or base ends, at most `limit`.
__device__ __forceinline__ uint32_t chunks_equal(const Work& w, uint64_t base, uint64_t other,
                                                 uint32_t d, uint32_t limit)
{
    uint32_t c = 0;
    const uint64_t ob = h_off(w, base) + d, oo = h_off(w, other) + d;
    while (c < limit) {
        const uint64_t ka = load_key(w.chars, w.nchars, ob + 8ull * c);
        const uint64_t kb = load_key(w.chars, w.nchars, oo + 8ull * c);
        if (ka != kb || key_terminated(ka)) break;
        ++c;
    }
    return c;
}

// Warp rounds for one group of c <= 32 strings sharing d chars; lane i holds
// handle i on entry and the i-th smallest handle's string on return. LCPs go
// to lcp[pos0 + lane] for lanes >= 1. first_keys (may be null) holds the keys
// at depth d, saving the first gather. Each round sorts (group, key, source
// lane) with a 32-lane bitonic network on three shuffled words and then
// fetches the rest of the element from its source lane.
__device__ __forceinline__ uint64_t warp_rounds(const Work& w, uint64_t myh, uint32_t c,
                                                uint32_t d, uint32_t pos0,
                                                const uint64_t* first_keys)
{
    const uint32_t lane = threadIdx.x & 31;
    const bool real = lane < c;
    uint32_t mygrp = real ? 0u : 32u;   // lanes past c sort last
    uint32_t mydep = d;
    uint32_t mystate = real ? 0u : 1u;  // 0 active, 1 done
    uint64_t mykey = 0;
    uint32_t prev_active = c;
    bool stalled = false;
    bool first = first_keys != nullptr;
    while (true) {
        const uint32_t A = __ballot_sync(0xffffffffu, mystate == 0);
        if (A == 0) break;
        if (stalled) {
            // exactly one active group that did not split: jump to its
            // common prefix, 32 chunks of 8 bytes per step
            const int f = __ffs(A) - 1;
            const uint64_t base = __shfl_sync(0xffffffffu, myh, f);
            const uint32_t dd = __shfl_sync(0xffffffffu, mydep, f);
            uint32_t best = 0xFFFFFFFFu;
            uint32_t rest = A & ~(1u << f);
            const uint64_t ob = h_off(w, base) + dd;
            while (rest) {
                const int j = __ffs(rest) - 1;
                rest &= rest - 1;
                const uint64_t other = __shfl_sync(0xffffffffu, myh, j);
                const uint64_t oo = h_off(w, other) + dd;
                for (uint32_t t = 0; t * 32 < best; ++t) {
                    const uint32_t ch = t * 32 + lane;
                    const uint64_t ka = load_key(w.chars, w.nchars, ob + 8ull * ch);
                    const uint64_t kb = load_key(w.chars, w.nchars, oo + 8ull * ch);
                    const uint32_t bal = __ballot_sync(0xffffffffu, ka != kb || key_terminated(ka));
                    if (bal) {
                        best = min(best, t * 32 + (uint32_t)(__ffs(bal) - 1));
                        break;
                    }
                }
            }
            if (mystate == 0) mydep = dd + 8u * best;
        }
        if (mystate == 0) mykey = first ? first_keys[lane] : h_key(w, myh, mydep);
        first = false;
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
                const uint32_t pos = pos0 + lane;
                if (pk != mykey) w.lcp[pos] = mydep + lcp_key_type(pk, mykey);
                else if (key_terminated(mykey)) w.lcp[pos] = mydep + lcp_key_depth(mykey);
            }
            if (len == 1 || key_terminated(mykey)) mystate = 1;
            else mydep += 8;
            mygrp = rs;
        }
        const uint32_t A2 = __ballot_sync(0xffffffffu, mystate == 0);
        const uint32_t G2 = __ballot_sync(0xffffffffu, mystate == 0 && rs == lane);
        const uint32_t na = __popc(A2);
        stalled = (na == prev_active) && (__popc(G2) == 1);
        prev_active = na;
    }
    return myh;
}

// One warp per segment of at most 32 strings; 8 segments per block.
constexpr int TINY_WARPS = 8;
__global__ void __launch_bounds__(32 * TINY_WARPS) k_tiny(Work w, const Seg* list, uint32_t count)
{
    const uint32_t g = blockIdx.x * TINY_WARPS + (threadIdx.x >> 5);
    if (g >= count) return;  // whole warp
    const uint32_t lane = threadIdx.x & 31;
    const Seg sg = list[g];
    const int buf = sg.meta & META_BUF;
    if (lane == 0) atomicAdd(w.counters + C_P_SMALL, sg.size);
    uint64_t myh = lane < sg.size ? w.hnd[buf][sg.begin + lane] : ~0ull;
    const uint64_t* fk = (sg.meta & META_VALID) ? w.keys[buf] + sg.begin : nullptr;
    myh = warp_rounds(w, myh, sg.size, sg.depth, sg.begin, fk);
    if (lane < sg.size) w.perm[sg.begin + lane] = h_id(w, myh);
}

// Bitonic sort of sm.{grp,key,hnd}[0, npad) by (grp, key, hnd).
template <int MAXN, int THREADS>
__device__ void small_bitonic(SmallSmem<MAXN>& sm, uint32_t npad)
{
    for (uint32_t kk = 2; kk <= npad; kk <<= 1) {
        for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < npad / 2; i += THREADS) {
                const uint32_t a = 2 * i - (i & (j - 1));
                const uint32_t b = a + j;
                const bool asc = (a & kk) == 0;
                const uint32_t ga = sm.grp[a], gb = sm.grp[b];
                const uint64_t ka = sm.key[a], kb = sm.key[b];
                const uint64_t ha = sm.hnd[a], hb = sm.hnd[b];
                if (tuple_less(gb, kb, hb, ga, ka, ha) == asc) {
                    sm.grp[a] = (uint16_t)gb; sm.grp[b] = (uint16_t)ga;
                    sm.key[a] = kb; sm.key[b] = ka;
                    sm.hnd[a] = hb; sm.hnd[b] = ha;
                }
            }
            __syncthreads();
        }
    }
}

// One block per segment of 33..MAXN strings (or an all-equal segment to copy).
template <int MAXN, int THREADS>
__global__ void __launch_bounds__(THREADS) k_small(Work w, const Seg* list)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmallSmem<MAXN>& sm = *reinterpret_cast<SmallSmem<MAXN>*>(smem_raw);
    const Seg sg = list[blockIdx.x];
    const uint32_t m = sg.size, begin = sg.begin;
    const int buf = sg.meta & META_BUF;
    const uint64_t* ghs = w.hnd[buf];
    if (threadIdx.x == 0) atomicAdd(w.counters + C_P_SMALL, m);
    if (sg.meta & META_FINAL) {
        for (uint32_t i = threadIdx.x; i < m; i += THREADS) {
            w.perm[begin + i] = h_id(w, ghs[begin + i]);
            if (w.lcp && i) w.lcp[begin + i] = sg.depth;
        }
        return;
    }
    if (threadIdx.x == 0) {
        sm.npark = 0;
        atomicAdd(w.counters + C_SMALLSEGS, 1u);
    }
    for (uint32_t i = threadIdx.x; i < m; i += THREADS) sm.hnd[i] = ghs[begin + i];
    __syncthreads();
    if (m <= (uint32_t)WARP_GROUP_MAX) {
        if (threadIdx.x == 0) {
            sm.park_start[0] = 0; sm.park_len[0] = (uint16_t)m; sm.park_dep[0] = sg.depth;
            sm.npark = 1;
        }
        __syncthreads();
    } else {
        // ---------------- block phase ----------------
        uint32_t npad = 1;
        while (npad < m) npad <<= 1;
        const bool valid = sg.meta & META_VALID;
        for (uint32_t i = threadIdx.x; i < npad; i += THREADS) {
            if (i < m) {
                sm.key[i] = valid ? w.keys[buf][begin + i] : h_key(w, sm.hnd[i], sg.depth);
                sm.grp[i] = 0;
                sm.state[i] = 0;
            } else {
                sm.key[i] = ~0ull;
                sm.hnd[i] = ~0ull;
                sm.grp[i] = 0xFFFF;
                sm.state[i] = 1;
            }
        }
        if (threadIdx.x == 0) sm.gdep[0] = sg.depth;
        uint32_t prev_active = m;
        bool stalled = false;
        const uint32_t per = (m + THREADS - 1) / THREADS;
        const uint32_t clo = min(threadIdx.x * per, m), chi = min(clo + per, m);
        while (true) {
            __syncthreads();
            if (stalled) {
                // one active group that did not split: jump to its common prefix
                const uint32_t g0 = sm.g0;
                const uint32_t d0 = sm.gdep[g0];
                const uint64_t base = sm.hnd[g0];
                if (threadIdx.x == 0) sm.jump = 0xFFFFFFFFu;
                __syncthreads();
                for (uint32_t i = threadIdx.x; i < m; i += THREADS) {
                    if (sm.state[i] != 0 || i == g0) continue;
                    const uint32_t lim = *((volatile uint32_t*)&sm.jump);
                    const uint32_t cc = chunks_equal(w, base, sm.hnd[i], d0, lim);
                    atomicMin(&sm.jump, cc);
                }
                __syncthreads();
                if (threadIdx.x == 0) sm.gdep[g0] = d0 + 8u * sm.jump;
                __syncthreads();
                for (uint32_t i = threadIdx.x; i < m; i += THREADS)
                    if (sm.state[i] == 0) sm.key[i] = h_key(w, sm.hnd[i], sm.gdep[sm.grp[i]]);
                __syncthreads();
            }
            small_bitonic<MAXN, THREADS>(sm, npad);
            // run starts: a run is a maximal stretch of equal (grp, key)
            uint32_t last = 0;
            for (uint32_t i = clo; i < chi; ++i) {
                const bool ns = i == 0 || sm.grp[i] != sm.grp[i - 1] || sm.key[i] != sm.key[i - 1];
                if (ns) last = i;
            }
            const bool any = clo < chi;
            uint32_t carry = block_excl_max<THREADS>(any ? last : 0u, sm.tmp);
            for (uint32_t i = clo; i < chi; ++i) {
                const bool ns = i == 0 || sm.grp[i] != sm.grp[i - 1] || sm.key[i] != sm.key[i - 1];
                if (ns) carry = i;
                sm.rs[i] = (uint16_t)carry;
                const bool end = (i + 1 == m) || sm.grp[i + 1] != sm.grp[i] || sm.key[i + 1] != sm.key[i];
                if (end) sm.runlen[carry] = (uint16_t)(i + 1 - carry);
            }
            if (threadIdx.x == 0) { sm.nactive = 0; sm.ngroups = 0; }
            __syncthreads();
            // resolve: LCPs, new states, parked groups (reads gdep only)
            for (uint32_t i = threadIdx.x; i < m; i += THREADS) {
                if (sm.state[i] != 0) continue;
                const uint64_t k = sm.key[i];
                const uint32_t d = sm.gdep[sm.grp[i]];
                if (i >= 1 && sm.grp[i - 1] == sm.grp[i] && w.lcp) {
                    const uint64_t pk = sm.key[i - 1];
                    if (pk != k) w.lcp[begin + i] = d + lcp_key_type(pk, k);
                    else if (key_terminated(k)) w.lcp[begin + i] = d + lcp_key_depth(k);
                }
                const uint32_t r = sm.rs[i];
                const uint32_t len = sm.runlen[r];
                if (i == r && len > 1 && !key_terminated(k)) {
                    if (len <= (uint32_t)WARP_GROUP_MAX) {
                        const uint32_t at = atomicAdd(&sm.npark, 1u);
                        sm.park_start[at] = (uint16_t)r;
                        sm.park_len[at] = (uint16_t)len;
                        sm.park_dep[at] = d + 8;
                    } else {
                        sm.ndep[r] = d + 8;
                    }
                }
            }
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < m; i += THREADS) {
                if (sm.state[i] != 0) continue;
                const uint32_t r = sm.rs[i];
                const uint32_t len = sm.runlen[r];
                const uint64_t k = sm.key[i];
                uint8_t ns;
                if (len == 1 || key_terminated(k)) ns = 1;
                else if (len <= (uint32_t)WARP_GROUP_MAX) ns = 2;
                else ns = 0;
                sm.grp[i] = (uint16_t)r;
                sm.state[i] = ns;
                if (ns == 0) {
                    atomicAdd(&sm.nactive, 1u);
                    if (i == r) {
                        sm.gdep[r] = sm.ndep[r];
                        atomicAdd(&sm.ngroups, 1u);
                        sm.g0 = r;
                    }
                }
            }
            __syncthreads();
            const uint32_t na = sm.nactive;
            if (na == 0) break;
            stalled = (na == prev_active) && (sm.ngroups == 1);
            prev_active = na;
            if (!stalled) {
                for (uint32_t i = threadIdx.x; i < m; i += THREADS)
                    if (sm.state[i] == 0) sm.key[i] = h_key(w, sm.hnd[i], sm.gdep[sm.grp[i]]);
            }
        }
        __syncthreads();
    }
    // ---------------- warp phase ----------------
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t np = sm.npark;
    for (uint32_t g = warp; g < np; g += THREADS / 32) {
        const uint32_t start = sm.park_start[g], c = sm.park_len[g];
        uint64_t myh = lane < c ? sm.hnd[start + lane] : ~0ull;
        myh = warp_rounds(w, myh, c, sm.park_dep[g], begin + start, nullptr);
        if (lane < c) sm.hnd[start + lane] = myh;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < m; i += THREADS) w.perm[begin + i] = h_id(w, sm.hnd[i]);
}

// the two block-sized classes
constexpr int SMALL_A = 256;
constexpr int SMALL_A_THREADS = 128;
#define K_SMALL_A k_small<SMALL_A, SMALL_A_THREADS>
#define K_SMALL_B k_small<SMALL_MAX, SMALL_THREADS>

}  // namespace pssgpu
