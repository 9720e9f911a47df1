// kernels_block.cuh -- block sample sort for segments of 33..MAXN strings.
//
// One block runs pS5's sequential sample-sort step (SeqSampleSortStep,
// src/parallel/bingmann-parallel_sample_sort.hpp:565-676) on its segment in
// shared memory: sample splitters, a level-order splitter tree, classify,
// counting-sort scatter, then recurse on the buckets. Buckets of at most 32
// strings go to the warp rounds (kernels_small.cuh); larger ones are
// processed again by the whole block, at the same depth ('<' buckets, keys
// still valid) or 8 chars deeper (equal buckets). A group whose samples are
// all equal first jumps to its common prefix. LCPs at bucket boundaries come
// from the neighbouring buckets' max / min keys (sample_sort_lcp,
// hpp:311-396); inside buckets the warp rounds write them.
#pragma once

#include "kernels_small.cuh"

namespace pssgpu {

constexpr int BLK_MAX_BITS = 8;  // at most 255 splitters, 511 buckets per step

// splitter-tree levels a block sorter of MAXN strings can use: about 8
// strings per '<' bucket (the L rule in k_block), at most BLK_MAX_BITS
__host__ __device__ constexpr int blk_bits(int maxn)
{
    int lg = 0;
    while ((2 << lg) <= maxn) ++lg;
    return lg - 3 < BLK_MAX_BITS ? lg - 3 : BLK_MAX_BITS;
}

template <int MAXN>
struct BlockSmem {
    static constexpr int NB = 2 << blk_bits(MAXN);  // bucket slots
    uint64_t key[MAXN];
    uint64_t hnd[MAXN];
    uint16_t dst[MAXN];                  // bucket, then destination, per element
    uint32_t cnt[NB];                    // bucket counts, then bucket starts
    uint32_t cur[NB];                    // scatter cursors
    uint64_t bmin[NB];
    uint64_t bmax[NB];
    uint64_t tree[NB / 2];               // level order, index 1..k
    uint64_t samp[NB];
    // groups larger than a warp, processed one at a time by the block
    uint16_t g_start[MAXN / 32];
    uint16_t g_len[MAXN / 32];
    uint32_t g_dep[MAXN / 32];
    uint8_t g_valid[MAXN / 32];
    // groups of at most 32 strings, finished by warps at the end
    uint16_t w_start[MAXN / 2];
    uint8_t w_len[MAXN / 2];
    uint8_t w_valid[MAXN / 2];
    uint32_t w_dep[MAXN / 2];
    uint32_t tmp32[32];
    uint32_t ng, nw, jump;
    uint32_t cs, cc, cd, cv;             // the group being processed
};

template <int MAXN, int THREADS>
__device__ __forceinline__ void blk_push(BlockSmem<MAXN>& sm, uint32_t start, uint32_t len,
                                         uint32_t dep, bool valid, uint32_t* err)
{
    if (len <= (uint32_t)WARP_GROUP_MAX) {
        const uint32_t at = atomicAdd(&sm.nw, 1u);
        if (at >= (uint32_t)(MAXN / 2)) { set_error(err, ERR_INTERNAL); return; }
        sm.w_start[at] = (uint16_t)start;
        sm.w_len[at] = (uint8_t)len;
        sm.w_valid[at] = valid ? 1 : 0;
        sm.w_dep[at] = dep;
    } else {
        const uint32_t at = atomicAdd(&sm.ng, 1u);
        if (at >= (uint32_t)(MAXN / 32)) { set_error(err, ERR_INTERNAL); return; }
        sm.g_start[at] = (uint16_t)start;
        sm.g_len[at] = (uint16_t)len;
        sm.g_dep[at] = dep;
        sm.g_valid[at] = valid ? 1 : 0;
    }
}

// The block sorter proper. On entry the block's strings are in
// sm.hnd[0, m) (keys in sm.key where a group's keys are valid), their output
// positions are begin + [0, m), and the initial groups are pushed (sm.ng /
// sm.nw lists, blk_push); strings in no group are final where they stand.
// Runs the sample-sort steps on groups of more than 32 strings, the warp
// windows on the rest, and writes perm[begin, begin + m). buf is the
// ping-pong buffer the strings came from (stalled warp groups are handed to
// the deep-group list there, when the Work has one). All threads call.
template <int MAXN, int THREADS>
__device__ __forceinline__ void block_sort_groups(const Work& w, BlockSmem<MAXN>& sm,
                                                  uint32_t begin, uint32_t m, int buf,
                                                  uint32_t (*wscratch)[32], uint32_t* err)
{
    while (true) {
        if (threadIdx.x == 0) {
            if (sm.ng) {
                const uint32_t g = --sm.ng;
                sm.cs = sm.g_start[g];
                sm.cc = sm.g_len[g];
                sm.cd = sm.g_dep[g];
                sm.cv = sm.g_valid[g];
            } else {
                sm.cc = 0;
            }
        }
        __syncthreads();
        const uint32_t s = sm.cs, c = sm.cc, d = sm.cd;
        if (c == 0) break;
        if (!sm.cv) {
            for (uint32_t i = threadIdx.x; i < c; i += THREADS) sm.key[s + i] = h_key(w, sm.hnd[s + i], d);
        }
        // sample: 2^(L+1) keys at pseudo-random positions of the group
        const int lg = 31 - __clz((int)c);
        const uint32_t L = (uint32_t)min(blk_bits(MAXN), max(1, lg - 3));
        const uint32_t k = (1u << L) - 1;
        const uint32_t S = 2u << L;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < S; i += THREADS) {
            const uint64_t h = mix64(((uint64_t)(begin + s) << 24) ^ ((uint64_t)d << 4) ^ i);
            sm.samp[i] = sm.key[s + (uint32_t)(((h >> 32) * c) >> 32)];
        }
        __syncthreads();
        if (S <= 64u && S <= (uint32_t)THREADS) {
            // rank sort in place (ties by index): two barriers
            uint64_t x = 0;
            uint32_t r = 0;
            if (threadIdx.x < S) {
                x = sm.samp[threadIdx.x];
                for (uint32_t j = 0; j < S; ++j) {
                    const uint64_t y = sm.samp[j];
                    r += (y < x || (y == x && j < threadIdx.x)) ? 1u : 0u;
                }
            }
            __syncthreads();
            if (threadIdx.x < S) sm.samp[r] = x;
            __syncthreads();
        } else {
            bitonic_sort_block(sm.samp, S);
        }
        const uint64_t* sorted = sm.samp;
        if (sorted[0] == sorted[S - 1] && !key_terminated(sorted[0])) {
            // likely one tied group: measure its common prefix in chunks
            if (threadIdx.x == 0) sm.jump = 0xFFFFFFFFu;
            __syncthreads();
            const uint64_t base = sm.hnd[s];
            for (uint32_t i = 1 + threadIdx.x; i < c; i += THREADS)
                atomicMin(&sm.jump, chunks_equal(w, base, sm.hnd[s + i], d, &sm.jump));
            __syncthreads();
            const uint32_t jmp = sm.jump;
            if (jmp > 0) {
                // all strings share 8 * jmp more chars: continue deeper
                if (threadIdx.x == 0) blk_push<MAXN, THREADS>(sm, s, c, d + 8u * jmp, false, err);
                __syncthreads();
                continue;
            }
        }
        // level-order tree over every second sample
        for (uint32_t v = 1 + threadIdx.x; v <= k; v += THREADS) {
            const uint32_t h = 31 - __clz((int)v);
            const uint32_t p = v - (1u << h);
            const uint32_t r = ((2 * p + 1) << (L - 1 - h)) - 1;
            sm.tree[v] = sorted[2 * r + 1];
        }
        const uint32_t B = 2 * k + 1;
        for (uint32_t b = threadIdx.x; b < B; b += THREADS) {
            sm.cnt[b] = 0;
            sm.bmin[b] = ~0ull;
            sm.bmax[b] = 0;
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < c; i += THREADS) {
            const uint64_t key = sm.key[s + i];
            uint32_t v = 1;
            uint64_t cand = 0;
            for (uint32_t l = 0; l < L; ++l) {
                const uint64_t tv = sm.tree[v];
                const bool gt = key > tv;
                cand = gt ? cand : tv;
                v = 2 * v + (gt ? 1u : 0u);
            }
            const uint32_t r = v - (1u << L);
            const uint32_t b = 2 * r + ((r < k && cand == key) ? 1u : 0u);
            sm.dst[s + i] = (uint16_t)b;
            atomicAdd(&sm.cnt[b], 1u);
            if (w.lcp) {  // bucket key ranges, for the LCPs at bucket boundaries
                atomicMin((unsigned long long*)&sm.bmin[b], (unsigned long long)key);
                atomicMax((unsigned long long*)&sm.bmax[b], (unsigned long long)key);
            }
        }
        __syncthreads();
        block_scan_array<THREADS>(sm.cnt, (int)B, sm.tmp32);  // counts -> starts
        for (uint32_t b = threadIdx.x; b < B; b += THREADS) sm.cur[b] = sm.cnt[b];
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < c; i += THREADS)
            sm.dst[s + i] = (uint16_t)atomicAdd(&sm.cur[sm.dst[s + i]], 1u);
        __syncthreads();
        {
            // permute keys, then handles, through registers
            constexpr int PER = MAXN / THREADS;
            uint64_t v[PER];
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                const uint32_t i = threadIdx.x + j * THREADS;
                if (i < c) v[j] = sm.key[s + i];
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                const uint32_t i = threadIdx.x + j * THREADS;
                if (i < c) {
                    sm.key[s + sm.dst[s + i]] = v[j];
                    v[j] = sm.hnd[s + i];
                }
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                const uint32_t i = threadIdx.x + j * THREADS;
                if (i < c) sm.hnd[s + sm.dst[s + i]] = v[j];
            }
        }
        // children and boundary LCPs; cnt now holds bucket starts
        for (uint32_t b = threadIdx.x; b < B; b += THREADS) {
            const uint32_t st = sm.cnt[b];
            const uint32_t en = b + 1 < B ? sm.cnt[b + 1] : c;
            const uint32_t cb = en - st;
            if (cb == 0) continue;
            if (st > 0 && w.lcp) {
                uint32_t pb = b - 1;  // previous non-empty bucket
                while (sm.cnt[pb] == st) --pb;
                w.lcp[begin + s + st] = d + lcp_key_type(sm.bmax[pb], sm.bmin[b]);
            }
            if (cb == 1) continue;
            if (b & 1) {
                const uint64_t key = sorted[b];  // the splitter: sorted sample 2r + 1
                if (key_terminated(key)) {
                    if (w.lcp) {
                        const uint32_t v = d + lcp_key_depth(key);
                        for (uint32_t q = 1; q < cb; ++q) w.lcp[begin + s + st + q] = v;
                    }
                } else {
                    blk_push<MAXN, THREADS>(sm, s + st, cb, d + 8, false, err);
                }
            } else {
                blk_push<MAXN, THREADS>(sm, s + st, cb, d, true, err);
            }
        }
        __syncthreads();
    }
    // groups of at most 32 strings: every warp packs a contiguous share of
    // the list into warp windows
    constexpr uint32_t NWARP = THREADS / 32;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t nw = sm.nw;
    const uint32_t per = (nw + NWARP - 1) / NWARP;
    const uint32_t first = min(warp * per, nw), ng = min(first + per, nw) - first;
    for_each_window(ng, [&](uint32_t j) { return (uint32_t)sm.w_len[first + j]; },
                    [&](uint32_t j0, uint32_t cnt) {
        uint32_t off = 0, mygrp = 32, start = 0, dep = 0;
        bool valid = false;
        for (uint32_t q = 0; q < cnt; ++q) {
            const uint32_t g = first + j0 + q;
            const uint32_t len = sm.w_len[g];
            if (lane >= off && lane < off + len) {
                mygrp = off;
                start = sm.w_start[g] + (lane - off);
                dep = sm.w_dep[g];
                valid = sm.w_valid[g];
            }
            off += len;
        }
        const bool real = mygrp < 32;
        const uint64_t h = real ? sm.hnd[start] : ~0ull;
        const uint64_t k0 = (real && valid) ? sm.key[start] : 0ull;
        // stalled groups go to the deep-group list when there is one
        const uint64_t r = warp_window(w, h, mygrp, dep, begin + start, real && valid, k0,
                                       wscratch[warp], w.deep[w.cur ^ 1] ? w.hnd[buf] : nullptr,
                                       (uint32_t)buf);
        if (real) sm.hnd[start] = r;
    });
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < m; i += THREADS) w.perm[begin + i] = h_id(w, sm.hnd[i]);
}

template <int MAXN, int THREADS>
__global__ void __launch_bounds__(THREADS, THREADS <= 64 ? 20 : 4) k_block(Work w, const Seg* list)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BlockSmem<MAXN>& sm = *reinterpret_cast<BlockSmem<MAXN>*>(smem_raw);
    __shared__ uint32_t wscratch[THREADS / 32][32];
    const Seg sg = list[blockIdx.x];
    const uint32_t m = sg.size, begin = sg.begin;
    const int buf = sg.meta & META_BUF;
    const uint64_t* ghs = w.hnd[buf];
    uint32_t* err = w.counters + C_ERR;
    // an offset outside the arena (flagged before this launch) fails the
    // sort: skip the work on handles that may be corrupt
    if (threadIdx.x == 0) sm.ng = *(volatile uint32_t*)err & ERR_OFFSET;
    __syncthreads();
    if (sm.ng) return;
    __syncthreads();
    if (sg.meta & META_FINAL) {
        for (uint32_t i = threadIdx.x; i < m; i += THREADS) {
            w.perm[begin + i] = h_id(w, ghs[begin + i]);
            if (w.lcp && i) w.lcp[begin + i] = sg.depth;
        }
        return;
    }
    const bool valid0 = sg.meta & META_VALID;
    for (uint32_t i = threadIdx.x; i < m; i += THREADS) {
        sm.hnd[i] = __ldg(ghs + begin + i);
        if (valid0) sm.key[i] = __ldg(w.keys[buf] + begin + i);
    }
    if (threadIdx.x == 0) {
        sm.ng = 0;
        sm.nw = 0;
        blk_push<MAXN, THREADS>(sm, 0, m, sg.depth, valid0, err);
    }
    __syncthreads();
    block_sort_groups<MAXN, THREADS>(w, sm, begin, m, buf, wscratch, err);
}

#define K_BLOCK_A k_block<SMALL_A, SMALL_A_THREADS>
#define K_BLOCK_B k_block<SMALL_MAX, SMALL_THREADS>
// the allocation-free entry point's sorter: up to 2048 strings in one block
#define K_BLOCK_NOALLOC k_block<2048, 256>

}  // namespace pssgpu
