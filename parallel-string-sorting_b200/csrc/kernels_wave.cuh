// kernels_wave.cuh -- the whole sort of an input that fits one wave of
// resident blocks, in one cooperative launch (no host round trip between
// the steps, no kernel boundaries).
//
// pS5 runs an input of this size as one sample-sort step over all strings
// followed by a SmallsortJob per bucket on its job queue
// (src/parallel/bingmann-parallel_sample_sort.hpp:1613-1634, 1264-1611,
// 405-676). Here the same steps are phases of one kernel, separated by grid
// barriers (all blocks are co-resident by the cooperative launch):
//   A  every block gathers the first 8 chars (get_char_uint64_simple) of its
//      tile of strings into registers; the first blocks also draw 2^(L+1)
//      samples in chunks of 512 and sort their chunk
//   B  every block merges the sorted chunks and builds the splitters and the
//      level-order tree itself (SampleSortStep::sample,
//      TreeBuilderLevelOrder), classifies its tile (find_bkt), counts per bucket in
//      shared memory, reserve the tile's share of every bucket with one
//      global atomic per non-empty bucket (count, hpp:1414-1435)
//   C  bucket starts (count_finished), scatter keys and handles in bucket
//      order (distribute, hpp:1464-1490)
//   D  a dynamic queue of windows of WAVE_WINDOW positions: the runs of
//      buckets of at most WAVE_WINDOW strings that start in a window are
//      finished by the block sorter as one group (block_sort_groups, the
//      SmallsortJob counterpart); larger buckets are finished alone (up to
//      WAVE_SORT_MAX strings), copied out when their strings are all equal,
//      or handed to the level-synchronous passes as a segment
//      (distribute_finished, hpp:1492-1584). With LCP output a fourth
//      barrier precedes the LCPs at the bucket boundaries, which come from
//      the neighbouring buckets' key ranges (sample_sort_lcp, hpp:311-396).
// Every barrier wait is bounded: after `limit` polls a block sets
// ERR_TIMEOUT and returns, and the blocks still waiting see the flag and
// return as well.
#pragma once

#include "kernels_big.cuh"
#include "kernels_block.cuh"

namespace pssgpu {

constexpr int WAVE_THREADS = 512;
constexpr int WAVE_PER = 8;           // strings per thread through phases A-C
constexpr int WAVE_MAX_BITS = 11;     // at most 2047 splitters, 4095 buckets
constexpr int WAVE_BKT = 2 << WAVE_MAX_BITS;   // 4096 bucket slots
constexpr int WAVE_WINDOW = 1024;     // positions per window task
constexpr int WAVE_SORT_MAX = 2048;   // the block sorter of phase D
constexpr uint32_t WAVE_TILE_MAX = (uint32_t)WAVE_THREADS * WAVE_PER;
constexpr uint32_t WAVE_SAMPLE_CHUNK = WAVE_THREADS;  // samples one block draws and sorts

// Global state of one wave sort (in the workspace). The header is zeroed by
// the host before the launch; everything else is written inside.
struct WaveState {
    uint32_t bar;        // grid barrier arrivals
    uint32_t next_task;  // phase-D windows taken
    uint32_t pad[4];
    // with tracing on: the largest SM-clock cycles any block spent in phase
    // A (incl. block 0's samples), the first barrier wait, B (+ the second
    // wait), C (+ the third) and D (+ the LCPs)
    unsigned long long cycles[5];
    uint32_t gcount[WAVE_BKT];   // bucket counts
    uint64_t spl[WAVE_BKT / 2];  // sorted splitters
    uint64_t samp[WAVE_BKT];     // the samples, sorted in chunks of WAVE_SAMPLE_CHUNK
    uint64_t bmin[WAVE_BKT];     // key range of '<' buckets (LCP output only)
    uint64_t bmax[WAVE_BKT];
};

// Dynamic shared memory of k_wave: bucket starts, then either the phase A-C
// view (samples / tree, per-bucket counts) or the block sorter's.
struct WaveSmemABC {
    uint64_t m[2][WAVE_BKT];     // sample chunks merged back and forth; then the tree
    uint32_t cnt[WAVE_BKT];      // per bucket: count in the tile, then the tile's base
};
struct WaveSmem {
    uint32_t start[WAVE_BKT + 1];  // bucket starts (exclusive scan), start[B] = n
    uint32_t pad[3];
    union {
        WaveSmemABC abc;
        BlockSmem<WAVE_SORT_MAX> sort;
    } u;
};

// Grid barrier number `round` (1, 2, ...): every block arrives once; false
// when the wait gave up (ERR_TIMEOUT set here or by another block).
__device__ __forceinline__ bool wave_barrier(WaveState* ws, uint32_t round, uint32_t* err,
                                             uint32_t limit)
{
    __shared__ uint32_t ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&ws->bar, 1u);
        const uint32_t target = round * gridDim.x;
        uint32_t polls = 0;
        ok = 1;
        while (*(volatile uint32_t*)&ws->bar < target) {
            if ((*(volatile uint32_t*)err & ERR_TIMEOUT) || ++polls > limit) {
                set_error(err, ERR_TIMEOUT);
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// first b in [0, B] with start[b] >= x (start is non-decreasing, start[B] = n)
__device__ __forceinline__ uint32_t wave_lower(const uint32_t* start, uint32_t B, uint32_t x)
{
    uint32_t lo = 0, hi = B;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (start[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Key range of '<' bucket b (c >= 1 strings at position P of keys[1]) into
// ws->bmin / bmax, by the whole block; red is two words of shared memory.
__device__ __forceinline__ void wave_range_block(const Work& w, WaveState* ws, uint32_t b,
                                                 uint32_t P, uint32_t c, uint64_t* red)
{
    uint64_t mn = ~0ull, mx = 0;
    for (uint32_t q = threadIdx.x; q < c; q += WAVE_THREADS) {
        const uint64_t k = __ldcg(w.keys[1] + P + q);
        mn = min(mn, k);
        mx = max(mx, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (threadIdx.x == 0) {
        red[0] = ~0ull;
        red[1] = 0;
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        atomicMin((unsigned long long*)&red[0], (unsigned long long)mn);
        atomicMax((unsigned long long*)&red[1], (unsigned long long)mx);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ws->bmin[b] = red[0];
        ws->bmax[b] = red[1];
    }
    __syncthreads();
}

// Phase D: sort the strings at positions [P, P + m) of buffer 1, the buckets
// [b0, b1) (all of at most WAVE_SORT_MAX strings together), with the block
// sorter. The run is one group at depth 0: its buckets are consecutive key
// ranges and the keys at depth 0 are cached, so one sample-sort step over
// the whole run (about 8 strings per bucket) replaces a step per bucket.
// Bucket key ranges are recorded when the LCP array is wanted (the LCPs at
// the run's bucket boundaries follow from them).
__device__ __forceinline__ void wave_sort_run(const Work& w, WaveState* ws, WaveSmem& sm,
                                              uint32_t b0, uint32_t b1, uint32_t (*wscratch)[32],
                                              uint32_t* err)
{
    BlockSmem<WAVE_SORT_MAX>& bs = sm.u.sort;
    const uint32_t P = sm.start[b0], m = sm.start[b1] - P;
    if (m == 0) return;
    for (uint32_t i = threadIdx.x; i < m; i += WAVE_THREADS) {
        bs.hnd[i] = __ldcg(w.hnd[1] + P + i);
        bs.key[i] = __ldcg(w.keys[1] + P + i);
    }
    if (threadIdx.x == 0) {
        bs.ng = 0;
        bs.nw = 0;
        if (m > 1) blk_push<WAVE_SORT_MAX, WAVE_THREADS>(bs, 0, m, 0u, true, err);
    }
    __syncthreads();
    if (w.lcp) {
        for (uint32_t b = b0 + threadIdx.x; b < b1; b += WAVE_THREADS) {
            const uint32_t st = sm.start[b], c = sm.start[b + 1] - st;
            if (c == 0 || (b & 1)) continue;  // '=' buckets: the splitter is their key
            uint64_t mn = ~0ull, mx = 0;
            for (uint32_t q = 0; q < c; ++q) {
                mn = min(mn, bs.key[st - P + q]);
                mx = max(mx, bs.key[st - P + q]);
            }
            ws->bmin[b] = mn;
            ws->bmax[b] = mx;
        }
    }
    block_sort_groups<WAVE_SORT_MAX, WAVE_THREADS>(w, bs, P, m, 1, wscratch, err);
    __syncthreads();
}

// w.cur must be 0: the wave's leftovers (big segments, deep groups) go to
// the lists of parity 1, with their strings in buffer 1.
__global__ void __launch_bounds__(WAVE_THREADS, 2) k_wave(Work w, WaveState* ws, uint32_t L,
                                                          uint32_t limit, int trace)
{
    const long long c0 = clock64();
    long long cl = c0;
    auto lap = [&](int k) {  // phase k ended here (tracing only)
        if (!trace || threadIdx.x) return;
        const long long t = clock64();
        atomicMax(ws->cycles + k, (unsigned long long)(t - cl));
        cl = t;
    };
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WaveSmem& sm = *reinterpret_cast<WaveSmem*>(smem_raw);
    __shared__ uint32_t wscratch[WAVE_THREADS / 32][32];
    __shared__ uint32_t tmp[32];
    __shared__ uint64_t red[2];
    __shared__ uint32_t task, big_at;
    uint32_t* err = w.counters + C_ERR;
    const uint32_t G = gridDim.x, n = w.n;
    const uint32_t k = (1u << L) - 1, B = 2 * k + 1;
    const uint32_t per_blk = (n + G - 1) / G;  // <= WAVE_TILE_MAX (host)
    const uint32_t t0 = min(blockIdx.x * per_blk, n), t1 = min(t0 + per_blk, n);

    // ---- A: keys of the tile; samples and tree (block 0) ----------------
    for (uint32_t b = blockIdx.x * WAVE_THREADS + threadIdx.x; b < (uint32_t)WAVE_BKT;
         b += G * WAVE_THREADS)
        ws->gcount[b] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0 && w.chars[w.nchars - 1] != 0)
        set_error(err, ERR_UNTERMINATED);
    uint64_t key[WAVE_PER], hnd[WAVE_PER];
#pragma unroll
    for (int j = 0; j < WAVE_PER; ++j) {
        const uint32_t i = t0 + threadIdx.x + j * WAVE_THREADS;
        key[j] = 0;
        hnd[j] = 0;
        if (i < t1) {
            const uint64_t off = __ldg(w.offs + i);
            if (off >= w.nchars) set_error(err, ERR_OFFSET);
            hnd[j] = h_make(w, i, off);
            key[j] = load_key(w.chars, w.nchars, off);
        }
    }
    // 2^(L+1) samples (oversampling factor 2, hpp:1388), drawn and sorted in
    // chunks of WAVE_SAMPLE_CHUNK by the first blocks
    const uint32_t S = 2u << L;
    const uint32_t chunk = min(S, WAVE_SAMPLE_CHUNK);
    for (uint32_t c = blockIdx.x; c < S / chunk; c += G) {
        uint64_t* samp = sm.u.abc.m[0];
        if (threadIdx.x < chunk) {
            const uint64_t h = mix64(0x7761766573616d70ull ^ (c * chunk + threadIdx.x));
            const uint32_t r = (uint32_t)(((h >> 32) * n) >> 32);
            samp[threadIdx.x] = load_key(w.chars, w.nchars, __ldg(w.offs + r));
        }
        __syncthreads();
        bitonic_sort_block(samp, chunk);
        if (threadIdx.x < chunk) ws->samp[c * chunk + threadIdx.x] = samp[threadIdx.x];
        __syncthreads();
    }
    lap(0);
    if (!wave_barrier(ws, 1, err, limit)) return;
    lap(1);
    // input errors are all flagged in phase A: every block sees the same
    // bits here and leaves together
    if (*(volatile uint32_t*)err & (ERR_OFFSET | ERR_UNTERMINATED)) return;

    // ---- B: the splitter tree (every block), classify, count, reserve -----
    // Merge the sorted sample chunks (merge path: each thread makes 8
    // consecutive outputs of a pair of runs), then the splitters are every
    // second sample and the tree is their level order.
    uint64_t* src = sm.u.abc.m[0];
    uint64_t* dst = sm.u.abc.m[1];
    for (uint32_t i = threadIdx.x; i < S; i += WAVE_THREADS) src[i] = __ldcg(ws->samp + i);
    __syncthreads();
    for (uint32_t R = chunk; R < S; R <<= 1) {
        for (uint32_t o0 = 8 * threadIdx.x; o0 < S; o0 += 8 * WAVE_THREADS) {
            const uint64_t* A = src + (o0 / (2 * R)) * (2 * R);
            const uint64_t* Bv = A + R;
            const uint32_t d = o0 % (2 * R);
            // A-run members among the first d outputs (ties: A first)
            uint32_t lo = d > R ? d - R : 0u, hi = min(d, R);
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (A[mid] <= Bv[d - mid - 1]) lo = mid + 1; else hi = mid;
            }
            uint32_t i = lo, j = d - lo;
            uint64_t* out = dst + (o0 - d) + d;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const bool ta = j >= R || (i < R && A[i] <= Bv[j]);
                out[q] = ta ? A[i] : Bv[j];
                if (ta) ++i; else ++j;
            }
        }
        __syncthreads();
        uint64_t* t = src;
        src = dst;
        dst = t;
    }
    uint64_t* tree = dst;  // src holds the sorted samples
    uint32_t* cnt = sm.u.abc.cnt;
    if (blockIdx.x == 0)
        for (uint32_t j = threadIdx.x; j < k; j += WAVE_THREADS) ws->spl[j] = src[2 * j + 1];
    for (uint32_t v = 1 + threadIdx.x; v <= k; v += WAVE_THREADS) {
        const uint32_t h = 31 - __clz((int)v);
        const uint32_t p = v - (1u << h);
        const uint32_t r = ((2 * p + 1) << (L - 1 - h)) - 1;  // in-order rank
        tree[v] = src[2 * r + 1];
    }
    for (uint32_t b = threadIdx.x; b < B; b += WAVE_THREADS) cnt[b] = 0;
    __syncthreads();
    uint32_t pk[WAVE_PER];  // (bucket << 16) | rank inside the tile's share
#pragma unroll
    for (int j = 0; j < WAVE_PER; ++j) {
        const uint32_t i = t0 + threadIdx.x + j * WAVE_THREADS;
        pk[j] = 0xFFFFFFFFu;
        if (i < t1) {
            uint32_t v = 1;
            uint64_t cand = 0;
            for (uint32_t l = 0; l < L; ++l) {
                const uint64_t tv = tree[v];
                const bool gt = key[j] > tv;
                cand = gt ? cand : tv;
                v = 2 * v + (gt ? 1u : 0u);
            }
            const uint32_t r = v - (1u << L);
            const uint32_t b = 2 * r + ((r < k && cand == key[j]) ? 1u : 0u);
            pk[j] = (b << 16) | atomicAdd(&cnt[b], 1u);
        }
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < B; b += WAVE_THREADS) {
        const uint32_t c = cnt[b];
        cnt[b] = c ? atomicAdd(&ws->gcount[b], c) : 0u;
    }
    if (!wave_barrier(ws, 2, err, limit)) return;
    lap(2);

    // ---- C: bucket starts, scatter ----------------------------------------
    for (uint32_t b = threadIdx.x; b < B; b += WAVE_THREADS) sm.start[b] = __ldcg(ws->gcount + b);
    __syncthreads();
    block_scan_array<WAVE_THREADS>(sm.start, (int)B, tmp);
    if (threadIdx.x == 0) sm.start[B] = n;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < WAVE_PER; ++j) {
        if (pk[j] == 0xFFFFFFFFu) continue;
        const uint32_t b = pk[j] >> 16;
        const uint32_t dest = sm.start[b] + cnt[b] + (pk[j] & 0xFFFFu);
        if (dest >= n) {  // counts and starts disagree
            set_error(err, ERR_INTERNAL);
            continue;
        }
        w.keys[1][dest] = key[j];
        w.hnd[1][dest] = hnd[j];
    }
    if (!wave_barrier(ws, 3, err, limit)) return;
    lap(3);
    (void)c0;

    // ---- D: buckets over WAVE_WINDOW strings, one block each --------------
    for (uint32_t b = blockIdx.x; b < B; b += G) {
        const uint32_t P = sm.start[b], c = sm.start[b + 1] - P;
        if (c <= (uint32_t)WAVE_WINDOW) continue;
        const uint64_t s = (b & 1) ? __ldcg(ws->spl + (b >> 1)) : 0ull;
        if ((b & 1) && key_terminated(s)) {
            for (uint32_t q = threadIdx.x; q < c; q += WAVE_THREADS) {
                w.perm[P + q] = h_id(w, __ldcg(w.hnd[1] + P + q));
                if (w.lcp && q) w.lcp[P + q] = lcp_key_depth(s);
            }
        } else if (c <= (uint32_t)WAVE_SORT_MAX) {
            wave_sort_run(w, ws, sm, b, b + 1, wscratch, err);
        } else {
            if (w.lcp && !(b & 1)) wave_range_block(w, ws, b, P, c, red);
            if (threadIdx.x == 0)
                push_seg(w, 1, (b & 1) ? Seg{P, c, 8u, 1u} : Seg{P, c, 0u, 1u | META_VALID});
        }
        __syncthreads();
    }
    // ---- D: windows of small buckets ---------------------------------------
    const uint32_t ntask = (n + WAVE_WINDOW - 1) / WAVE_WINDOW;
    while (true) {
        if (threadIdx.x == 0) {
            task = atomicAdd(&ws->next_task, 1u);
            big_at = B;
        }
        __syncthreads();
        const uint32_t t = task;
        if (t >= ntask) break;
        const uint32_t lo = t * WAVE_WINDOW, hi = min(lo + WAVE_WINDOW, n);
        const uint32_t b_lo = wave_lower(sm.start, B, lo);
        const uint32_t b_hi = wave_lower(sm.start, B, hi);
        // at most one bucket over WAVE_WINDOW strings starts in a window
        for (uint32_t b = b_lo + threadIdx.x; b < b_hi; b += WAVE_THREADS)
            if (sm.start[b + 1] - sm.start[b] > (uint32_t)WAVE_WINDOW) atomicMin(&big_at, b);
        __syncthreads();
        const uint32_t bb = big_at;
        if (bb < b_hi) {
            wave_sort_run(w, ws, sm, b_lo, bb, wscratch, err);
            wave_sort_run(w, ws, sm, bb + 1, b_hi, wscratch, err);
        } else {
            wave_sort_run(w, ws, sm, b_lo, b_hi, wscratch, err);
        }
        __syncthreads();  // task and big_at are rewritten next round
    }
    if (!w.lcp) {
        lap(4);
        return;
    }

    // ---- LCPs at the bucket boundaries ---------------------------------------
    if (!wave_barrier(ws, 4, err, limit)) return;
    for (uint32_t b = blockIdx.x * WAVE_THREADS + threadIdx.x; b < B; b += G * WAVE_THREADS) {
        const uint32_t P = sm.start[b];
        if (P == 0 || sm.start[b + 1] == P) continue;
        uint32_t p = b - 1;  // previous non-empty bucket
        while (sm.start[p] == P) --p;
        const uint64_t hi_prev = (p & 1) ? __ldcg(ws->spl + (p >> 1)) : __ldcg(ws->bmax + p);
        const uint64_t lo_this = (b & 1) ? __ldcg(ws->spl + (b >> 1)) : __ldcg(ws->bmin + b);
        w.lcp[P] = lcp_key_type(hi_prev, lo_this);
    }
    lap(4);
}

}  // namespace pssgpu
