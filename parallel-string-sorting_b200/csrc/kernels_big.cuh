// kernels_big.cuh -- one sample-sort pass over the big segments (> SMALL_MAX
// strings). Restates pS5's SampleSortStep (src/parallel/
// bingmann-parallel_sample_sort.hpp:1264-1611) as a device pipeline:
//   k_tile_scan  tile offsets of the big segments
//   k_sample     SampleSortStep::sample + TreeBuilderLevelOrder (hpp:1384-1410,
//                src/sequential/bingmann-sample_sort_tree_builder.hpp:189-288)
//   k_classify   key gather + ClassifyTreeSimple::find_bkt + CountJob
//                (src/sequential/bingmann-sample_sortBTC.hpp:45-72, hpp:1414-1435)
//   k_bstart     count_finished: bucket prefix sums (hpp:1437-1460)
//   k_scatter    distribute: decoupled look-back + shared-memory staged scatter
//                (hpp:1464-1490)
//   k_children   distribute_finished: next segments, finished buckets, split
//                boundaries for the LCP array (hpp:1492-1584, 311-396)
//
// A segment whose samples are all equal takes the common-prefix jump instead
// of a classification: k_classify measures, for every string, the chars it
// shares with the segment's first string beyond the current depth; the
// segment then continues at depth + min (or is finished when all strings are
// equal). pS5 advances such a tied group 8 bytes per step (hpp:1527-1528,
// 1555-1556); the jump reaches the same depth in one pass.
#pragma once

#include "block_util.cuh"
#include "work.cuh"

namespace pssgpu {

__device__ __forceinline__ int find_tile_seg(const uint32_t* tile_start, int nbig, uint32_t t)
{
    // last s with tile_start[s] <= t
    int lo = 0, hi = nbig;  // invariant: tile_start[lo] <= t < tile_start[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(tile_start + mid) <= t) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t tree_bits_for(const Work& w, uint32_t m)
{
    // a tuned value for this size class, else about 16 strings per '<'
    // bucket; at most pS5's 10 tree levels
    const int lg = 31 - __clz((int)m);
    const uint32_t tuned = w.tree_bits_by_size[lg];
    if (tuned) return min((uint32_t)MAX_TREE_BITS, tuned);
    return (uint32_t)min(MAX_TREE_BITS, max(1, lg - 4));
}

__global__ void k_tile_scan(Work w, uint32_t nbig)
{
    __shared__ uint32_t tmp[32];
    const Seg* big = w.list[L_BIG][w.cur];
    const uint32_t per = (nbig + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = min(threadIdx.x * per, nbig), hi = min(lo + per, nbig);
    uint32_t s = 0;
    for (uint32_t i = lo; i < hi; ++i) s += (big[i].size + TILE - 1) / TILE;
    uint32_t total;
    uint32_t run = block_excl_sum<1024>(s, tmp, &total);
    for (uint32_t i = lo; i < hi; ++i) {
        w.tile_start[i] = run;
        run += (big[i].size + TILE - 1) / TILE;
    }
    if (threadIdx.x == 0) w.tile_start[nbig] = total;
}

// One block of 1024 threads per big segment.
__global__ void __launch_bounds__(1024) k_sample(Work w)
{
    __shared__ uint64_t samp[2 << MAX_TREE_BITS];
    const int s = blockIdx.x;
    const Seg sg = w.list[L_BIG][w.cur][s];
    uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    for (int b = threadIdx.x; b < MAX_BKT; b += blockDim.x) bc[b] = 0;
    if (sg.meta & META_FINAL) {
        if (threadIdx.x == 0) {
            w.tree_bits[s] = 0;
            atomicAdd(w.counters + C_P_FINAL, sg.size);
        }
        return;
    }
    const uint32_t L = tree_bits_for(w, sg.size);
    const uint32_t k = (1u << L) - 1;
    const uint32_t S = 2u << L;  // oversampling factor 2 (hpp:1388)
    const int buf = sg.meta & META_BUF;
    const bool valid = sg.meta & META_VALID;
    for (uint32_t i = threadIdx.x; i < S; i += blockDim.x) {
        const uint64_t h = mix64(((uint64_t)sg.begin << 32) ^ ((uint64_t)sg.depth << 12) ^ i);
        const uint32_t r = sg.begin + (uint32_t)(h % sg.size);
        samp[i] = valid ? w.keys[buf][r]
                        : h_key(w, w.hnd[buf][r], sg.depth);
    }
    __syncthreads();
    // bitonic sort of the S samples
    for (uint32_t kk = 2; kk <= S; kk <<= 1) {
        for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < S / 2; i += blockDim.x) {
                const uint32_t a = 2 * i - (i & (j - 1));
                const uint32_t b = a + j;
                const bool asc = (a & kk) == 0;
                const uint64_t x = samp[a], y = samp[b];
                if ((x > y) == asc) { samp[a] = y; samp[b] = x; }
            }
            __syncthreads();
        }
    }
    if (samp[0] == samp[S - 1] && !(sg.meta & META_NOTIE)) {
        // all samples equal: most likely one tied group -> common-prefix jump
        if (threadIdx.x == 0) {
            w.tree_bits[s] = TREE_TIE;
            w.jump_min[s] = 0xFFFFFFFFu;
            w.jump_diff[s] = 0;
            atomicAdd(w.counters + C_P_TIE, sg.size);
        }
        return;
    }
    if (threadIdx.x == 0) {
        atomicAdd(w.counters + C_P_BIG, sg.size);
        if (!valid) atomicAdd(w.counters + C_P_STALE, sg.size);
    }
    // splitters: every second sample; level-order tree over them
    uint64_t* spl = w.spl + (size_t)s * 1024;
    uint64_t* tree = w.tree + (size_t)s * 1024;
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) spl[j] = samp[2 * j + 1];
    for (uint32_t v = 1 + threadIdx.x; v <= k; v += blockDim.x) {
        const uint32_t h = 31 - __clz((int)v);
        const uint32_t p = v - (1u << h);
        const uint32_t r = ((2 * p + 1) << (L - 1 - h)) - 1;  // in-order rank
        tree[v] = samp[2 * r + 1];
    }
    if (threadIdx.x == 0) w.tree_bits[s] = (uint8_t)L;
}

// Chars the string behind handle h shares with the base string (at arena
// offset boff, both from depth d on); *differs is set when the two strings
// are not equal. Gives up (returning a value > stop) once the shared length
// exceeds `stop`, which then cannot lower the segment minimum. Two 8-byte
// chunks per step keep two loads of each string in flight.
__device__ __forceinline__ uint32_t shared_chars(const Work& w, uint64_t boff, uint64_t h,
                                                 uint32_t d, uint32_t stop, bool* differs)
{
    const uint64_t o = h_off(w, h) + d;
    for (uint32_t c = 0;; c += 2) {
        if (8u * c > stop) return 8u * c;
        const uint64_t ka0 = load_key(w.chars, w.nchars, boff + 8ull * c);
        const uint64_t kb0 = load_key(w.chars, w.nchars, o + 8ull * c);
        const uint64_t ka1 = load_key(w.chars, w.nchars, boff + 8ull * c + 8);
        const uint64_t kb1 = load_key(w.chars, w.nchars, o + 8ull * c + 8);
        if (ka0 != kb0) {
            *differs = true;
            return 8u * c + lcp_key_type(ka0, kb0);
        }
        if (key_terminated(ka0)) return 8u * c + lcp_key_depth(ka0);
        if (ka1 != kb1) {
            *differs = true;
            return 8u * c + 8 + lcp_key_type(ka1, kb1);
        }
        if (key_terminated(ka1)) return 8u * c + 8 + lcp_key_depth(ka1);
    }
}

// One block per tile of a big segment: gather keys if stale, classify,
// store bucket ids, add the tile histogram into the segment's counts.
// Tiles of finished (all-equal) segments copy ids and LCPs to the output;
// tiles of jump segments measure the common prefix.
__global__ void __launch_bounds__(TILE_THREADS) k_classify(Work w, uint32_t nbig)
{
    __shared__ uint64_t tree[1024];
    __shared__ uint32_t hist[MAX_BKT];
    __shared__ uint32_t best;
    __shared__ uint32_t anydiff;
    const uint32_t t = blockIdx.x;
    const int s = find_tile_seg(w.tile_start, nbig, t);
    const Seg sg = w.list[L_BIG][w.cur][s];
    const uint32_t lo = sg.begin + (t - w.tile_start[s]) * TILE;
    const uint32_t hi = min(lo + TILE, sg.begin + sg.size);
    const int buf = sg.meta & META_BUF;
    const uint64_t* hs = w.hnd[buf];
    if (sg.meta & META_FINAL) {
        for (uint32_t p = lo + threadIdx.x; p < hi; p += TILE_THREADS) {
            w.perm[p] = h_id(w, hs[p]);
            if (w.lcp && p > sg.begin) w.lcp[p] = sg.depth;
        }
        return;
    }
    const uint32_t L = w.tree_bits[s];
    if (L == TREE_TIE) {
        if (threadIdx.x == 0) {
            best = *((volatile uint32_t*)(w.jump_min + s));
            anydiff = 0;
        }
        __syncthreads();
        const uint64_t boff = h_off(w, hs[sg.begin]) + sg.depth;
        bool differs = false;
        for (uint32_t p = lo + threadIdx.x; p < hi; p += TILE_THREADS) {
            const uint32_t stop = *((volatile uint32_t*)&best);
            const uint32_t l = shared_chars(w, boff, hs[p], sg.depth, stop, &differs);
            if (l < stop) atomicMin(&best, l);
        }
        if (differs) anydiff = 1;
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicMin(w.jump_min + s, best);
            if (anydiff) atomicOr(w.jump_diff + s, 1u);
        }
        return;
    }
    const uint32_t k = (1u << L) - 1;
    const uint32_t B = 2 * k + 1;
    const uint64_t* gtree = w.tree + (size_t)s * 1024;
    for (uint32_t v = threadIdx.x; v <= k; v += TILE_THREADS) tree[v] = gtree[v];
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS) hist[b] = 0;
    __syncthreads();
    const bool valid = sg.meta & META_VALID;
    uint64_t* keys = w.keys[buf];
    for (uint32_t p = lo + threadIdx.x; p < hi; p += TILE_THREADS) {
        uint64_t key;
        if (valid) {
            key = keys[p];
        } else {
            key = h_key(w, hs[p], sg.depth);
            keys[p] = key;
        }
        uint32_t i = 1;
        uint64_t cand = 0;
        for (uint32_t l = 0; l < L; ++l) {
            const uint64_t tv = tree[i];
            const bool gt = key > tv;
            cand = gt ? cand : tv;
            i = 2 * i + (gt ? 1u : 0u);
        }
        const uint32_t r = i - (1u << L);  // splitters < key
        const uint32_t b = 2 * r + ((r < k && cand == key) ? 1u : 0u);
        w.bkt[p] = (uint16_t)b;
        atomicAdd(&hist[b], 1u);
    }
    __syncthreads();
    uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS)
        if (hist[b]) atomicAdd(bc + b, hist[b]);
}

__device__ __forceinline__ bool classified(uint8_t L)
{
    return L != 0 && L != TREE_TIE;
}

// Bucket starts (exclusive prefix over buckets) and the one-bucket test.
__global__ void __launch_bounds__(1024) k_bstart(Work w)
{
    __shared__ uint32_t a[MAX_BKT];
    __shared__ uint32_t tmp[32];
    __shared__ int one;
    const int s = blockIdx.x;
    const Seg sg = w.list[L_BIG][w.cur][s];
    const uint8_t L = w.tree_bits[s];
    if (!classified(L)) return;
    const uint32_t B = (2u << L) - 1;
    const uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    if (threadIdx.x == 0) one = 0;
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < MAX_BKT; b += 1024) {
        const uint32_t c = b < B ? bc[b] : 0u;
        a[b] = c;
        if (c == sg.size) one = 1;
    }
    __syncthreads();
    block_scan_array<1024>(a, MAX_BKT, tmp);
    uint32_t* bs = w.bstart + (size_t)s * MAX_BKT;
    for (uint32_t b = threadIdx.x; b < MAX_BKT; b += 1024) bs[b] = a[b];
    if (threadIdx.x == 0) {
        w.bflags[s] = (uint8_t)one;
        if (!one) atomicAdd(w.counters + C_P_SCATTER, sg.size);
    }
}

// Decoupled look-back status word: epoch (16) | flag (2) | count (46).
constexpr uint64_t LB_AGG = 1ull, LB_PRE = 2ull;
__device__ __forceinline__ uint64_t lb_word(uint32_t epoch, uint64_t flag, uint64_t v)
{
    return ((uint64_t)epoch << 48) | (flag << 46) | v;
}

struct ScatterSmem {
    uint64_t stage[TILE];      // the tile's keys in bucket order, then its handles
    uint16_t sbkt[TILE];       // bucket of each staged slot
    uint32_t lcount[MAX_BKT];  // per-bucket count in the tile, then its start
    uint32_t gdelta[MAX_BKT];  // per bucket: global position - tile slot
    uint32_t tmp[32];
    uint32_t vt;
};

// One block per tile, tiles taken in ticket order so that every tile's
// predecessors in its segment are already resident or done.
__global__ void __launch_bounds__(TILE_THREADS) k_scatter(Work w, uint32_t nbig)
{
    constexpr int PER = TILE / TILE_THREADS;
    constexpr int NB = MAX_BKT / TILE_THREADS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScatterSmem& sm = *reinterpret_cast<ScatterSmem*>(smem_raw);
    if (threadIdx.x == 0) sm.vt = atomicAdd(w.counters + C_TICKET, 1u);
    __syncthreads();
    const uint32_t vt = sm.vt;
    const int s = find_tile_seg(w.tile_start, nbig, vt);
    const Seg sg = w.list[L_BIG][w.cur][s];
    const uint8_t L = w.tree_bits[s];
    if (!classified(L) || w.bflags[s]) return;
    const uint32_t tin = vt - w.tile_start[s];
    const uint32_t lo = sg.begin + tin * TILE;
    const uint32_t hi = min(lo + TILE, sg.begin + sg.size);
    const uint32_t cnt = hi - lo;
    const uint32_t B = (2u << L) - 1;
    const int buf = sg.meta & META_BUF;
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS) sm.lcount[b] = 0;
    __syncthreads();
    // rank of every string inside its bucket in this tile: (bucket << 16) | rank
    uint32_t pk[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint32_t p = lo + threadIdx.x + j * TILE_THREADS;
        pk[j] = 0xFFFFFFFFu;
        if (p < hi) {
            const uint32_t b = w.bkt[p];
            pk[j] = (b << 16) | atomicAdd(&sm.lcount[b], 1u);
        }
    }
    __syncthreads();
    // publish this tile's per-bucket counts, then look back for the prefix
    volatile uint64_t* st = w.status + (size_t)vt * MAX_BKT;
    const uint32_t ep = w.epoch;
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS)
        st[b] = lb_word(ep, tin == 0 ? LB_PRE : LB_AGG, sm.lcount[b]);
    // Look back for every bucket this thread owns at once: each round issues
    // one status load per unfinished bucket, so the chains overlap in memory.
    uint64_t excl[NB];
    uint32_t jb[NB];
    uint32_t open = 0;  // bit i: bucket threadIdx.x + i * TILE_THREADS still walking
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        excl[i] = 0;
        jb[i] = vt - 1;
        const uint32_t b = threadIdx.x + i * TILE_THREADS;
        if (tin > 0 && b < B) open |= 1u << i;
    }
    uint32_t spins = 0;
    while (open) {
        uint64_t wd[NB];
#pragma unroll
        for (int i = 0; i < NB; ++i)
            if (open & (1u << i))
                wd[i] = *((volatile uint64_t*)(w.status + (size_t)jb[i] * MAX_BKT + threadIdx.x +
                                               i * TILE_THREADS));
        bool waiting = false;
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            if (!(open & (1u << i))) continue;
            const uint64_t flag = (wd[i] >> 46) & 3u;
            if ((uint32_t)(wd[i] >> 48) != ep || flag == 0) {
                waiting = true;
                continue;
            }
            excl[i] += wd[i] & ((1ull << 46) - 1);
            if (flag == LB_PRE) open &= ~(1u << i);
            else --jb[i];
        }
        if (waiting) {
            // bounded wait: give up (and make every later wait give up at
            // once) after SPIN_CAP polls
            if (++spins > SPIN_CAP || (*((volatile uint32_t*)(w.counters + C_ERR)) & ERR_TIMEOUT)) {
                set_error(w.counters + C_ERR, ERR_TIMEOUT);
                break;
            }
            if (spins > 64) __nanosleep(64);
        }
    }
    if (tin > 0) {
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            const uint32_t b = threadIdx.x + i * TILE_THREADS;
            if (b < B) st[b] = lb_word(ep, LB_PRE, excl[i] + sm.lcount[b]);
        }
    }
    __syncthreads();
    block_scan_array<TILE_THREADS>(sm.lcount, (int)B, sm.tmp);  // counts -> tile starts
    const uint32_t* bs = w.bstart + (size_t)s * MAX_BKT;
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const uint32_t b = threadIdx.x + i * TILE_THREADS;
        if (b < B) sm.gdelta[b] = sg.begin + bs[b] + (uint32_t)excl[i] - sm.lcount[b];
    }
    // stage keys in bucket order and write bucket runs contiguously; then ids
    const uint64_t* ikeys = w.keys[buf];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        if (pk[j] == 0xFFFFFFFFu) continue;
        const uint32_t b = pk[j] >> 16;
        const uint32_t slot = sm.lcount[b] + (pk[j] & 0xFFFFu);
        sm.stage[slot] = ikeys[lo + threadIdx.x + j * TILE_THREADS];
        sm.sbkt[slot] = (uint16_t)b;
    }
    __syncthreads();
    uint64_t* okeys = w.keys[buf ^ 1];
    for (uint32_t slot = threadIdx.x; slot < cnt; slot += TILE_THREADS) {
        const uint32_t dest = slot + sm.gdelta[sm.sbkt[slot]];
        if (dest - sg.begin >= sg.size) {  // only after a failed look-back
            set_error(w.counters + C_ERR, ERR_INTERNAL);
            continue;
        }
        okeys[dest] = sm.stage[slot];
    }
    __syncthreads();
    const uint64_t* ihs = w.hnd[buf];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        if (pk[j] == 0xFFFFFFFFu) continue;
        const uint32_t slot = sm.lcount[pk[j] >> 16] + (pk[j] & 0xFFFFu);
        sm.stage[slot] = ihs[lo + threadIdx.x + j * TILE_THREADS];
    }
    __syncthreads();
    uint64_t* ohs = w.hnd[buf ^ 1];
    for (uint32_t slot = threadIdx.x; slot < cnt; slot += TILE_THREADS) {
        const uint32_t dest = slot + sm.gdelta[sm.sbkt[slot]];
        if (dest - sg.begin >= sg.size) continue;
        ohs[dest] = sm.stage[slot];
    }
}

__device__ __forceinline__ void push_seg(Work& w, int nxt, Seg c)
{
    int cls;
    if (c.size > SMALL_MAX) cls = L_BIG;
    else if (c.size > 256) cls = L_SMALLB;
    else if (c.size > WARP_GROUP_MAX) cls = L_SMALLA;
    else cls = L_TINY;
    const uint32_t at = atomicAdd(w.counters + C_PAR * nxt + cls, 1u);
    if (at >= w.cap[cls]) {
        set_error(w.counters + C_ERR, ERR_OVERFLOW);
        return;
    }
    w.list[cls][nxt][at] = c;
    if (cls == L_BIG) atomicAdd(w.counters + C_PAR * nxt + C_NTILES, (c.size + TILE - 1) / TILE);
    else atomicAdd(w.counters + C_PAR * nxt + C_NSTR + cls, c.size);
}

// Children of each bucket, after the scatter has placed them; the next
// segment of a jump segment.
__global__ void __launch_bounds__(1024) k_children(Work w)
{
    const int s = blockIdx.x;
    const Seg sg = w.list[L_BIG][w.cur][s];
    const uint8_t L = w.tree_bits[s];
    const int buf = sg.meta & META_BUF;
    const int nxt = w.cur ^ 1;
    if (L == TREE_TIE) {
        if (threadIdx.x == 0) {
            const uint32_t mn = w.jump_min[s];
            if (!w.jump_diff[s])  // every string equals the base
                push_seg(w, nxt, Seg{sg.begin, sg.size, sg.depth + mn, (uint32_t)buf | META_FINAL});
            else if (mn == 0)     // no shared char: classify at this depth
                push_seg(w, nxt, Seg{sg.begin, sg.size, sg.depth, (uint32_t)buf | META_NOTIE});
            else
                push_seg(w, nxt, Seg{sg.begin, sg.size, sg.depth + mn, (uint32_t)buf});
        }
        return;
    }
    if (!classified(L)) return;
    // block-aggregated appends: slots in shared memory first, then one
    // global reservation per list
    __shared__ uint32_t lcnt[L_NCLASS], gbase[L_NCLASS], lstr[L_NCLASS];
    __shared__ uint32_t ltiles, lbnd, bbase;
    if (threadIdx.x < L_NCLASS) { lcnt[threadIdx.x] = 0; lstr[threadIdx.x] = 0; }
    if (threadIdx.x == 0) { ltiles = 0; lbnd = 0; }
    __syncthreads();
    const uint32_t B = (2u << L) - 1;
    const int nbuf = w.bflags[s] ? buf : buf ^ 1;
    const uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    const uint32_t* bs = w.bstart + (size_t)s * MAX_BKT;
    const uint64_t* spl = w.spl + (size_t)s * 1024;
    const uint64_t* hs = w.hnd[nbuf];
    constexpr int PER = (MAX_BKT + 1023) / 1024;
    Seg child[PER];
    int cls[PER];
    uint32_t slot[PER], bslot[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        cls[j] = -1;
        bslot[j] = 0xFFFFFFFFu;
        const uint32_t b = threadIdx.x + 1024u * j;
        if (b >= B) continue;
        const uint32_t c = bc[b];
        if (c == 0) continue;
        const uint32_t P = sg.begin + bs[b];
        if (P > sg.begin && w.lcp) bslot[j] = atomicAdd(&lbnd, 1u);
        if (c == 1) {
            w.perm[P] = h_id(w, hs[P]);
            continue;
        }
        if (b & 1) {
            const uint64_t key = spl[b >> 1];
            if (key_terminated(key)) {
                const uint32_t v = sg.depth + lcp_key_depth(key);
                if (c <= FINAL_INLINE) {
                    for (uint32_t q = 0; q < c; ++q) {
                        w.perm[P + q] = h_id(w, hs[P + q]);
                        if (w.lcp && q) w.lcp[P + q] = v;
                    }
                    continue;
                }
                child[j] = Seg{P, c, v, (uint32_t)nbuf | META_FINAL};
            } else {
                child[j] = Seg{P, c, sg.depth + 8, (uint32_t)nbuf};
            }
        } else {
            child[j] = Seg{P, c, sg.depth, (uint32_t)nbuf | META_VALID};
        }
        if (c > SMALL_MAX) cls[j] = L_BIG;
        else if (c > 256) cls[j] = L_SMALLB;
        else if (c > WARP_GROUP_MAX) cls[j] = L_SMALLA;
        else cls[j] = L_TINY;
        slot[j] = atomicAdd(&lcnt[cls[j]], 1u);
        if (cls[j] == L_BIG) atomicAdd(&ltiles, (c + TILE - 1) / TILE);
        else atomicAdd(&lstr[cls[j]], c);
    }
    __syncthreads();
    if (threadIdx.x < L_NCLASS && lcnt[threadIdx.x])
        gbase[threadIdx.x] = atomicAdd(w.counters + C_PAR * nxt + threadIdx.x, lcnt[threadIdx.x]);
    if (threadIdx.x == 32 && ltiles) atomicAdd(w.counters + C_PAR * nxt + C_NTILES, ltiles);
    if (threadIdx.x >= 33 && threadIdx.x < 32 + L_NCLASS && lstr[threadIdx.x - 32])
        atomicAdd(w.counters + C_PAR * nxt + C_NSTR + (threadIdx.x - 32), lstr[threadIdx.x - 32]);
    if (threadIdx.x == 64 && lbnd) bbase = atomicAdd(w.counters + C_NBND, lbnd);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint32_t b = threadIdx.x + 1024u * j;
        if (b >= B) continue;
        if (bslot[j] != 0xFFFFFFFFu) {
            const uint32_t at = bbase + bslot[j];
            if (at < w.bnd_cap) w.bnd[at] = make_uint2(sg.begin + bs[b], sg.depth);
            else set_error(w.counters + C_ERR, ERR_OVERFLOW);
        }
        if (cls[j] >= 0) {
            const uint32_t at = gbase[cls[j]] + slot[j];
            if (at < w.cap[cls[j]]) w.list[cls[j]][nxt][at] = child[j];
            else set_error(w.counters + C_ERR, ERR_OVERFLOW);
        }
    }
}

// LCP at each split boundary: the two strings met at `depth` in different
// buckets, so their keys at that depth differ (sample_sort_lcp, hpp:311-396).
__global__ void k_boundary_lcp(Work w)
{
    const uint32_t nb = min(w.counters[C_NBND], w.bnd_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
        const uint2 e = w.bnd[i];
        const uint32_t P = e.x, d = e.y;
        const uint64_t ka = gather_key(w.chars, w.nchars, w.offs, w.perm[P - 1], d);
        const uint64_t kb = gather_key(w.chars, w.nchars, w.offs, w.perm[P], d);
        w.lcp[P] = d + lcp_key_type(ka, kb);
    }
}

}  // namespace pssgpu
