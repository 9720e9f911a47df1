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

__device__ __forceinline__ uint32_t tree_bits_for(uint32_t m)
{
    // about 32 strings per '<' bucket, at most pS5's 10 tree levels
    const int lg = 31 - __clz((int)m);
    return (uint32_t)min(MAX_TREE_BITS, max(1, lg - 5));
}

__global__ void k_tile_scan(Work w, uint32_t nbig)
{
    __shared__ uint32_t tmp[32];
    const Seg* big = w.big[w.cur];
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
    const Seg sg = w.big[w.cur][s];
    uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    for (int b = threadIdx.x; b < MAX_BKT; b += blockDim.x) bc[b] = 0;
    if (sg.meta & META_FINAL) {
        if (threadIdx.x == 0) {
            w.tree_bits[s] = 0;
            atomicAdd(w.counters + C_P_FINAL, sg.size);
        }
        return;
    }
    if (threadIdx.x == 0) {
        atomicAdd(w.counters + C_P_BIG, sg.size);
        if (!(sg.meta & META_VALID)) atomicAdd(w.counters + C_P_STALE, sg.size);
    }
    const uint32_t L = tree_bits_for(sg.size);
    const uint32_t k = (1u << L) - 1;
    const uint32_t S = 2u << L;  // oversampling factor 2 (hpp:1388)
    const int buf = sg.meta & META_BUF;
    const bool valid = sg.meta & META_VALID;
    for (uint32_t i = threadIdx.x; i < S; i += blockDim.x) {
        const uint64_t h = mix64(((uint64_t)sg.begin << 32) ^ ((uint64_t)sg.depth << 12) ^ i);
        const uint32_t r = sg.begin + (uint32_t)(h % sg.size);
        samp[i] = valid ? w.keys[buf][r]
                        : gather_key(w.chars, w.nchars, w.offs, w.ids[buf][r], sg.depth);
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

// One block per tile of a big segment: gather keys if stale, classify,
// store bucket ids, add the tile histogram into the segment's counts.
// Tiles of finished (all-equal) segments copy ids and LCPs to the output.
__global__ void __launch_bounds__(TILE_THREADS) k_classify(Work w, uint32_t nbig)
{
    __shared__ uint64_t tree[1024];
    __shared__ uint32_t hist[MAX_BKT];
    const uint32_t t = blockIdx.x;
    const int s = find_tile_seg(w.tile_start, nbig, t);
    const Seg sg = w.big[w.cur][s];
    const uint32_t lo = sg.begin + (t - w.tile_start[s]) * TILE;
    const uint32_t hi = min(lo + TILE, sg.begin + sg.size);
    const int buf = sg.meta & META_BUF;
    if (sg.meta & META_FINAL) {
        for (uint32_t p = lo + threadIdx.x; p < hi; p += TILE_THREADS) {
            w.perm[p] = w.ids[buf][p];
            if (w.lcp && p > sg.begin) w.lcp[p] = sg.depth;
        }
        return;
    }
    const uint32_t L = w.tree_bits[s];
    const uint32_t k = (1u << L) - 1;
    const uint32_t B = 2 * k + 1;
    const uint64_t* gtree = w.tree + (size_t)s * 1024;
    for (uint32_t v = threadIdx.x; v <= k; v += TILE_THREADS) tree[v] = gtree[v];
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS) hist[b] = 0;
    __syncthreads();
    const bool valid = sg.meta & META_VALID;
    const uint32_t* ids = w.ids[buf];
    uint64_t* keys = w.keys[buf];
    for (uint32_t p = lo + threadIdx.x; p < hi; p += TILE_THREADS) {
        uint64_t key;
        if (valid) {
            key = keys[p];
        } else {
            key = gather_key(w.chars, w.nchars, w.offs, ids[p], sg.depth);
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

// Bucket starts (exclusive prefix over buckets) and the one-bucket test.
__global__ void __launch_bounds__(1024) k_bstart(Work w)
{
    __shared__ uint32_t a[MAX_BKT];
    __shared__ uint32_t tmp[32];
    __shared__ int one;
    const int s = blockIdx.x;
    const Seg sg = w.big[w.cur][s];
    if (sg.meta & META_FINAL) return;
    const uint32_t L = w.tree_bits[s];
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
    uint64_t key[TILE];
    uint32_t id[TILE];
    uint16_t bkt[TILE];
    uint32_t lcount[MAX_BKT];
    uint32_t lstart[MAX_BKT];
    uint32_t gbase[MAX_BKT];
    uint32_t tmp[32];
    uint32_t vt;
};

// One block per tile, tiles taken in ticket order so that every tile's
// predecessors in its segment are already resident or done.
__global__ void __launch_bounds__(TILE_THREADS) k_scatter(Work w, uint32_t nbig)
{
    constexpr int PER = TILE / TILE_THREADS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScatterSmem& sm = *reinterpret_cast<ScatterSmem*>(smem_raw);
    uint64_t* skey = sm.key;
    uint32_t* sid = sm.id;
    uint16_t* sbkt = sm.bkt;
    uint32_t* lcount = sm.lcount;
    uint32_t* lstart = sm.lstart;
    uint32_t* gbase = sm.gbase;
    uint32_t* tmp = sm.tmp;
    uint32_t& vt_s = sm.vt;
    if (threadIdx.x == 0) vt_s = atomicAdd(w.counters + C_TICKET, 1u);
    __syncthreads();
    const uint32_t vt = vt_s;
    const int s = find_tile_seg(w.tile_start, nbig, vt);
    const Seg sg = w.big[w.cur][s];
    if ((sg.meta & META_FINAL) || w.bflags[s]) return;
    const uint32_t tin = vt - w.tile_start[s];
    const uint32_t lo = sg.begin + tin * TILE;
    const uint32_t hi = min(lo + TILE, sg.begin + sg.size);
    const uint32_t cnt = hi - lo;
    const uint32_t L = w.tree_bits[s];
    const uint32_t B = (2u << L) - 1;
    const int buf = sg.meta & META_BUF;
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS) lcount[b] = 0;
    __syncthreads();
    uint64_t key[PER];
    uint32_t id[PER], bk[PER], rank[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint32_t p = lo + threadIdx.x + j * TILE_THREADS;
        if (p < hi) {
            key[j] = w.keys[buf][p];
            id[j] = w.ids[buf][p];
            bk[j] = w.bkt[p];
            rank[j] = atomicAdd(&lcount[bk[j]], 1u);
        }
    }
    __syncthreads();
    // publish this tile's per-bucket counts, then look back for the prefix
    volatile uint64_t* st = w.status + (size_t)vt * MAX_BKT;
    const uint32_t ep = w.epoch;
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS)
        st[b] = lb_word(ep, tin == 0 ? LB_PRE : LB_AGG, lcount[b]);
    const uint32_t* bs = w.bstart + (size_t)s * MAX_BKT;
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS) {
        uint64_t excl = 0;
        if (tin > 0) {
            uint32_t j = vt - 1;
            uint32_t spins = 0;
            while (true) {
                const uint64_t wd = *((volatile uint64_t*)(w.status + (size_t)j * MAX_BKT + b));
                const uint64_t flag = (wd >> 46) & 3u;
                if ((uint32_t)(wd >> 48) != ep || flag == 0) {
                    // bounded wait: give up (and make every later wait give up
                    // at once) after SPIN_CAP polls
                    if (++spins > SPIN_CAP ||
                        (*((volatile uint32_t*)(w.counters + C_ERR)) & ERR_TIMEOUT)) {
                        set_error(w.counters + C_ERR, ERR_TIMEOUT);
                        break;
                    }
                    if (spins > 64) __nanosleep(64);
                    continue;
                }
                excl += wd & ((1ull << 46) - 1);
                if (flag == LB_PRE) break;
                --j;
            }
            st[b] = lb_word(ep, LB_PRE, excl + lcount[b]);
        }
        gbase[b] = sg.begin + bs[b] + (uint32_t)excl;
        lstart[b] = lcount[b];
    }
    __syncthreads();
    block_scan_array<TILE_THREADS>(lstart, (int)B, tmp);
    // stage the tile in bucket order, then write bucket runs contiguously
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint32_t p = lo + threadIdx.x + j * TILE_THREADS;
        if (p < hi) {
            const uint32_t slot = lstart[bk[j]] + rank[j];
            skey[slot] = key[j];
            sid[slot] = id[j];
            sbkt[slot] = (uint16_t)bk[j];
        }
    }
    __syncthreads();
    uint64_t* okeys = w.keys[buf ^ 1];
    uint32_t* oids = w.ids[buf ^ 1];
    for (uint32_t slot = threadIdx.x; slot < cnt; slot += TILE_THREADS) {
        const uint32_t b = sbkt[slot];
        const uint32_t dest = gbase[b] + (slot - lstart[b]);
        if (dest - sg.begin >= sg.size) {  // only after a failed look-back
            set_error(w.counters + C_ERR, ERR_INTERNAL);
            continue;
        }
        okeys[dest] = skey[slot];
        oids[dest] = sid[slot];
    }
}

__device__ __forceinline__ void push_seg(Work& w, int nxt, Seg c)
{
    if (c.size > SMALL_MAX) {
        const uint32_t at = atomicAdd(w.counters + 3 * nxt + C_NBIG, 1u);
        if (at >= w.big_cap) { set_error(w.counters + C_ERR, ERR_OVERFLOW); return; }
        w.big[nxt][at] = c;
        atomicAdd(w.counters + 3 * nxt + C_NTILES, (c.size + TILE - 1) / TILE);
    } else {
        const uint32_t at = atomicAdd(w.counters + 3 * nxt + C_NSMALL, 1u);
        if (at >= w.small_cap) { set_error(w.counters + C_ERR, ERR_OVERFLOW); return; }
        w.small[nxt][at] = c;
    }
}

// Children of each bucket, after the scatter has placed them.
__global__ void __launch_bounds__(1024) k_children(Work w)
{
    const int s = blockIdx.x;
    const Seg sg = w.big[w.cur][s];
    if (sg.meta & META_FINAL) return;
    const uint32_t L = w.tree_bits[s];
    const uint32_t B = (2u << L) - 1;
    const int buf = sg.meta & META_BUF;
    const int nbuf = w.bflags[s] ? buf : buf ^ 1;
    const uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    const uint32_t* bs = w.bstart + (size_t)s * MAX_BKT;
    const uint64_t* spl = w.spl + (size_t)s * 1024;
    const int nxt = w.cur ^ 1;
    const uint32_t* ids = w.ids[nbuf];
    for (uint32_t b = threadIdx.x; b < B; b += blockDim.x) {
        const uint32_t c = bc[b];
        if (c == 0) continue;
        const uint32_t P = sg.begin + bs[b];
        if (P > sg.begin && w.lcp) {
            const uint32_t at = atomicAdd(w.counters + C_NBND, 1u);
            if (at < w.bnd_cap) w.bnd[at] = make_uint2(P, sg.depth);
            else set_error(w.counters + C_ERR, ERR_OVERFLOW);
        }
        if (c == 1) {
            w.perm[P] = ids[P];
            continue;
        }
        if (b & 1) {
            const uint64_t key = spl[b >> 1];
            if (key_terminated(key)) {
                const uint32_t v = sg.depth + lcp_key_depth(key);
                if (c <= FINAL_INLINE) {
                    for (uint32_t q = 0; q < c; ++q) {
                        w.perm[P + q] = ids[P + q];
                        if (w.lcp && q) w.lcp[P + q] = v;
                    }
                } else {
                    push_seg(w, nxt, Seg{P, c, v, (uint32_t)nbuf | META_FINAL});
                }
            } else {
                push_seg(w, nxt, Seg{P, c, sg.depth + 8, (uint32_t)nbuf});
            }
        } else {
            push_seg(w, nxt, Seg{P, c, sg.depth, (uint32_t)nbuf | META_VALID});
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
