// kernels_big.cuh -- one sample-sort pass over the big segments (> SMALL_MAX
// strings). Restates pS5's SampleSortStep (src/parallel/
// bingmann-parallel_sample_sort.hpp:1264-1611) as a device pipeline:
//   k_tile_scan  tile offsets of the big segments
//   k_sample     SampleSortStep::sample + TreeBuilderLevelOrder (hpp:1384-1410,
//                src/sequential/bingmann-sample_sort_tree_builder.hpp:189-288)
//   k_classify   key gather + ClassifyTreeSimple::find_bkt + CountJob
//                (src/sequential/bingmann-sample_sortBTC.hpp:45-72, hpp:1414-1435)
//   k_bstart     count_finished: bucket prefix sums and every tile's first
//                destination per bucket (hpp:1437-1460)
//   k_chunk_sum, k_chunk_scan, k_tile_offsets
//                the same for segments of more than CHUNK tiles, in chunks
//   k_scatter    distribute: shared-memory staged scatter (hpp:1464-1490)
//   k_children   distribute_finished: next segments, finished buckets, split
//                boundaries for the LCP array (hpp:1492-1584, 311-396)
//
// A segment whose samples all share more chars beyond the current depth
// takes a common-prefix jump inside its pass: k_sample measures the shared
// chunks (up to JMAX_CHUNKS) and builds the tree behind them; k_classify
// checks every string against the shared chunks and sends the few that leave
// the prefix early to two extra buckets. pS5 advances such a tied group 8
// bytes per step (hpp:1527-1528, 1555-1556).
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
    // a tuned value for this size class, else about 8 strings per '<'
    // bucket; at most pS5's 10 tree levels
    const int lg = 31 - __clz((int)m);
    const uint32_t tuned = w.tree_bits_by_size[lg];
    if (tuned) return min((uint32_t)MAX_TREE_BITS, tuned);
    return (uint32_t)min(MAX_TREE_BITS, max(1, lg - 3));
}

__global__ void k_tile_scan(Work w, uint32_t nbig)
{
    __shared__ uint32_t tmp[32];
    const Seg* big = w.list[L_BIG][w.cur];
    const uint32_t per = (nbig + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = min(threadIdx.x * per, nbig), hi = min(lo + per, nbig);
    auto tiles = [&](uint32_t i) { return (big[i].size + TILE - 1) / TILE; };
    auto chunks = [&](uint32_t i) { return (tiles(i) + CHUNK - 1) / CHUNK; };
    uint32_t s = 0, sc = 0;
    for (uint32_t i = lo; i < hi; ++i) {
        s += tiles(i);
        sc += chunks(i);
    }
    uint32_t total, ctotal;
    uint32_t run = block_excl_sum<1024>(s, tmp, &total);
    uint32_t crun = block_excl_sum<1024>(sc, tmp, &ctotal);
    for (uint32_t i = lo; i < hi; ++i) {
        w.tile_start[i] = run;
        w.chunk_start[i] = crun;
        run += tiles(i);
        crun += chunks(i);
    }
    if (threadIdx.x == 0) {
        w.tile_start[nbig] = total;
        w.chunk_start[nbig] = ctotal;
    }
}

// One block per big segment (256 threads, or 1024 when the pass has few
// segments and each block's latency is the pass's).
__global__ void __launch_bounds__(1024) k_sample(Work w)
{
    __shared__ uint64_t samp[2 << MAX_TREE_BITS];
    __shared__ uint64_t shnd[2 << MAX_TREE_BITS];
    __shared__ uint64_t smin, smax;
    __shared__ uint32_t jrun;
    const int s = blockIdx.x;
    const Seg sg = w.list[L_BIG][w.cur][s];
    uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    for (int b = threadIdx.x; b < MAX_BKT; b += blockDim.x) bc[b] = 0;
    if (sg.meta & META_FINAL) {
        if (threadIdx.x == 0) {
            w.tree_bits[s] = 0;
            w.jump[s] = 0;
            atomicAdd(w.counters + C_P_FINAL, sg.size);
        }
        return;
    }
    const uint32_t L = tree_bits_for(w, sg.size);
    const uint32_t k = (1u << L) - 1;
    // one sample per bucket slot: 2^L sorted samples, the splitters are all
    // but the first. pS5 oversamples by 2 (hpp:1388); here half the
    // samples halve the bitonic sort, which is most of this kernel's work,
    // while '<' buckets still hold about 8 strings on average
    const uint32_t S = 1u << L;
    const int buf = sg.meta & META_BUF;
    const bool valid = sg.meta & META_VALID;
    // handles (and cached keys) of the samples, then the keys of stale ones:
    // every load of a round is independent
#pragma unroll 8
    for (uint32_t i = threadIdx.x; i < S; i += blockDim.x) {
        const uint64_t h = mix64(((uint64_t)sg.begin << 32) ^ ((uint64_t)sg.depth << 12) ^ i);
        const uint32_t r = sg.begin + (uint32_t)(((h >> 32) * sg.size) >> 32);
        shnd[i] = w.hnd[buf][r];
        if (valid) samp[i] = w.keys[buf][r];
    }
    if (!valid) {
        __syncthreads();
#pragma unroll 8
        for (uint32_t i = threadIdx.x; i < S; i += blockDim.x) samp[i] = h_key(w, shnd[i], sg.depth);
    }
    // all samples equal? (a min / max reduction; the sort comes once the
    // depth of the splitters is known)
    if (threadIdx.x == 0) {
        smin = ~0ull;
        smax = 0;
    }
    __syncthreads();
    {
        uint64_t mn = ~0ull, mx = 0;
        for (uint32_t i = threadIdx.x; i < S; i += blockDim.x) {
            mn = min(mn, samp[i]);
            mx = max(mx, samp[i]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin((unsigned long long*)&smin, (unsigned long long)mn);
            atomicMax((unsigned long long*)&smax, (unsigned long long)mx);
        }
    }
    __syncthreads();
    uint32_t J = 0;  // chunks of the common-prefix jump
    if (smin == smax && !key_terminated(smin)) {
        // Every sample shares the chunk at the segment depth: count the
        // further chunks that the first (up to blockDim) samples share with
        // sample 0, four per round, up to JMAX_CHUNKS. pS5 would advance such
        // a tied group one chunk per step (hpp:1527-1528, 1555-1556). Any
        // jump that sample 0 has is correct: strings leaving its prefix go
        // to the two prefix buckets, and splitters may be any keys.
        const uint64_t ref = h_off(w, shnd[0]) + sg.depth;
        const uint32_t JS = min(S, blockDim.x);
        J = 1;
        while (J < (uint32_t)JMAX_CHUNKS) {
            if (threadIdx.x == 0) jrun = 4;
            __syncthreads();
            uint64_t rk[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) rk[q] = load_key(w.chars, w.nchars, ref + 8ull * (J + q));
            uint32_t mine = 4;
            if (threadIdx.x < JS) {
                const uint64_t o = h_off(w, shnd[threadIdx.x]) + sg.depth;
                uint32_t e = 0;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint64_t kq = load_key(w.chars, w.nchars, o + 8ull * (J + q));
                    if (e == (uint32_t)q && kq == rk[q] && !key_terminated(kq)) e = q + 1;
                }
                mine = min(mine, e);
            }
            if (mine < 4) atomicMin(&jrun, mine);
            __syncthreads();
            const uint32_t e = jrun;
            __syncthreads();
            J += e;
            if (e < 4) break;
        }
        J = min(J, (uint32_t)JMAX_CHUNKS);
        // the shared chunks as keys, and the samples' keys behind them
        uint64_t* jp = w.jpre + (size_t)s * JMAX_CHUNKS;
        for (uint32_t c = threadIdx.x; c < J; c += blockDim.x)
            jp[c] = load_key(w.chars, w.nchars, ref + 8ull * c);
#pragma unroll 8
        for (uint32_t i = threadIdx.x; i < S; i += blockDim.x)
            samp[i] = h_key(w, shnd[i], sg.depth + 8 * J);
        __syncthreads();
    }
    bitonic_sort_block(samp, S);
    if (threadIdx.x == 0) {
        w.jump[s] = 8 * J;
        atomicAdd(w.counters + C_P_BIG, sg.size);
        if (!valid || J) atomicAdd(w.counters + C_P_STALE, sg.size);
        if (J) {
            atomicAdd(w.counters + C_P_TIE, sg.size);
            atomicAdd(w.counters + C_P_JCHUNKS, sg.size * J);
        }
    }
    // splitters: every sample but the first; level-order tree over them
    uint64_t* spl = w.spl + (size_t)s * 1024;
    uint64_t* tree = w.tree + (size_t)s * 1024;
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) spl[j] = samp[j + 1];
    for (uint32_t v = 1 + threadIdx.x; v <= k; v += blockDim.x) {
        const uint32_t h = 31 - __clz((int)v);
        const uint32_t p = v - (1u << h);
        const uint32_t r = ((2 * p + 1) << (L - 1 - h)) - 1;  // in-order rank
        tree[v] = samp[r + 1];
    }
    if (threadIdx.x == 0) w.tree_bits[s] = (uint8_t)L;
}

// One block per tile of a big segment: gather keys if stale, classify,
// store bucket ids and the tile histogram, add it into the segment's counts.
// Behind a common-prefix jump a string first compares its chunks with the
// shared ones (all loads of a string in flight at once): an earlier
// difference puts it into the first or last bucket, else its key after the
// prefix goes through the tree (bucket + 1).
// Tiles of finished (all-equal) segments copy ids and LCPs to the output.
__global__ void __launch_bounds__(TILE_THREADS, 1536 / TILE_THREADS) k_classify(Work w, uint32_t nbig)
{
    __shared__ uint64_t tree[1024];
    __shared__ uint64_t jp[JMAX_CHUNKS];   // the shared chunks as keys
    __shared__ uint64_t jpr[JMAX_CHUNKS];  // and as raw windows
    __shared__ uint32_t hist[MAX_BKT];
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
    const uint32_t J = w.jump[s];
    const uint32_t nc = J / 8;
    const uint32_t k = (1u << L) - 1;
    const uint32_t B = seg_buckets(w, s);
    const uint64_t* gtree = w.tree + (size_t)s * 1024;
    for (uint32_t v = threadIdx.x; v <= k; v += TILE_THREADS) tree[v] = gtree[v];
    for (uint32_t c = threadIdx.x; c < nc; c += TILE_THREADS) {
        const uint64_t kc = w.jpre[(size_t)s * JMAX_CHUNKS + c];
        jp[c] = kc;
        jpr[c] = bswap64(kc);  // no NUL inside a shared chunk
    }
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS) hist[b] = 0;
    __syncthreads();
    const bool valid = (sg.meta & META_VALID) && !J;
    uint64_t* keys = w.keys[buf];
    for (uint32_t p = lo + threadIdx.x; p < hi; p += TILE_THREADS) {
        uint64_t key = 0;
        int side = 0;  // -1: below the prefix, +1: above it
        if (valid) {
            key = keys[p];
        } else if (!J) {
            key = h_key(w, hs[p], sg.depth);
            keys[p] = key;
        } else {
            const uint64_t o = h_off(w, hs[p]) + sg.depth;
            constexpr uint32_t NB = 7;  // chunks per batch: a 6-chunk prefix and its key
            for (uint32_t c0 = 0; c0 <= nc && !side; c0 += NB) {
                uint64_t raw[NB];
                load_raw_chunks<NB>(w.chars, w.nchars, o + 8ull * c0, min(NB, nc + 1 - c0), raw);
#pragma unroll
                for (uint32_t q = 0; q < NB; ++q) {
                    const uint32_t c = c0 + q;
                    if (side || c > nc) continue;
                    if (c == nc) {
                        key = finish_key(raw[q]);
                    } else if (raw[q] != jpr[c]) {
                        // equal raw windows hold no NUL (the shared chunk has
                        // none); the first unequal one decides the side
                        const uint64_t kq = finish_key(raw[q]);
                        side = kq < jp[c] ? -1 : 1;
                    }
                }
            }
            keys[p] = key;
        }
        uint32_t b;
        if (side) {
            b = side < 0 ? 0u : B - 1;
        } else {
            uint32_t i = 1;
            uint64_t cand = 0;
            for (uint32_t l = 0; l < L; ++l) {
                const uint64_t tv = tree[i];
                const bool gt = key > tv;
                cand = gt ? cand : tv;
                i = 2 * i + (gt ? 1u : 0u);
            }
            const uint32_t r = i - (1u << L);  // splitters < key
            b = 2 * r + ((r < k && cand == key) ? 1u : 0u) + (J ? 1u : 0u);
        }
        w.bkt[p] = (uint16_t)b;
        atomicAdd(&hist[b], 1u);
    }
    __syncthreads();
    uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    uint32_t* row = w.tcount + (size_t)t * MAX_BKT;
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS) {
        const uint32_t h = hist[b];
        row[b] = h;
        if (h) atomicAdd(bc + b, h);
    }
}

__device__ __forceinline__ bool classified(uint8_t L)
{
    return L != 0;
}

// Bucket starts (exclusive prefix over buckets) and the one-bucket test. For
// a segment of at most CHUNK tiles also every tile's first destination per
// bucket (count_finished over (tile, bucket), hpp:1437-1460); longer
// segments take the chunked scan below.
__global__ void __launch_bounds__(512) k_bstart(Work w)
{
    constexpr uint32_t T = 512;
    __shared__ uint32_t a[MAX_BKT];
    __shared__ uint32_t tmp[32];
    __shared__ int one;
    const int s = blockIdx.x;
    const Seg sg = w.list[L_BIG][w.cur][s];
    const uint8_t L = w.tree_bits[s];
    if (!classified(L)) return;
    const uint32_t B = seg_buckets(w, s);
    const uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    if (threadIdx.x == 0) one = 0;
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < B; b += T) {
        const uint32_t c = bc[b];
        a[b] = c;
        if (c == sg.size) one = 1;
    }
    __syncthreads();
    block_scan_array<T>(a, (int)B, tmp);
    uint32_t* bs = w.bstart + (size_t)s * MAX_BKT;
    for (uint32_t b = threadIdx.x; b < B; b += T) bs[b] = a[b];
    if (threadIdx.x == 0) {
        w.bflags[s] = (uint8_t)one;
        if (!one) atomicAdd(w.counters + C_P_SCATTER, sg.size);
    }
    const uint32_t t0 = w.tile_start[s], nt = w.tile_start[s + 1] - t0;
    if (one || nt > (uint32_t)CHUNK) return;
    for (uint32_t b = threadIdx.x; b < B; b += T) {
        uint32_t run = sg.begin + a[b];
        uint32_t* col = w.tcount + (size_t)t0 * MAX_BKT + b;
        uint32_t v[CHUNK];  // all of the column's loads in flight
#pragma unroll
        for (uint32_t j = 0; j < (uint32_t)CHUNK; ++j) v[j] = j < nt ? col[(size_t)j * MAX_BKT] : 0u;
        hold_loaded(v);
#pragma unroll
        for (uint32_t j = 0; j < (uint32_t)CHUNK; ++j) {
            if (j < nt) col[(size_t)j * MAX_BKT] = run;
            run += v[j];
        }
    }
}

// Segments of more than CHUNK tiles (rare: over CHUNK * TILE strings) scan
// their (tile, bucket) counts in chunks of CHUNK tiles: chunk sums, their
// scan per bucket, then the tiles inside each chunk. The kernels loop over
// chunks / segments with a fixed grid and skip the short segments.
__device__ __forceinline__ bool multi_chunk(const Work& w, int s)
{
    return classified(w.tree_bits[s]) && !w.bflags[s] &&
           w.chunk_start[s + 1] - w.chunk_start[s] > 1;
}

// Per chunk of a multi-chunk segment and slice of 256 buckets (blockIdx.y):
// bucket sums over the chunk's tiles.
__global__ void __launch_bounds__(256) k_chunk_sum(Work w, uint32_t nbig)
{
    const uint32_t nchunk = w.chunk_start[nbig];
    for (uint32_t c = blockIdx.x; c < nchunk; c += gridDim.x) {
        const int s = find_tile_seg(w.chunk_start, nbig, c);
        if (!multi_chunk(w, s)) continue;
        const uint32_t B = seg_buckets(w, s);
        const uint32_t b = blockIdx.y * 256 + threadIdx.x;
        if (b >= B) continue;
        const uint32_t t0 = w.tile_start[s] + (c - w.chunk_start[s]) * CHUNK;
        const uint32_t nt = min(t0 + CHUNK, w.tile_start[s + 1]) - t0;
        const uint32_t* col = w.tcount + (size_t)t0 * MAX_BKT + b;
        uint32_t sum = 0;
#pragma unroll
        for (uint32_t j = 0; j < (uint32_t)CHUNK; ++j)
            if (j < nt) sum += col[(size_t)j * MAX_BKT];
        w.ccount[(size_t)c * MAX_BKT + b] = sum;
    }
}

// Per multi-chunk segment and slice of 128 buckets: exclusive scan of the
// chunk sums over the segment's chunks, offset by the segment begin and
// bucket start.
__global__ void __launch_bounds__(128) k_chunk_scan(Work w, uint32_t nbig)
{
    for (uint32_t s = blockIdx.x; s < nbig; s += gridDim.x) {
        if (!multi_chunk(w, s)) continue;
        const uint32_t B = seg_buckets(w, s);
        const uint32_t b = blockIdx.y * 128 + threadIdx.x;
        if (b >= B) continue;
        const uint32_t c0 = w.chunk_start[s], C = w.chunk_start[s + 1] - c0;
        uint32_t run = w.list[L_BIG][w.cur][s].begin + w.bstart[(size_t)s * MAX_BKT + b];
        uint32_t* cc = w.ccount + (size_t)c0 * MAX_BKT + b;
        constexpr uint32_t U = 16;  // loads in flight per thread
        for (uint32_t j = 0; j < C; j += U) {
            uint32_t v[U];
#pragma unroll
            for (uint32_t q = 0; q < U; ++q) v[q] = j + q < C ? cc[(size_t)(j + q) * MAX_BKT] : 0u;
            hold_loaded(v);
#pragma unroll
            for (uint32_t q = 0; q < U; ++q) {
                if (j + q < C) cc[(size_t)(j + q) * MAX_BKT] = run;
                run += v[q];
            }
        }
    }
}

// Per chunk of a multi-chunk segment and slice of 256 buckets: each tile's
// first destination per bucket (the chunk base plus the counts of the
// chunk's earlier tiles), written over the tile counts.
__global__ void __launch_bounds__(256) k_tile_offsets(Work w, uint32_t nbig)
{
    const uint32_t nchunk = w.chunk_start[nbig];
    for (uint32_t c = blockIdx.x; c < nchunk; c += gridDim.x) {
        const int s = find_tile_seg(w.chunk_start, nbig, c);
        if (!multi_chunk(w, s)) continue;
        const uint32_t B = seg_buckets(w, s);
        const uint32_t b = blockIdx.y * 256 + threadIdx.x;
        if (b >= B) continue;
        const uint32_t t0 = w.tile_start[s] + (c - w.chunk_start[s]) * CHUNK;
        const uint32_t nt = min(t0 + CHUNK, w.tile_start[s + 1]) - t0;
        uint32_t* col = w.tcount + (size_t)t0 * MAX_BKT + b;
        uint32_t run = w.ccount[(size_t)c * MAX_BKT + b];
        uint32_t v[CHUNK];
#pragma unroll
        for (uint32_t j = 0; j < (uint32_t)CHUNK; ++j) v[j] = j < nt ? col[(size_t)j * MAX_BKT] : 0u;
        hold_loaded(v);
#pragma unroll
        for (uint32_t j = 0; j < (uint32_t)CHUNK; ++j) {
            if (j < nt) col[(size_t)j * MAX_BKT] = run;
            run += v[j];
        }
    }
}

struct ScatterSmem {
    uint64_t stage[TILE];      // the tile's keys in bucket order, then its handles
    uint16_t sbkt[TILE];       // bucket of each staged slot
    uint32_t lcount[MAX_BKT];  // per bucket: count in the tile, then its first slot,
                               // then global position - slot
    uint32_t tmp[32];
};

// One block per tile: rank every string inside its bucket, stage the tile in
// bucket order in shared memory, write bucket runs contiguously from the
// tile's destinations (k_tile_offsets). Global loads are issued a phase
// ahead of their use: the bucket ids, the destination row and half of the
// keys together; the other half of the keys before the bucket scan; all
// handles before the keys are written out. Each thread's slots are packed
// two to a register while the handles are held.
__global__ void __launch_bounds__(TILE_THREADS, 2) k_scatter(Work w, uint32_t nbig)
{
    constexpr int PER = TILE / TILE_THREADS;
    constexpr int HALF = PER / 2;
    constexpr int NBT = (MAX_BKT + TILE_THREADS - 1) / TILE_THREADS;
    static_assert(TILE <= 0xFFFF, "slots and ranks take 16 bits");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScatterSmem& sm = *reinterpret_cast<ScatterSmem*>(smem_raw);
    const uint32_t t = blockIdx.x;
    const int s = find_tile_seg(w.tile_start, nbig, t);
    const Seg sg = w.list[L_BIG][w.cur][s];
    const uint8_t L = w.tree_bits[s];
    if (!classified(L) || w.bflags[s]) return;
    const uint32_t lo = sg.begin + (t - w.tile_start[s]) * TILE;
    const uint32_t hi = min(lo + TILE, sg.begin + sg.size);
    const uint32_t cnt = hi - lo;
    const uint32_t B = seg_buckets(w, s);
    const int buf = sg.meta & META_BUF;
    const uint64_t* ikeys = w.keys[buf];
    const uint64_t* ihs = w.hnd[buf];
    const uint32_t* dst = w.tcount + (size_t)t * MAX_BKT;
    uint32_t first[NBT];
#pragma unroll
    for (int i = 0; i < NBT; ++i) {
        const uint32_t b = threadIdx.x + i * TILE_THREADS;
        first[i] = b < B ? dst[b] : 0u;
    }
    uint32_t pk[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint32_t p = lo + threadIdx.x + j * TILE_THREADS;
        pk[j] = p < hi ? (uint32_t)__ldg(w.bkt + p) : 0xFFFFFFFFu;
    }
    uint64_t v[PER];
#pragma unroll
    for (int j = 0; j < HALF; ++j) {
        const uint32_t p = lo + threadIdx.x + j * TILE_THREADS;
        v[j] = p < hi ? __ldg(ikeys + p) : 0ull;
    }
    for (uint32_t b = threadIdx.x; b < B; b += TILE_THREADS) sm.lcount[b] = 0;
    __syncthreads();
    // rank of every string inside its bucket in this tile: (bucket << 16) | rank
#pragma unroll
    for (int j = 0; j < PER; ++j)
        if (pk[j] != 0xFFFFFFFFu) pk[j] = (pk[j] << 16) | atomicAdd(&sm.lcount[pk[j]], 1u);
#pragma unroll
    for (int j = HALF; j < PER; ++j) {
        const uint32_t p = lo + threadIdx.x + j * TILE_THREADS;
        v[j] = p < hi ? __ldg(ikeys + p) : 0ull;
    }
    __syncthreads();
    block_scan_array<TILE_THREADS>(sm.lcount, (int)B, sm.tmp);  // counts -> first slots
    // stage keys in bucket order; slots packed two to a register
    uint32_t ps[HALF];
#pragma unroll
    for (int j = 0; j < PER; j += 2) {
        uint32_t pair = 0xFFFFFFFFu;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (pk[j + q] == 0xFFFFFFFFu) continue;
            const uint32_t b = pk[j + q] >> 16;
            const uint32_t slot = sm.lcount[b] + (pk[j + q] & 0xFFFFu);
            sm.stage[slot] = v[j + q];
            sm.sbkt[slot] = (uint16_t)b;
            pair = q ? ((pair & 0xFFFFu) | (slot << 16)) : ((pair & 0xFFFF0000u) | slot);
        }
        ps[j / 2] = pair;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NBT; ++i) {
        const uint32_t b = threadIdx.x + i * TILE_THREADS;
        if (b < B) sm.lcount[b] = first[i] - sm.lcount[b];
    }
    // the handles, in flight while the keys go out
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint32_t p = lo + threadIdx.x + j * TILE_THREADS;
        v[j] = p < hi ? __ldg(ihs + p) : 0ull;
    }
    hold_loaded64(v);
    __syncthreads();
    // write bucket runs contiguously: keys, then handles
    uint64_t* okeys = w.keys[buf ^ 1];
    for (uint32_t slot = threadIdx.x; slot < cnt; slot += TILE_THREADS) {
        const uint32_t dest = slot + sm.lcount[sm.sbkt[slot]];
        if (dest - sg.begin >= sg.size) {  // counts and destinations disagree
            set_error(w.counters + C_ERR, ERR_INTERNAL);
            continue;
        }
        okeys[dest] = sm.stage[slot];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint32_t slot = (ps[j / 2] >> (16 * (j & 1))) & 0xFFFFu;
        if (slot != 0xFFFFu) sm.stage[slot] = v[j];
    }
    __syncthreads();
    uint64_t* ohs = w.hnd[buf ^ 1];
    for (uint32_t slot = threadIdx.x; slot < cnt; slot += TILE_THREADS) {
        const uint32_t dest = slot + sm.lcount[sm.sbkt[slot]];
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
    if (cls == L_BIG) {
        const uint32_t tiles = (c.size + TILE - 1) / TILE;
        atomicAdd(w.counters + C_PAR * nxt + C_NTILES, tiles);
        if (tiles > (uint32_t)CHUNK) atomicAdd(w.counters + C_MULTI + nxt, 1u);
    } else {
        atomicAdd(w.counters + C_PAR * nxt + C_NSTR + cls, c.size);
    }
}

// push_seg for a whole warp: lanes with push set append c. One reservation
// per class and warp, and the class's tile or string count added once (a
// launch that pushes many segments would otherwise serialise on these few
// counters).
__device__ __forceinline__ void push_seg_warp(Work& w, int nxt, bool push, const Seg& c)
{
    const uint32_t lane = threadIdx.x & 31;
    int cls = -1;
    if (push)
        cls = c.size > SMALL_MAX ? L_BIG : c.size > 256 ? L_SMALLB : c.size > WARP_GROUP_MAX ? L_SMALLA : L_TINY;
#pragma unroll
    for (int k = 0; k < L_NCLASS; ++k) {
        const uint32_t m = __ballot_sync(0xffffffffu, cls == k);
        if (!m) continue;
        const int leader = __ffs(m) - 1;
        const uint32_t tiles = cls == k && k == L_BIG ? (c.size + TILE - 1) / TILE : 0u;
        const uint32_t amount = __reduce_add_sync(0xffffffffu, cls != k ? 0u : k == L_BIG ? tiles : c.size);
        const uint32_t multi = __reduce_add_sync(0xffffffffu, tiles > (uint32_t)CHUNK ? 1u : 0u);
        uint32_t base = 0;
        if (lane == (uint32_t)leader) {
            base = atomicAdd(w.counters + C_PAR * nxt + k, (uint32_t)__popc(m));
            if (k == L_BIG) {
                atomicAdd(w.counters + C_PAR * nxt + C_NTILES, amount);
                if (multi) atomicAdd(w.counters + C_MULTI + nxt, multi);
            } else {
                atomicAdd(w.counters + C_PAR * nxt + C_NSTR + k, amount);
            }
        }
        base = __shfl_sync(0xffffffffu, base, leader);
        if (cls == k) {
            const uint32_t at = base + __popc(m & ((1u << lane) - 1u));
            if (at >= w.cap[k]) set_error(w.counters + C_ERR, ERR_OVERFLOW);
            else w.list[k][nxt][at] = c;
        }
    }
}

// Children of each bucket, after the scatter has placed them (hpp:1492-1584):
// '<' buckets keep their depth and keys, '=' buckets go 8 chars deeper or
// are finished when their splitter ends the string. Behind a common-prefix
// jump the tree buckets sit at depth + jump, and the two prefix buckets stay
// at the segment depth without keys.
__global__ void __launch_bounds__(1024) k_children(Work w)
{
    const int s = blockIdx.x;
    const Seg sg = w.list[L_BIG][w.cur][s];
    const uint8_t L = w.tree_bits[s];
    const int buf = sg.meta & META_BUF;
    const int nxt = w.cur ^ 1;
    if (!classified(L)) return;
    // block-aggregated appends, blockDim.x (>= 128) buckets per round: slots
    // in shared memory first, then one global reservation per list
    __shared__ uint32_t lcnt[L_NCLASS], gbase[L_NCLASS], lstr[L_NCLASS];
    __shared__ uint32_t ltiles, lmulti, lbnd, bbase;
    const uint32_t J = w.jump[s];
    const uint32_t B = seg_buckets(w, s);
    const uint32_t dj = sg.depth + J;  // depth of the tree buckets
    const int nbuf = w.bflags[s] ? buf : buf ^ 1;
    const uint32_t* bc = w.bcount + (size_t)s * MAX_BKT;
    const uint32_t* bs = w.bstart + (size_t)s * MAX_BKT;
    const uint64_t* spl = w.spl + (size_t)s * 1024;
    const uint64_t* hs = w.hnd[nbuf];
    for (uint32_t base = 0; base < B; base += blockDim.x) {
        if (threadIdx.x < L_NCLASS) { lcnt[threadIdx.x] = 0; lstr[threadIdx.x] = 0; }
        if (threadIdx.x == 0) { ltiles = 0; lmulti = 0; lbnd = 0; }
        __syncthreads();
        const uint32_t b = base + threadIdx.x;
        Seg child{};
        int cls = -1;
        uint32_t slot = 0, bslot = 0xFFFFFFFFu, bdep = 0;
        const uint32_t c = b < B ? bc[b] : 0u;
        if (c) {
            const uint32_t P = sg.begin + bs[b];
            const bool edge = J && (b == 0 || b == B - 1);  // a prefix bucket
            if (P > sg.begin && w.lcp) {
                bslot = atomicAdd(&lbnd, 1u);
                // the string before P is in a prefix bucket, or this one is:
                // the two strings are only known to share the segment depth
                bdep = (J && (b == B - 1 || bs[b] == bc[0])) ? sg.depth : dj;
            }
            if (c == 1) {
                w.perm[P] = h_id(w, hs[P]);
            } else {
                const uint32_t tb = J ? b - 1 : b;  // tree bucket
                bool inline_done = false;
                if (edge) {
                    child = Seg{P, c, sg.depth, (uint32_t)nbuf};
                } else if (tb & 1) {
                    const uint64_t key = spl[tb >> 1];
                    if (key_terminated(key)) {
                        const uint32_t v = dj + lcp_key_depth(key);
                        if (c <= FINAL_INLINE) {
                            for (uint32_t q = 0; q < c; ++q) {
                                w.perm[P + q] = h_id(w, hs[P + q]);
                                if (w.lcp && q) w.lcp[P + q] = v;
                            }
                            inline_done = true;
                        } else {
                            child = Seg{P, c, v, (uint32_t)nbuf | META_FINAL};
                        }
                    } else if (w.suffix && c <= DBL_MAX) {
                        // a suffix set: the group is sorted by rank doubling
                        // after the passes
                        const uint32_t at = atomicAdd(w.counters + C_DBL, 1u);
                        if (at < w.dbl_cap) w.dbl[at] = Seg{P, c, dj + 8, (uint32_t)nbuf};
                        else set_error(w.counters + C_ERR, ERR_OVERFLOW);
                        inline_done = true;
                    } else {
                        child = Seg{P, c, dj + 8, (uint32_t)nbuf};
                    }
                } else {
                    child = Seg{P, c, dj, (uint32_t)nbuf | META_VALID};
                }
                if (!inline_done) {
                    if (c > SMALL_MAX) cls = L_BIG;
                    else if (c > 256) cls = L_SMALLB;
                    else if (c > WARP_GROUP_MAX) cls = L_SMALLA;
                    else cls = L_TINY;
                    slot = atomicAdd(&lcnt[cls], 1u);
                    if (cls == L_BIG) {
                        const uint32_t tiles = (c + TILE - 1) / TILE;
                        atomicAdd(&ltiles, tiles);
                        if (tiles > (uint32_t)CHUNK) atomicAdd(&lmulti, 1u);
                    } else {
                        atomicAdd(&lstr[cls], c);
                    }
                }
            }
        }
        __syncthreads();
        if (threadIdx.x < L_NCLASS && lcnt[threadIdx.x])
            gbase[threadIdx.x] = atomicAdd(w.counters + C_PAR * nxt + threadIdx.x, lcnt[threadIdx.x]);
        if (threadIdx.x == 32 && ltiles) atomicAdd(w.counters + C_PAR * nxt + C_NTILES, ltiles);
        if (threadIdx.x == 33 && lmulti) atomicAdd(w.counters + C_MULTI + nxt, lmulti);
        if (threadIdx.x >= 64 + 1 && threadIdx.x < 64 + L_NCLASS && lstr[threadIdx.x - 64])
            atomicAdd(w.counters + C_PAR * nxt + C_NSTR + (threadIdx.x - 64), lstr[threadIdx.x - 64]);
        if (threadIdx.x == 96 && lbnd) bbase = atomicAdd(w.counters + C_NBND, lbnd);
        __syncthreads();
        if (bslot != 0xFFFFFFFFu) {
            const uint32_t at = bbase + bslot;
            if (at < w.bnd_cap) w.bnd[at] = make_uint2(sg.begin + bs[b], bdep);
            else set_error(w.counters + C_ERR, ERR_OVERFLOW);
        }
        if (cls >= 0) {
            const uint32_t at = gbase[cls] + slot;
            if (at < w.cap[cls]) w.list[cls][nxt][at] = child;
            else set_error(w.counters + C_ERR, ERR_OVERFLOW);
        }
        __syncthreads();
    }
}

// LCP at each split boundary (sample_sort_lcp, hpp:311-396): the two strings
// share at least `depth` chars and lie in different buckets; compare 8 chars
// at a time from there (one step unless a common-prefix jump lies between).
__global__ void k_boundary_lcp(Work w)
{
    const uint32_t nb = min(w.counters[C_NBND], w.bnd_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
        const uint2 e = w.bnd[i];
        const uint32_t P = e.x;
        uint32_t d = e.y;
        const uint32_t ia = w.perm[P - 1], ib = w.perm[P];
        uint64_t ka, kb;
        while (true) {
            ka = gather_key(w.chars, w.nchars, w.offs, ia, d);
            kb = gather_key(w.chars, w.nchars, w.offs, ib, d);
            if (ka != kb || key_terminated(ka)) break;
            d += 8;
        }
        w.lcp[P] = d + (ka != kb ? lcp_key_type(ka, kb) : lcp_key_depth(ka));
    }
}

}  // namespace pssgpu
