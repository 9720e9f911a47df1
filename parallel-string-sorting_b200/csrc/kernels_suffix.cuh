// kernels_suffix.cuh -- the suffix-sorting specialisation: prefix doubling
// on ranks for inputs that are all suffixes of one text.
//
// The reference sorts suffixes as strings (UCharSuffixSet,
// src/tools/stringset.hpp:732-804: string i is text + i up to the text's
// end), so a group of suffixes sharing a long repeat is walked 8 chars per
// step. Suffixes allow more: two suffixes x, y that share d chars compare as
// the suffixes x + d and y + d do. So once the string sort has placed every
// suffix either at its final position or in an unsorted group whose members
// share d chars (the group's depth), each group sorts by the rank of suffix
// x + d -- a final position, or the start of that suffix's own group. Ties
// form subgroups whose depth is d plus the depth of the tied group, so the
// depth at least doubles per round (prefix doubling on the ranks the string
// passes produced): a group of 10 KB repeats needs about 11 rounds instead
// of 1,280 chunk steps.
//
// Arrays (positions p, suffixes x, both in [0, n)): perm[p] = the suffix at p;
// isa[x] = its rank (final position, or its group's start); gd[par][s] = depth
// of the group starting at s (read from one parity, written to the other, so
// a round reads a consistent snapshot); key[p] = the rank used this round;
// lb[p] (LCP output only) = the depth at which positions p - 1 and p were
// separated, a lower bound of their LCP, or ~0 when p did not lie inside a
// doubled group.
#pragma once

#include "kernels_small.cuh"

namespace pssgpu {

constexpr uint32_t DBL_NONE = 0xFFFFFFFFu;  // lb: no doubling bound
// largest group of the smaller block sort (256 threads, 12 KB of shared
// memory); groups just above 512, common when a text's 8-char prefixes each
// head about 512 suffixes, sort here rather than in 512-thread blocks of
// 48 KB
constexpr uint32_t DBL_MID = 1024;

// Round 0 sorts every handed-over group by the DBL_ROUND0_CHARS chars that
// follow its shared prefix, read from the text (a text of this size stays in
// L2), instead of by ranks: no rank has to be written before it and none
// read in it, and its ties form groups DBL_ROUND0_CHARS deeper. The key and
// a member index of up to 16 bits fill one 64-bit sort word.
constexpr uint32_t DBL_ROUND0_CHARS = 6;

// Group lists of a round, by size class: 0 at most 32 members (one warp
// each), 1 at most DBL_MID (a block of 256 threads), 2 at most DBL_MAX (a
// block of 512 threads); double-buffered by round parity.
struct DblArrays {
    const uint8_t* text;  // the text the suffixes belong to (round 0 reads it)
    uint64_t ntext;
    uint32_t* isa;
    uint32_t* gd[2];
    uint32_t* key;
    uint32_t* lb;   // null without LCP output
    Seg* list[3][2];
    uint32_t cap[3];
};

__host__ __device__ constexpr int dbl_class(uint32_t size)
{
    return size <= (uint32_t)WARP_GROUP_MAX ? 0 : size <= DBL_MID ? 1 : 2;
}

// The input is a suffix set when offs[i] == i for all i and no NUL lies
// before the last char (n == nchars is checked by the host): any other
// input sets *flag.
__global__ void k_suffix_check(const uint8_t* __restrict__ chars, const uint64_t* __restrict__ offs,
                               uint64_t n, uint32_t* flag)
{
    bool bad = false;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        if (__ldg(offs + i) != i) bad = true;
        if (i + 1 < n && __ldg(chars + i) == 0) bad = true;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

// Members of the groups the string passes handed over: their ids into perm
// (the handles sit in the group's ping-pong buffer) and a mark in `taken`;
// the group's depth into gd[0]. Their ranks come from round 0, which sorts
// by text chars. The groups are sorted into the round lists of parity 0
// (dbl_push, below) and their members counted.
__global__ void k_dbl_init(Work w, const Seg* __restrict__ list, uint32_t count, DblArrays a,
                           uint8_t* __restrict__ taken, uint32_t* counters,
                           unsigned long long* members);

// Every other position (not in a handed-over group) is final: its suffix's
// rank is the position.
__global__ void k_dbl_isa(const uint32_t* __restrict__ perm, uint32_t n,
                          const uint8_t* __restrict__ taken, uint32_t* __restrict__ isa)
{
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        if (!taken[p]) isa[perm[p]] = p;
}

__device__ __forceinline__ void dbl_push(DblArrays& a, uint32_t* counters, int par, Seg s)
{
    const int cls = dbl_class(s.size);
    const uint32_t at = atomicAdd(counters + C_DBL_CNT + 3 * par + cls, 1u);
    if (at < a.cap[cls]) a.list[cls][par][at] = s;
    else set_error(counters + C_ERR, ERR_OVERFLOW);
}

// The list appends of a block are staged in shared memory, DBL_INIT_STAGE
// per class, and reserved with one global atomic per full stage (a global
// atomic per group serialises on the three list counters).
constexpr uint32_t DBL_INIT_STAGE = 64;
__global__ void k_dbl_init(Work w, const Seg* __restrict__ list, uint32_t count, DblArrays a,
                           uint8_t* __restrict__ taken, uint32_t* counters,
                           unsigned long long* members)
{
    __shared__ Seg stage[3][DBL_INIT_STAGE];
    __shared__ uint32_t staged[3];
    if (threadIdx.x == 0) staged[0] = staged[1] = staged[2] = 0;  // thread 0 alone uses them
    auto flush = [&](int c) {  // thread 0
        const uint32_t m = staged[c];
        if (!m) return;
        const uint32_t base = atomicAdd(counters + C_DBL_CNT + c, m);  // parity 0
        for (uint32_t q = 0; q < m; ++q) {
            if (base + q < a.cap[c]) a.list[c][0][base + q] = stage[c][q];
            else set_error(counters + C_ERR, ERR_OVERFLOW);
        }
        staged[c] = 0;
    };
    for (uint32_t g = blockIdx.x; g < count; g += gridDim.x) {
        const Seg s = list[g];
        const uint64_t* hs = w.hnd[s.meta & META_BUF];
        for (uint32_t q = threadIdx.x; q < s.size; q += blockDim.x) {
            w.perm[s.begin + q] = h_id(w, hs[s.begin + q]);
            taken[s.begin + q] = 1;
        }
        if (threadIdx.x == 0) {
            a.gd[0][s.begin] = s.depth;
            atomicAdd(members, (unsigned long long)s.size);
            const int c = dbl_class(s.size);
            stage[c][staged[c]++] = Seg{s.begin, s.size, s.depth, 0u};
            if (staged[c] == DBL_INIT_STAGE) flush(c);
        }
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c) flush(c);
}

// Warp-aggregated append to the round lists: every lane of the warp calls;
// lanes with push set append s (one global reservation per class and warp).
__device__ __forceinline__ void dbl_push_warp(DblArrays& a, uint32_t* counters, int par, bool push,
                                              const Seg& s)
{
    const uint32_t lane = threadIdx.x & 31;
    const int cls = push ? dbl_class(s.size) : 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const uint32_t m = __ballot_sync(0xffffffffu, cls == c);
        if (!m) continue;
        const int leader = __ffs(m) - 1;
        uint32_t base = 0;
        if (lane == (uint32_t)leader) base = atomicAdd(counters + C_DBL_CNT + 3 * par + c, (uint32_t)__popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (cls == c) {
            const uint32_t at = base + __popc(m & ((1u << lane) - 1u));
            if (at < a.cap[c]) a.list[c][par][at] = s;
            else set_error(counters + C_ERR, ERR_OVERFLOW);
        }
    }
}

// Round step 1: every member's key, the rank of the suffix `depth` chars
// further (members share depth chars, none of them NUL, so x + depth < n).
// k_dbl_keys_small: one thread per group of at most 32; k_dbl_keys: one warp
// per larger group.
__global__ void k_dbl_keys_small(const Seg* __restrict__ list, uint32_t count,
                                 const uint32_t* __restrict__ perm, DblArrays a,
                                 unsigned long long* members)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const Seg s = g < count ? list[g] : Seg{0u, 0u, 0u, 0u};
    const uint32_t m = __reduce_add_sync(0xFFFFFFFFu, s.size);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(members, (unsigned long long)m);
    // four members at a time: their ids, then their ranks, all in flight
    // together (stores to key would otherwise order every next load)
    for (uint32_t q = 0; q < s.size; q += 4) {
        uint32_t x[4], r[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) x[j] = q + j < s.size ? __ldg(perm + s.begin + q + j) : 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j) r[j] = q + j < s.size ? a.isa[x[j] + s.depth] : 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (q + j < s.size) a.key[s.begin + q + j] = r[j];
    }
}

__global__ void k_dbl_keys(const Seg* __restrict__ list, uint32_t count,
                           const uint32_t* __restrict__ perm, DblArrays a,
                           unsigned long long* members)
{
    const uint32_t g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (g >= count) return;
    const Seg s = list[g];
    if ((threadIdx.x & 31) == 0) atomicAdd(members, (unsigned long long)s.size);
    for (uint32_t q = threadIdx.x & 31; q < s.size; q += 32)
        a.key[s.begin + q] = a.isa[perm[s.begin + q] + s.depth];
}

// The run of equal keys K that starts at offset i0 of group s and has len
// members: the LCP bound at its start, and for len >= 2 the subgroup (with
// its depth recorded for the next round) into *out. The subgroup lies
// `step` chars deeper (round 0's text chars), or, with step 0, as deep as
// the group ranked K. Returns whether *out is to be appended.
__device__ __forceinline__ bool dbl_run(DblArrays& a, int par, const Seg& s, uint32_t i0,
                                        uint32_t len, uint32_t K, Seg* out, uint32_t step)
{
    const uint32_t p = s.begin + i0;
    if (a.lb && i0 > 0) a.lb[p] = s.depth;  // separated from p - 1 at this depth
    if (len < 2) return false;
    const uint32_t nd = s.depth + (step ? step : a.gd[par][K]);
    a.gd[par ^ 1][p] = nd;
    *out = Seg{p, len, nd, 0u};
    return true;
}

// Round 0's key of suffix x in a group of depth d: the DBL_ROUND0_CHARS chars
// at x + d, big-endian (load_key's NUL convention).
__device__ __forceinline__ uint64_t dbl_round0_key(const DblArrays& a, uint32_t x, uint32_t d)
{
    return load_key(a.text, a.ntext, (uint64_t)x + d) >> (64 - 8 * DBL_ROUND0_CHARS);
}

// Round step 2 for groups of at most 32 members: each warp takes
// DBL_PER_WARP consecutive list entries and packs them into windows of 32
// lanes; a window sorts by (group, key, lane), writes perm and the new ranks,
// and splits every group into runs of equal keys.
constexpr uint32_t DBL_PER_WARP = 16;
__global__ void k_dbl_sort_small(const Seg* __restrict__ list, uint32_t count,
                                 uint32_t* __restrict__ perm, DblArrays a, uint32_t* counters, int par,
                                 int round0)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t g0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * DBL_PER_WARP;
    if (g0 >= count) return;  // whole warp
    const uint32_t ng = min(DBL_PER_WARP, count - g0);
    warp_seg_windows(list + g0, ng, [&](const Seg& s, uint32_t gq, uint32_t gs, bool real) {
        const uint32_t mem = real ? lane - gs : 0u;
        const uint32_t x = real ? perm[s.begin + mem] : 0u;
        const uint64_t key = !real ? 0ull : round0 ? dbl_round0_key(a, x, s.depth) : a.key[s.begin + mem];
        uint64_t t = real ? ((uint64_t)gq << 58) | (key << 5) | lane : ~0ull;
#pragma unroll
        for (uint32_t kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
            for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
                const uint64_t o = __shfl_xor_sync(0xffffffffu, t, j);
                const bool lower = (lane & j) == 0, asc = (lane & kk) == 0;
                if ((lower == asc) ? (o < t) : (o > t)) t = o;
            }
        }
        // groups keep their lane ranges: sorted by group first
        const uint64_t K = (t >> 5) & ((1ull << 53) - 1);  // the key (group bits dropped)
        const uint32_t mx = __shfl_sync(0xffffffffu, x, (uint32_t)t & 31u);
        const uint64_t pk = __shfl_up_sync(0xffffffffu, K, 1);
        const bool start = real && (lane == gs || pk != K);
        const uint32_t S = __ballot_sync(0xffffffffu, start);
        const uint32_t rs = 31u - __clz(S & (0xFFFFFFFFu >> (31 - lane)));
        const uint32_t above = lane == 31 ? 0u : (S & (0xFFFFFFFFu << (lane + 1)));
        const uint32_t ge = gs + (real ? s.size : 0u);
        const uint32_t re = above ? min((uint32_t)(__ffs(above) - 1), ge) : ge;
        bool push = false;
        Seg ns{};
        if (real) {
            // unchanged values are not written back: a member that kept its
            // place keeps its perm entry, and after round 0 (which writes
            // every rank) a run at its group's start keeps the group's rank
            if (mx != x) perm[s.begin + mem] = mx;
            if (round0 || rs != gs) a.isa[mx] = s.begin + (rs - gs);  // final position for a single member
            if (start)
                push = dbl_run(a, par, s, rs - gs, re - rs, (uint32_t)K, &ns, round0 ? DBL_ROUND0_CHARS : 0u);
        }
        dbl_push_warp(a, counters, par ^ 1, push, ns);
    });
}

// Round step 2 for groups of 33..MAXM members, one block each: a bitonic
// sort of (key << 32 | member index) in shared memory (dynamic: MAXM keys,
// then MAXM member ids), padded to a power of two with keys that the network
// never moves (bitonic_sort_block_padded).
template <uint32_t MAXM>
__global__ void __launch_bounds__(MAXM <= DBL_MID ? 256 : 512) k_dbl_sort_block(
    const Seg* __restrict__ list, uint32_t* __restrict__ perm, DblArrays a, uint32_t* counters,
    int par, int round0)
{
    static_assert(MAXM <= (1u << (64 - 8 * DBL_ROUND0_CHARS)), "member index beside round 0's key");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* sk = reinterpret_cast<uint64_t*>(smem_raw);
    uint32_t* sx = reinterpret_cast<uint32_t*>(smem_raw + 8 * MAXM);
    const Seg s = list[blockIdx.x];
    const uint32_t m = s.size;
    uint32_t S = 64;
    while (S < m) S <<= 1;
    for (uint32_t q = threadIdx.x; q < S; q += blockDim.x) {
        if (q < m) {
            const uint32_t x = perm[s.begin + q];
            sx[q] = x;
            sk[q] = round0 ? (dbl_round0_key(a, x, s.depth) << (64 - 8 * DBL_ROUND0_CHARS)) | q
                           : ((uint64_t)a.key[s.begin + q] << 32) | q;
        } else {
            sk[q] = ~0ull;
        }
    }
    __syncthreads();
    bitonic_sort_block_padded(sk, S, m);
    // warp-uniform trip counts, so that appends aggregate per warp
    for (uint32_t i0 = threadIdx.x & ~31u; i0 < m; i0 += blockDim.x) {
        const uint32_t i = i0 + (threadIdx.x & 31);
        bool push = false;
        Seg ns{};
        if (i < m) {
            const uint32_t ksh = round0 ? 64 - 8 * DBL_ROUND0_CHARS : 32;
            const uint64_t K = sk[i] >> ksh;
            const uint32_t src = (uint32_t)sk[i] & (MAXM - 1);
            if (src != i) perm[s.begin + i] = sx[src];  // unchanged entries are not rewritten
            if (i == 0 || (sk[i - 1] >> ksh) != K) {
                // a run starts here: its length, then every member's rank
                // (after round 0 a run at the group's start keeps its rank)
                uint32_t e = i + 1;
                while (e < m && (sk[e] >> ksh) == K) ++e;
                if (round0 || i)
                    for (uint32_t q = i; q < e; ++q) a.isa[sx[(uint32_t)sk[q] & (MAXM - 1)]] = s.begin + i;
                push = dbl_run(a, par, s, i, e - i, (uint32_t)K, &ns, round0 ? DBL_ROUND0_CHARS : 0u);
            }
        }
        dbl_push_warp(a, counters, par ^ 1, push, ns);
    }
}

// LCPs at the positions the doubling separated (lb[p] set), in text order
// so that the LCP of suffix x with its predecessor, minus one, bounds that of
// suffix x + 1 (the Phi-array argument of Kasai et al.): one thread per
// chunk of DBL_LCP_CHUNK suffixes, compares 8 chars a step from the bound.
constexpr uint32_t DBL_LCP_CHUNK = 32;
__global__ void k_dbl_lcp(const uint8_t* __restrict__ chars, uint64_t nchars,
                          const uint32_t* __restrict__ perm, const uint32_t* __restrict__ isa,
                          const uint32_t* __restrict__ lb, uint32_t* __restrict__ lcp, uint32_t n)
{
    const uint64_t nchunk = ((uint64_t)n + DBL_LCP_CHUNK - 1) / DBL_LCP_CHUNK;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nchunk;
         c += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x0 = (uint32_t)(c * DBL_LCP_CHUNK);
        const uint32_t x1 = (uint32_t)min((uint64_t)x0 + DBL_LCP_CHUNK, (uint64_t)n);
        uint32_t prev = 0;  // LCP of suffix x - 1 with its predecessor, when known
        bool have = false;
        for (uint32_t x = x0; x < x1; ++x) {
            const uint32_t p = isa[x];
            const uint32_t b = p ? lb[p] : DBL_NONE;
            if (b == DBL_NONE) {
                have = false;
                continue;
            }
            const uint32_t y = perm[p - 1];
            uint32_t d = max(b, have && prev ? prev - 1 : 0u);
            uint64_t ka, kb;
            while (true) {
                ka = load_key(chars, nchars, (uint64_t)x + d);
                kb = load_key(chars, nchars, (uint64_t)y + d);
                if (ka != kb || key_terminated(ka)) break;
                d += 8;
            }
            const uint32_t l = d + (ka != kb ? lcp_key_type(ka, kb) : lcp_key_depth(ka));
            lcp[p] = l;
            prev = l;
            have = true;
        }
    }
}

}  // namespace pssgpu
