// pssgpu.cu -- host driver and C ABI of the B200 string sample sort.
//
// The driver replaces pS5's job queue (src/tools/jobqueue.hpp:74-261) and
// Enqueue (src/parallel/bingmann-parallel_sample_sort.hpp:1613-1634) with
// level-synchronous passes: every pass runs one sample-sort step over all
// segments larger than SMALL_MAX strings (kernels_big.cuh) and finishes all
// smaller segments in shared memory (kernels_block.cuh, kernels_small.cuh).
// One device-to-host read of the counters per pass sizes the next grids.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pssgpu.h"
#include "kernels_big.cuh"
#include "kernels_block.cuh"
#include "kernels_wave.cuh"
#include "kernels_suffix.cuh"
#include "prepare.cuh"
#include "merge.cuh"

namespace pssgpu {

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}

#define PSS_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess)                                                      \
            return fail(e_ == cudaErrorMemoryAllocation ? PSSGPU_ENOMEM : PSSGPU_ECUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));       \
    } while (0)

__global__ void k_init(Work w)
{
    if (blockIdx.x == 0 && threadIdx.x == 0 && w.chars[w.nchars - 1] != 0)
        set_error(w.counters + C_ERR, ERR_UNTERMINATED);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < w.n; i += gridDim.x * blockDim.x) {
        w.hnd[0][i] = h_make(w, i, w.offs[i]);
        if (w.offs[i] >= w.nchars) set_error(w.counters + C_ERR, ERR_OFFSET);
    }
}

// Root segments: the whole input, or one per instance of a batch (instance k
// owns positions [inst[k], inst[k+1])). A one-string instance is final at
// once; the batch's ids are global until k_localize.
__global__ void k_roots(Work w, const uint64_t* __restrict__ inst, uint32_t ninst)
{
    if (!inst) {
        if (blockIdx.x == 0 && threadIdx.x == 0) push_seg(w, 0, Seg{0u, w.n, 0u, 0u});
        return;
    }
    // warp-uniform trips, so that the list appends aggregate per warp
    for (uint32_t k0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); k0 < ninst;
         k0 += gridDim.x * blockDim.x) {
        const uint32_t k = k0 + (threadIdx.x & 31);
        uint32_t b = 0, e = 0;
        if (k < ninst) {
            b = (uint32_t)inst[k];
            e = (uint32_t)inst[k + 1];
        }
        if (e - b == 1) w.perm[b] = b;
        push_seg_warp(w, 0, e - b >= 2, Seg{b, e - b, 0u, 0u});
    }
}

// Batch output: ids relative to their instance; the first LCP of every
// instance is 0. One block per chunk of LOC_CHUNK positions (work follows
// the strings, whether a batch holds many small instances or a few large
// ones); a thread finds the instance of its first position by a search and
// then only moves forward, as its positions increase.
constexpr uint32_t LOC_CHUNK = 4096;

// last k in [lo, hi] with inst[k] <= p (inst[lo] <= p)
__device__ __forceinline__ uint32_t last_inst_at_or_below(const uint64_t* inst, uint32_t lo, uint32_t hi,
                                                          uint64_t p)
{
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (inst[mid] <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_localize(uint32_t* __restrict__ perm, uint32_t* __restrict__ lcp,
                           const uint64_t* __restrict__ inst, uint32_t ninst, uint32_t n)
{
    for (uint64_t c0 = (uint64_t)blockIdx.x * LOC_CHUNK; c0 < n; c0 += (uint64_t)gridDim.x * LOC_CHUNK) {
        const uint64_t c1 = min(c0 + LOC_CHUNK, (uint64_t)n);
        uint64_t p = c0 + threadIdx.x;
        if (p >= c1) continue;
        uint32_t k = last_inst_at_or_below(inst, 0, ninst - 1, p);
        for (; p < c1; p += blockDim.x) {
            while (k + 1 < ninst && inst[k + 1] <= p) ++k;
            const uint64_t b = inst[k];
            perm[p] -= (uint32_t)b;
            if (lcp && p == b) lcp[p] = 0;
        }
    }
}

static uint32_t bit_length(uint64_t x) { return x ? 64u - (uint32_t)__builtin_clzll(x) : 0u; }

// Packed handles (id << hbits | offset) when id and offset fit 64 bits.
static void set_handle_format(Work& w, bool force_indirect)
{
    w.hbits = std::max<uint32_t>(1, bit_length(w.nchars ? w.nchars - 1 : 0));
    w.hmask = w.hbits >= 64 ? ~0ull : ((1ull << w.hbits) - 1);
    const uint32_t idbits = bit_length(w.n ? w.n - 1 : 0);
    w.packed = (!force_indirect && w.hbits <= 63 && idbits + w.hbits <= 64) ? 1 : 0;
}

struct Sizes {
    uint64_t n, cap[L_NCLASS], tile_cap, deep_cap;
};

static Sizes sizes_for(uint64_t n)
{
    Sizes s;
    s.n = std::max<uint64_t>(n, 1);
    // a segment of class c has more strings than the class below it holds
    s.cap[L_BIG] = s.n / (SMALL_MAX + 1) + 2;
    s.cap[L_SMALLB] = s.n / 257 + 2;
    s.cap[L_SMALLA] = s.n / (WARP_GROUP_MAX + 1) + 2;
    s.cap[L_TINY] = s.n / 2 + 2;
    s.tile_cap = s.n / TILE + s.cap[L_BIG] + 1;
    // deep groups hold 2..32 strings; a fuller list falls back to walking
    // the group inside the block sorter
    s.deep_cap = s.n / 32 + 64;
    return s;
}

static uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }

static uint64_t workspace_bytes(const Sizes& s)
{
    const uint64_t big = s.cap[L_BIG];
    uint64_t b = 0;
    b += 2 * align256(8 * s.n);                    // string handles
    b += 2 * align256(8 * s.n);                    // keys
    b += align256(2 * s.n);                        // bucket ids
    b += align256(8 * s.n);                        // boundary list
    for (int c = 0; c < L_NCLASS; ++c)
        b += 2 * align256(16 * s.cap[c]);          // segment lists
    b += 2 * align256(4 * (big + 1));              // tile starts, chunk starts
    b += 2 * align256(big);                        // tree bits, one-bucket flags
    b += align256(4 * big);                        // jump lengths
    b += align256(8ull * JMAX_CHUNKS * big);       // jump prefixes
    b += 2 * align256(8ull * 1024 * big);          // trees, splitters
    b += 2 * align256(4ull * MAX_BKT * big);       // bucket counts, starts
    b += 2 * align256(4ull * MAX_BKT * s.tile_cap);  // tile and chunk counts (chunks <= tiles)
    b += 2 * align256(16 * s.deep_cap);            // deep-group lists
    b += align256(4 * C_COUNT);                    // counters
    b += align256(sizeof(WaveState));              // single-launch sort state
    return b;
}

// Kernel classes reported by pssgpu_ctx_kernel_stats.
enum KClass { K_INIT = 0, K_SAMPLE, K_CLASSIFY, K_BSTART, K_SCATTER, K_CHILDREN, K_TINY,
              K_SMALLA, K_SMALLB, K_DEEP, K_BOUNDARY, K_WAVE, K_DBL, K_NCLASS };
static const char* const kclass_name[K_NCLASS] = {
    "init", "sample", "classify", "bstart", "scatter", "children", "tiny",
    "small256", "small1024", "deep", "boundary", "wave", "doubling"};

struct KStat {
    uint32_t launches = 0;
    uint64_t strings = 0;
    uint64_t alg_bytes = 0;
    double ms = 0;
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::mutex mu;
    // workspace
    unsigned char* ws = nullptr;
    uint64_t ws_bytes = 0;
    Sizes cap{};
    Work base{};
    WaveState* wave = nullptr;          // right behind the counters (one memset)
    uint32_t* host_counters = nullptr;  // pinned
    // staging for the host entry points
    unsigned char* io = nullptr;
    uint64_t io_bytes = 0;
    unsigned char* gap_host = nullptr;  // pinned: offset gaps on their way to the device
    uint64_t gap_host_bytes = 0;
    // pinned: the pointer-array entry points' offsets, permutation and LCPs
    unsigned char* ptr_host = nullptr;
    uint64_t ptr_host_bytes = 0;
    // text entry point: offsets, perm and lcp beside the text in io;
    // chunk counts and bases of the line split
    unsigned char* io2 = nullptr;
    uint64_t io2_bytes = 0;
    unsigned char* prep = nullptr;
    uint64_t prep_bytes = 0;
    // merge rounds: ids / LCP ping-pong, source positions, run boundaries
    unsigned char* mbuf = nullptr;
    uint64_t mbuf_bytes = 0;
    pssgpu_stats stats{};
    // profile mode: events around every kernel class, per-class totals
    bool profile = false;
    // PSSGPU_TRACE set in the environment: one line per pass on stderr
    // (segments, tiles, strings per class; kernel-class times in profile mode)
    bool trace = false;
    // carry bare ids and read offsets through offs[] (the path taken when
    // id and offset do not fit one 64-bit handle); settable for testing
    bool indirect_handles = false;
    // inputs that fit one wave of resident blocks sort in one cooperative
    // launch (k_wave); off: always the level-synchronous passes
    bool single_launch = true;
    // polls of a grid-barrier wait in k_wave before it gives up
    uint32_t wait_limit = 1u << 22;
    // outputs one thread merges in a round of pssgpu_merge_lcp_device (0:
    // chosen per merge, merge_piece_for)
    uint32_t merge_piece = 0;
    // suffix sets finish their deep groups by rank doubling (off: the string
    // passes sort them like any strings)
    bool suffix_doubling = true;
    // the list of groups the passes hand to rank doubling (allocated on the
    // first suffix-set sort)
    unsigned char* sfx = nullptr;
    uint64_t sfx_bytes = 0;
    // splitter-tree levels per size class of big segments (0 = default)
    uint8_t tree_bits_by_size[33] = {};
    // device copy of a batch's instance boundaries
    uint64_t* inst_buf = nullptr;
    uint64_t inst_cap = 0;
    cudaEvent_t kev[2 * K_NCLASS] = {};
    KStat kstat[K_NCLASS];
    // the small-segment classes of a pass run on their own streams, beside
    // the big-segment chain on the caller's stream (disjoint ranges of the
    // permutation); fork / join through events
    cudaStream_t side[3] = {};
    cudaEvent_t fork_ev = nullptr;
    cudaEvent_t join_ev[3] = {};
};

// Record the start / end of a kernel class in profile mode.
struct KTimer {
    Ctx* c;
    cudaStream_t st;
    bool used[K_NCLASS] = {};
    float pass_ms[K_NCLASS] = {};  // times of the last collected pass
    void begin(int k)
    {
        if (c->profile) { cudaEventRecord(c->kev[2 * k], st); used[k] = true; }
    }
    void end(int k)
    {
        if (c->profile) cudaEventRecord(c->kev[2 * k + 1], st);
    }
    // after a stream synchronisation
    void collect()
    {
        if (!c->profile) return;
        for (int k = 0; k < K_NCLASS; ++k) {
            pass_ms[k] = 0;
            if (!used[k]) continue;
            float ms = 0;
            cudaEventElapsedTime(&ms, c->kev[2 * k], c->kev[2 * k + 1]);
            c->kstat[k].ms += ms;
            pass_ms[k] = ms;
            used[k] = false;
        }
    }
};

static int ensure_workspace(Ctx* c, uint64_t n)
{
    if (c->ws && n <= c->cap.n) return PSSGPU_OK;
    if (c->ws) {
        cudaFree(c->ws);
        c->ws = nullptr;
    }
    const Sizes s = sizes_for(std::max<uint64_t>(n, 1024));
    const uint64_t bytes = workspace_bytes(s);
    PSS_CUDA(cudaMalloc(&c->ws, bytes));
    c->ws_bytes = bytes;
    c->cap = s;
    unsigned char* p = c->ws;
    auto take = [&](uint64_t b) { unsigned char* r = p; p += align256(b); return r; };
    Work& w = c->base;
    w = Work{};
    for (int i = 0; i < 2; ++i) w.hnd[i] = (uint64_t*)take(8 * s.n);
    for (int i = 0; i < 2; ++i) w.keys[i] = (uint64_t*)take(8 * s.n);
    w.bkt = (uint16_t*)take(2 * s.n);
    w.bnd = (uint2*)take(8 * s.n);
    w.bnd_cap = (uint32_t)s.n;
    for (int c = 0; c < L_NCLASS; ++c) {
        for (int i = 0; i < 2; ++i) w.list[c][i] = (Seg*)take(16 * s.cap[c]);
        w.cap[c] = (uint32_t)s.cap[c];
    }
    const uint64_t big = s.cap[L_BIG];
    w.tile_start = (uint32_t*)take(4 * (big + 1));
    w.chunk_start = (uint32_t*)take(4 * (big + 1));
    w.tree_bits = (uint8_t*)take(big);
    w.bflags = (uint8_t*)take(big);
    w.jump = (uint32_t*)take(4 * big);
    w.jpre = (uint64_t*)take(8ull * JMAX_CHUNKS * big);
    w.tree = (uint64_t*)take(8ull * 1024 * big);
    w.spl = (uint64_t*)take(8ull * 1024 * big);
    w.bcount = (uint32_t*)take(4ull * MAX_BKT * big);
    w.bstart = (uint32_t*)take(4ull * MAX_BKT * big);
    w.tcount = (uint32_t*)take(4ull * MAX_BKT * s.tile_cap);
    w.ccount = (uint32_t*)take(4ull * MAX_BKT * s.tile_cap);
    w.tile_cap = (uint32_t)s.tile_cap;
    for (int i = 0; i < 2; ++i) w.deep[i] = (Seg*)take(16 * s.deep_cap);
    w.deep_cap = (uint32_t)s.deep_cap;
    w.counters = (uint32_t*)take(4 * C_COUNT);
    c->wave = (WaveState*)take(sizeof(WaveState));
    return PSSGPU_OK;
}

// Shared-memory limits of the kernels that need more than 48 KB, set once
// per device (the attribute belongs to the device's context), and the
// number of k_wave blocks one wave holds on that device (0: no
// cooperative launch).
constexpr int MAXDEV = 64;
static uint32_t g_wave_blocks[MAXDEV];

static int setup_kernels()
{
    static bool done[MAXDEV] = {};
    static std::mutex mu;
    int dev = 0;
    PSS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAXDEV) return fail(PSSGPU_ENODEV, "device index out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (done[dev]) return PSSGPU_OK;
    PSS_CUDA(cudaFuncSetAttribute(k_wave, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(WaveSmem)));
    PSS_CUDA(cudaFuncSetAttribute(k_dbl_sort_block<DBL_MAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(12 * DBL_MAX)));
    {
        int coop = 0, sms = 0, per_sm = 0;
        PSS_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        PSS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        PSS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wave, WAVE_THREADS,
                                                               sizeof(WaveSmem)));
        g_wave_blocks[dev] = coop ? (uint32_t)(per_sm * sms) : 0u;
    }
    PSS_CUDA(cudaFuncSetAttribute(K_BLOCK_A, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(BlockSmem<SMALL_A>)));
    PSS_CUDA(cudaFuncSetAttribute(K_BLOCK_B, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(BlockSmem<SMALL_MAX>)));
    PSS_CUDA(cudaFuncSetAttribute(k_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(ScatterSmem)));
    done[dev] = true;
    return PSSGPU_OK;
}

static int map_device_error(uint32_t err)
{
    if (err & ERR_UNTERMINATED) return fail(PSSGPU_EINVAL, "arena does not end with NUL");
    if (err & ERR_OFFSET) return fail(PSSGPU_EINVAL, "a string offset lies outside the arena");
    if (err & ERR_TIMEOUT) return fail(PSSGPU_ETIMEOUT, "a bounded device-side wait gave up");
    if (err & ERR_OVERFLOW) return fail(PSSGPU_ECUDA, "an internal work list overflowed");
    return fail(PSSGPU_ECUDA, "internal device error");
}

// A device buffer of at least `bytes`, grown (contents dropped) when short.
static int ensure_buf(unsigned char** buf, uint64_t* have, uint64_t bytes)
{
    if (*buf && bytes <= *have) return PSSGPU_OK;
    if (*buf) {
        cudaFree(*buf);
        *buf = nullptr;
        *have = 0;
    }
    PSS_CUDA(cudaMalloc(buf, bytes));
    *have = bytes;
    return PSSGPU_OK;
}

// Rank doubling over the ndbl groups the passes handed over (a suffix set):
// ranks of every suffix, then rounds that sort each group by the rank of its
// members' suffixes `depth` chars further, until every group is split into
// single suffixes; with LCP output, the LCPs at the separated positions.
// Works in the workspace's key and handle arrays, which the passes no longer
// need. Caller holds c->mu; *err receives the device error bits.
static int run_doubling(Ctx* c, Work& w, uint32_t ndbl, cudaStream_t st, pssgpu_stats& stats,
                        uint32_t* err)
{
    const uint32_t n = w.n;
    const uint64_t capn = c->cap.n;
    DblArrays a{};
    a.text = w.chars;
    a.ntext = w.nchars;
    a.isa = reinterpret_cast<uint32_t*>(w.keys[0]);
    a.gd[0] = a.isa + capn;
    a.gd[1] = reinterpret_cast<uint32_t*>(w.keys[1]);
    a.key = a.gd[1] + capn;
    a.lb = w.lcp ? reinterpret_cast<uint32_t*>(w.hnd[0]) : nullptr;
    const int lcls[3] = {L_TINY, L_SMALLA, L_SMALLB};
    for (int k = 0; k < 3; ++k) {
        a.list[k][0] = w.list[lcls[k]][0];
        a.list[k][1] = w.list[lcls[k]][1];
        a.cap[k] = w.cap[lcls[k]];
    }
    uint32_t* hc = c->host_counters;
    const unsigned gblocks = std::min<uint32_t>(ndbl, 148u * 16u);
    // marks of the handed-over positions, in the round-key array (free
    // until the first round)
    uint8_t* taken = reinterpret_cast<uint8_t*>(a.key);
    auto* members = reinterpret_cast<unsigned long long*>(w.counters + C_DBL_MEMB);
    PSS_CUDA(cudaMemsetAsync(w.counters + C_DBL_CNT, 0, 4 * (C_COUNT - C_DBL_CNT), st));
    PSS_CUDA(cudaMemsetAsync(taken, 0, n, st));
    k_dbl_init<<<gblocks, 256, 0, st>>>(w, w.dbl, ndbl, a, taken, w.counters, members);
    if (a.lb) PSS_CUDA(cudaMemsetAsync(a.lb, 0xFF, 4ull * n, st));
    k_dbl_isa<<<1184, 256, 0, st>>>(w.perm, n, taken, a.isa);
    stats.kernel_launches += 2;
    c->kstat[K_DBL].launches += 2;
    c->kstat[K_DBL].strings += n;
    PSS_CUDA(cudaGetLastError());
    PSS_CUDA(cudaMemcpyAsync(hc, w.counters, 4 * C_COUNT, cudaMemcpyDeviceToHost, st));
    PSS_CUDA(cudaStreamSynchronize(st));
    int par = 0;
    // the depth of every group at least doubles per round after the first
    // (n <= 2^32 chars): a loop beyond this many rounds is an internal error
    constexpr int MAX_ROUNDS = 64;
    for (int round = 0; !hc[C_ERR]; ++round) {
        uint32_t cnt[3];
        for (int k = 0; k < 3; ++k) cnt[k] = std::min(hc[C_DBL_CNT + 3 * par + k], a.cap[k]);
        if (!cnt[0] && !cnt[1] && !cnt[2]) break;
        if (round >= MAX_ROUNDS) return fail(PSSGPU_ETIMEOUT, "rank doubling round limit exceeded");
        PSS_CUDA(cudaMemsetAsync(w.counters + C_DBL_CNT + 3 * (par ^ 1), 0, 12, st));
        // round 0 sorts by text chars (dbl_round0_key); later rounds by the
        // ranks of one snapshot, read first
        const int round0 = round == 0;
        if (!round0) {
            if (cnt[0])
                k_dbl_keys_small<<<(cnt[0] + 255) / 256, 256, 0, st>>>(a.list[0][par], cnt[0], w.perm, a,
                                                                       members);
            for (int k = 1; k < 3; ++k)
                if (cnt[k])
                    k_dbl_keys<<<(cnt[k] + 7) / 8, 256, 0, st>>>(a.list[k][par], cnt[k], w.perm, a, members);
        }
        if (cnt[0]) {
            constexpr uint32_t per_block = 8 * DBL_PER_WARP;  // 8 warps
            k_dbl_sort_small<<<(cnt[0] + per_block - 1) / per_block, 256, 0, st>>>(
                a.list[0][par], cnt[0], w.perm, a, w.counters, par, round0);
        }
        if (cnt[1])
            k_dbl_sort_block<DBL_MID><<<cnt[1], 256, 12 * DBL_MID, st>>>(a.list[1][par], w.perm, a,
                                                                         w.counters, par, round0);
        if (cnt[2])
            k_dbl_sort_block<DBL_MAX><<<cnt[2], 512, 12 * DBL_MAX, st>>>(a.list[2][par], w.perm, a,
                                                                         w.counters, par, round0);
        const uint32_t per_class = round0 ? 1 : 2;  // (keys and) sort
        const uint32_t launched = (cnt[0] ? per_class : 0) + (cnt[1] ? per_class : 0) + (cnt[2] ? per_class : 0);
        stats.kernel_launches += launched;
        c->kstat[K_DBL].launches += launched;
        PSS_CUDA(cudaGetLastError());
        PSS_CUDA(cudaMemcpyAsync(hc, w.counters, 4 * C_COUNT, cudaMemcpyDeviceToHost, st));
        PSS_CUDA(cudaStreamSynchronize(st));
        if (c->trace)
            std::fprintf(stderr, "pssgpu doubling round %d: groups %u / %u / %u (<=32 / <=%u / <=%u)\n",
                         round, cnt[0], cnt[1], cnt[2], DBL_MID, DBL_MAX);
        par ^= 1;
    }
    *err = hc[C_ERR];
    // algorithmic bytes: every suffix's first rank (its position read, its
    // rank written), then per group member and round its id and the rank
    // `depth` chars further read, its id and new rank written
    const uint64_t memb = (uint64_t)hc[C_DBL_MEMB] | ((uint64_t)hc[C_DBL_MEMB + 1] << 32);
    c->kstat[K_DBL].alg_bytes += 8ull * n + 16ull * memb;
    if (!*err && a.lb) {
        const uint64_t nchunk = ((uint64_t)n + DBL_LCP_CHUNK - 1) / DBL_LCP_CHUNK;
        k_dbl_lcp<<<(unsigned)std::min<uint64_t>((nchunk + 255) / 256, 148ull * 16), 256, 0, st>>>(
            w.chars, w.nchars, w.perm, a.isa, a.lb, w.lcp, n);
        stats.kernel_launches += 1;
        c->kstat[K_DBL].launches += 1;
        PSS_CUDA(cudaGetLastError());
    }
    return PSSGPU_OK;
}

// Sort n strings already resident on the device. Caller holds c->mu.
static int run_sort(Ctx* c, const uint8_t* chars, uint64_t nchars, const uint64_t* offs,
                    uint32_t n, uint32_t* perm, uint32_t* lcp, cudaStream_t st,
                    const uint64_t* d_inst = nullptr, uint32_t ninst = 0)
{
    int rc = ensure_workspace(c, n);
    if (rc) return rc;
    if ((rc = setup_kernels())) return rc;
    Work w = c->base;
    w.chars = chars;
    w.nchars = nchars;
    w.offs = offs;
    w.n = n;
    w.perm = perm;
    w.lcp = lcp;
    set_handle_format(w, c->indirect_handles);
    memcpy(w.tree_bits_by_size, c->tree_bits_by_size, sizeof(w.tree_bits_by_size));
    pssgpu_stats stats{};
    for (int k = 0; k < K_NCLASS; ++k) c->kstat[k] = KStat{};
    KTimer kt{c, st};
    const uint64_t out_bytes = lcp ? 8 : 4;  // perm (+ lcp) per string
    // An input that fits one wave of resident k_wave blocks sorts in one
    // cooperative launch; what it leaves (buckets over WAVE_SORT_MAX strings,
    // deep groups) continues in the passes below from the lists of parity 1.
    const uint32_t wave_cap = g_wave_blocks[c->device];
    const bool wave = !d_inst && c->single_launch && n >= 2 && wave_cap > 0 &&
                      (uint64_t)n <= (uint64_t)wave_cap * WAVE_TILE_MAX;
    int cur = 0;
    const bool suffix_try = !wave && !d_inst && c->suffix_doubling && n >= 2 && (uint64_t)n == nchars;
    PSS_CUDA(cudaEventRecord(c->ev0, st));
    if (wave) {
        // the counters and the wave state's header are adjacent: one memset
        const size_t head = (size_t)((unsigned char*)c->wave - (unsigned char*)w.counters) +
                            offsetof(WaveState, gcount);
        PSS_CUDA(cudaMemsetAsync(w.counters, 0, head, st));
        uint32_t G = std::min<uint32_t>(wave_cap, std::max<uint32_t>(1u, (n + WAVE_WINDOW - 1) / WAVE_WINDOW));
        G = std::max<uint32_t>(G, (n + WAVE_TILE_MAX - 1) / WAVE_TILE_MAX);
        // about 128 strings per bucket slot, at most WAVE_MAX_BITS levels
        const uint32_t lg = bit_length(n) - 1;
        uint32_t L = std::min<uint32_t>(WAVE_MAX_BITS, lg > 8 ? lg - 7 : 1u);
        w.cur = 0;
        WaveState* ws = c->wave;
        uint32_t limit = c->wait_limit;
        int trace = c->trace ? 1 : 0;
        void* args[] = {&w, &ws, &L, &limit, &trace};
        kt.begin(K_WAVE);
        PSS_CUDA(cudaLaunchCooperativeKernel((const void*)k_wave, dim3(G), dim3(WAVE_THREADS), args,
                                             sizeof(WaveSmem), st));
        kt.end(K_WAVE);
        c->kstat[K_WAVE].launches += 1;
        c->kstat[K_WAVE].strings += n;
        // offset 8 + chars 8 read, key + handle 16 written and read back, output
        c->kstat[K_WAVE].alg_bytes += (48 + out_bytes) * n;
        stats.kernel_launches += 1;
        stats.passes += 1;
        cur = 1;
    } else {
        PSS_CUDA(cudaMemsetAsync(w.counters, 0, 4 * C_COUNT, st));
        kt.begin(K_INIT);
        k_init<<<1184, 256, 0, st>>>(w);
        k_roots<<<d_inst ? std::max(1u, std::min((ninst + 255) / 256, 148u * 16u)) : 1u, 256, 0, st>>>(
            w, d_inst, ninst);
        // every string a suffix of one text (n == nchars is necessary)?
        if (suffix_try) k_suffix_check<<<1184, 256, 0, st>>>(chars, offs, n, w.counters + C_SFX);
        kt.end(K_INIT);
        c->kstat[K_INIT].launches += 2;
        c->kstat[K_INIT].strings += n;
        c->kstat[K_INIT].alg_bytes += 12ull * n;  // offset read + id write
        stats.kernel_launches += 2;
    }
    uint32_t* hc = c->host_counters;
    PSS_CUDA(cudaMemcpyAsync(hc, w.counters, 4 * C_COUNT, cudaMemcpyDeviceToHost, st));
    PSS_CUDA(cudaStreamSynchronize(st));
    kt.collect();
    uint32_t cnt[L_NCLASS], nstr[L_NCLASS];
    for (int k = 0; k < L_NCLASS; ++k) {
        cnt[k] = hc[C_PAR * cur + k];
        nstr[k] = k == L_BIG ? 0u : hc[C_PAR * cur + C_NSTR + k];
    }
    uint32_t ntiles = hc[C_PAR * cur + C_NTILES];
    uint32_t nmulti = hc[C_MULTI + cur];
    uint32_t ndeep = hc[C_DEEP + cur];
    uint64_t small_segments = 0;
    uint32_t err = hc[C_ERR];
    if (wave && c->trace) {
        unsigned long long cyc[5] = {};
        if (cudaMemcpy(cyc, c->wave->cycles, sizeof(cyc), cudaMemcpyDeviceToHost) == cudaSuccess)
            std::fprintf(stderr,
                         "pssgpu single launch: %u strings, SM cycles (max over blocks): keys + samples "
                         "%llu, first barrier wait %llu, classify %llu, scatter %llu, bucket sorts %llu\n",
                         n, cyc[0], cyc[1], cyc[2], cyc[3], cyc[4]);
    }
    const bool suffix = suffix_try && !err && hc[C_SFX] == 0;
    if (suffix) {
        // groups of at least 2 strings: at most n / 2 of them
        const uint64_t cap = (uint64_t)n / 2 + 2;
        if ((rc = ensure_buf(&c->sfx, &c->sfx_bytes, 16 * cap))) return rc;
        w.suffix = 1;
        w.dbl = reinterpret_cast<Seg*>(c->sfx);
        w.dbl_cap = (uint32_t)cap;
    }
    auto pending = [&]() {
        return cnt[L_BIG] || cnt[L_TINY] || cnt[L_SMALLA] || cnt[L_SMALLB] || ndeep;
    };
    // Every pass takes each open segment at least 8 chars deeper or splits
    // it; the limit turns a pass structure that stops making progress into
    // an error instead of an endless loop.
    constexpr uint32_t MAX_PASSES = 1u << 20;
    uint32_t npass = 0;
    while (!err && pending()) {
        if (++npass > MAX_PASSES) return fail(PSSGPU_ETIMEOUT, "pass limit exceeded");
        const int nxt = cur ^ 1;
        const uint32_t nbig = cnt[L_BIG];
        w.cur = cur;
        PSS_CUDA(cudaMemsetAsync(w.counters + C_PAR * nxt, 0, 4 * C_PAR, st));
        PSS_CUDA(cudaMemsetAsync(w.counters + C_MULTI + nxt, 0, 4, st));
        PSS_CUDA(cudaMemsetAsync(w.counters + C_DEEP + nxt, 0, 4, st));
        PSS_CUDA(cudaMemsetAsync(w.counters + C_P_FIRST, 0, 4 * (C_P_LAST - C_P_FIRST + 1), st));
        if (nbig && ntiles > c->cap.tile_cap) return fail(PSSGPU_ECUDA, "tile capacity exceeded");
        // small classes: on the side streams (after everything queued on st
        // so far), or serially on st in profile mode so that the per-class
        // events time one class at a time
        const bool fork = !c->profile && (cnt[L_TINY] || cnt[L_SMALLA] || cnt[L_SMALLB] || ndeep);
        if (fork) PSS_CUDA(cudaEventRecord(c->fork_ev, st));
        bool joined[3] = {};
        auto small_stream = [&](int q) -> cudaStream_t {
            if (!fork) return st;
            cudaStreamWaitEvent(c->side[q], c->fork_ev, 0);
            joined[q] = true;
            return c->side[q];
        };
        if (cnt[L_TINY]) {
            cudaStream_t s = small_stream(0);
            kt.begin(K_TINY);
            constexpr uint32_t per_block = TINY_WARPS * TINY_PER_WARP;
            k_tiny<<<(cnt[L_TINY] + per_block - 1) / per_block, 32 * TINY_WARPS, 0, s>>>(
                w, w.list[L_TINY][cur], cnt[L_TINY]);
            kt.end(K_TINY);
            c->kstat[K_TINY].launches += 1;
            stats.kernel_launches += 1;
        }
        if (cnt[L_SMALLA]) {
            cudaStream_t s = small_stream(1);
            kt.begin(K_SMALLA);
            K_BLOCK_A<<<cnt[L_SMALLA], SMALL_A_THREADS, sizeof(BlockSmem<SMALL_A>), s>>>(
                w, w.list[L_SMALLA][cur]);
            kt.end(K_SMALLA);
            c->kstat[K_SMALLA].launches += 1;
            stats.kernel_launches += 1;
        }
        if (ndeep) {
            // groups the previous pass's block sorters handed over; the same
            // stream as the block sorters, which add to the other list
            cudaStream_t s = small_stream(2);
            kt.begin(K_DEEP);
            constexpr uint32_t per_block = TINY_WARPS;
            k_deep<<<(std::min(ndeep, w.deep_cap) + per_block - 1) / per_block, 32 * TINY_WARPS, 0, s>>>(
                w, w.deep[cur], std::min(ndeep, w.deep_cap));
            kt.end(K_DEEP);
            c->kstat[K_DEEP].launches += 1;
            stats.kernel_launches += 1;
        }
        if (cnt[L_SMALLB]) {
            cudaStream_t s = small_stream(2);
            kt.begin(K_SMALLB);
            K_BLOCK_B<<<cnt[L_SMALLB], SMALL_THREADS, sizeof(BlockSmem<SMALL_MAX>), s>>>(
                w, w.list[L_SMALLB][cur]);
            kt.end(K_SMALLB);
            c->kstat[K_SMALLB].launches += 1;
            stats.kernel_launches += 1;
        }
        for (int q = 0; q < 3; ++q)
            if (joined[q]) PSS_CUDA(cudaEventRecord(c->join_ev[q], c->side[q]));
        if (nbig) {
            kt.begin(K_SAMPLE);
            k_tile_scan<<<1, 1024, 0, st>>>(w, nbig);
            // few segments: the pass waits on single blocks, give them more threads
            const uint32_t seg_threads = nbig < 2 * 148 ? 1024 : 256;
            k_sample<<<nbig, seg_threads, 0, st>>>(w);
            kt.end(K_SAMPLE);
            kt.begin(K_CLASSIFY);
            k_classify<<<ntiles, TILE_THREADS, 0, st>>>(w, nbig);
            kt.end(K_CLASSIFY);
            kt.begin(K_BSTART);
            k_bstart<<<nbig, 512, 0, st>>>(w);
            if (nmulti) {
                // segments of more than CHUNK tiles: chunked destination scan;
                // chunks <= tiles, and <= one per CHUNK tiles plus one per segment
                const uint32_t nchunk = std::min<uint32_t>(ntiles, ntiles / CHUNK + nbig);
                const uint32_t g = std::min<uint32_t>(nchunk, 1024);
                k_chunk_sum<<<dim3(g, (MAX_BKT + 255) / 256), 256, 0, st>>>(w, nbig);
                k_chunk_scan<<<dim3(std::min<uint32_t>(nbig, 256), (MAX_BKT + 127) / 128), 128, 0, st>>>(
                    w, nbig);
                k_tile_offsets<<<dim3(g, (MAX_BKT + 255) / 256), 256, 0, st>>>(w, nbig);
                c->kstat[K_BSTART].launches += 3;
                stats.kernel_launches += 3;
            }
            kt.end(K_BSTART);
            kt.begin(K_SCATTER);
            k_scatter<<<ntiles, TILE_THREADS, sizeof(ScatterSmem), st>>>(w, nbig);
            kt.end(K_SCATTER);
            kt.begin(K_CHILDREN);
            k_children<<<nbig, seg_threads, 0, st>>>(w);
            kt.end(K_CHILDREN);
            c->kstat[K_SAMPLE].launches += 2;
            c->kstat[K_CLASSIFY].launches += 1;
            c->kstat[K_BSTART].launches += 1;
            c->kstat[K_SCATTER].launches += 1;
            c->kstat[K_CHILDREN].launches += 1;
            stats.kernel_launches += 6;
            stats.passes += 1;
        }
        for (int q = 0; q < 3; ++q)
            if (joined[q]) PSS_CUDA(cudaStreamWaitEvent(st, c->join_ev[q], 0));
        PSS_CUDA(cudaGetLastError());
        PSS_CUDA(cudaMemcpyAsync(hc, w.counters, 4 * C_COUNT, cudaMemcpyDeviceToHost, st));
        PSS_CUDA(cudaStreamSynchronize(st));
        kt.collect();
        {
            // per-string algorithmic bytes of each kernel class: key gather
            // 4 id + 8 chars + 8 key write; classify 8 key read; scatter
            // 12 read + 12 write; base case 12 read + output
            // (a string behind a common-prefix jump also reads 8 chars per
            // shared chunk)
            const uint64_t big = hc[C_P_BIG], stale = hc[C_P_STALE], fin = hc[C_P_FINAL];
            const uint64_t jch = hc[C_P_JCHUNKS];
            const uint64_t sc = hc[C_P_SCATTER];
            stats.big_elements += big;
            c->kstat[K_SAMPLE].strings += big;
            c->kstat[K_CLASSIFY].strings += big + fin;
            c->kstat[K_CLASSIFY].alg_bytes +=
                20 * stale + 8 * (big - stale) + (4 + out_bytes) * fin + 8 * jch;
            c->kstat[K_SCATTER].strings += sc;
            c->kstat[K_SCATTER].alg_bytes += 24 * sc;
            const int sk[3] = {K_TINY, K_SMALLA, K_SMALLB};
            const int lk[3] = {L_TINY, L_SMALLA, L_SMALLB};
            for (int q = 0; q < 3; ++q) {
                c->kstat[sk[q]].strings += nstr[lk[q]];
                c->kstat[sk[q]].alg_bytes += (12 + out_bytes) * nstr[lk[q]];
                small_segments += cnt[lk[q]];
            }
            c->kstat[K_CHILDREN].strings += big;
            if (c->trace) {
                std::fprintf(stderr,
                             "pssgpu pass %u: big %u segs %u tiles %llu strings (%llu stale, %llu tied, "
                             "%llu jump chunks, %llu final) | tiny %u/%u small256 %u/%u small1024 %u/%u deep %u",
                             npass, nbig, ntiles, (unsigned long long)big, (unsigned long long)stale,
                             (unsigned long long)hc[C_P_TIE], (unsigned long long)jch, (unsigned long long)fin,
                             cnt[L_TINY], nstr[L_TINY], cnt[L_SMALLA], nstr[L_SMALLA], cnt[L_SMALLB],
                             nstr[L_SMALLB], ndeep);
                if (c->profile)
                    for (int k = 0; k < K_NCLASS; ++k)
                        if (kt.pass_ms[k] > 0) std::fprintf(stderr, " %s %.3f", kclass_name[k], kt.pass_ms[k]);
                std::fprintf(stderr, "\n");
            }
        }
        for (int k = 0; k < L_NCLASS; ++k) {
            cnt[k] = hc[C_PAR * nxt + k];
            nstr[k] = k == L_BIG ? 0u : hc[C_PAR * nxt + C_NSTR + k];
        }
        ntiles = hc[C_PAR * nxt + C_NTILES];
        nmulti = hc[C_MULTI + nxt];
        ndeep = hc[C_DEEP + nxt];
        err = hc[C_ERR];
        cur = nxt;
    }
    if (!err && suffix && hc[C_DBL]) {
        kt.begin(K_DBL);
        rc = run_doubling(c, w, std::min(hc[C_DBL], w.dbl_cap), st, stats, &err);
        kt.end(K_DBL);
        if (rc) return rc;
    }
    if (!err && lcp) {
        kt.begin(K_BOUNDARY);
        k_boundary_lcp<<<1184, 256, 0, st>>>(w);
        kt.end(K_BOUNDARY);
        c->kstat[K_BOUNDARY].launches += 1;
        stats.kernel_launches += 1;
    }
    if (!err && d_inst) {
        k_localize<<<std::max(1u, (n + LOC_CHUNK - 1) / LOC_CHUNK), 256, 0, st>>>(perm, lcp, d_inst, ninst, n);
        stats.kernel_launches += 1;
    }
    PSS_CUDA(cudaEventRecord(c->ev1, st));
    PSS_CUDA(cudaMemcpyAsync(hc, w.counters, 4 * C_COUNT, cudaMemcpyDeviceToHost, st));
    PSS_CUDA(cudaStreamSynchronize(st));
    kt.collect();
    if (lcp) {
        // boundary (position, depth) 8 + two perm reads 8 + two keys 16 + lcp 4
        c->kstat[K_BOUNDARY].strings += hc[C_NBND];
        c->kstat[K_BOUNDARY].alg_bytes += 36ull * hc[C_NBND];
    }
    PSS_CUDA(cudaGetLastError());
    err = hc[C_ERR];
    stats.small_segments = small_segments;
    stats.boundaries = hc[C_NBND];
    cudaEventElapsedTime(&stats.device_ms, c->ev0, c->ev1);
    c->stats = stats;
    if (err) return map_device_error(err);
    return PSSGPU_OK;
}

static void ctx_destroy(Ctx* c);

static int ctx_create(int device, Ctx** out)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return fail(PSSGPU_ENODEV, "no CUDA device available");
    if (device < 0 || device >= count) return fail(PSSGPU_EINVAL, "device index out of range");
    PSS_CUDA(cudaSetDevice(device));
    Ctx* c = new Ctx;
    c->trace = std::getenv("PSSGPU_TRACE") != nullptr;
    c->device = device;
    // the context's stream orders with the legacy default stream (a blocking
    // stream), so a call without a stream sees the caller's earlier work there
    bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault) == cudaSuccess &&
              cudaEventCreate(&c->ev0) == cudaSuccess && cudaEventCreate(&c->ev1) == cudaSuccess &&
              cudaHostAlloc((void**)&c->host_counters, 4 * C_COUNT, cudaHostAllocDefault) ==
                  cudaSuccess;
    for (int k = 0; ok && k < 2 * K_NCLASS; ++k) ok = cudaEventCreate(&c->kev[k]) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) == cudaSuccess;
    for (int q = 0; ok && q < 3; ++q)
        ok = cudaStreamCreateWithFlags(&c->side[q], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->join_ev[q], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        ctx_destroy(c);
        return fail(PSSGPU_ECUDA, "stream/event/pinned allocation failed");
    }
    *out = c;
    return PSSGPU_OK;
}

static void ctx_destroy(Ctx* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->ws) cudaFree(c->ws);
    if (c->io) cudaFree(c->io);
    if (c->io2) cudaFree(c->io2);
    if (c->prep) cudaFree(c->prep);
    if (c->mbuf) cudaFree(c->mbuf);
    if (c->sfx) cudaFree(c->sfx);
    if (c->inst_buf) cudaFree(c->inst_buf);
    if (c->host_counters) cudaFreeHost(c->host_counters);
    if (c->gap_host) cudaFreeHost(c->gap_host);
    if (c->ptr_host) cudaFreeHost(c->ptr_host);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (int k = 0; k < 2 * K_NCLASS; ++k)
        if (c->kev[k]) cudaEventDestroy(c->kev[k]);
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    for (int q = 0; q < 3; ++q) {
        if (c->join_ev[q]) cudaEventDestroy(c->join_ev[q]);
        if (c->side[q]) cudaStreamDestroy(c->side[q]);
    }
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

static int ensure_io(Ctx* c, uint64_t bytes) { return ensure_buf(&c->io, &c->io_bytes, bytes); }

static int check_args(uint64_t nchars, uint64_t n)
{
    if (n > PSSGPU_MAX_STRINGS) return fail(PSSGPU_EINVAL, "too many strings for one call");
    if (n > 0 && nchars == 0) return fail(PSSGPU_EINVAL, "empty arena with strings");
    return PSSGPU_OK;
}

// Text on the device -> arena + offsets (prepare.cuh), in two steps: the
// string count (for lines: separators per chunk and their scan, kept in
// c->prep for the second step), then the offsets and the NUL rewrite. Caller
// holds c->mu; d_text is 8-byte aligned and readable / writable for size +
// PSSGPU_ARENA_PAD bytes; size > 0.
static int text_count(Ctx* c, const uint8_t* d_text, uint64_t size, int mode, uint64_t* n_out,
                      cudaStream_t st)
{
    if (mode == PSSGPU_TEXT_SUFFIXES) {
        *n_out = size;
        return PSSGPU_OK;
    }
    const uint64_t nchunk = (size - 1 + PREP_CHUNK - 1) / PREP_CHUNK;
    if (nchunk > 0xFFFFFFFFull) return fail(PSSGPU_EINVAL, "text too large");
    const uint64_t b_cnt = align256(4 * nchunk), b_base = align256(8 * nchunk);
    int rc;
    if ((rc = ensure_buf(&c->prep, &c->prep_bytes, b_cnt + b_base + 256))) return rc;
    uint64_t total = 0;
    if (nchunk) {
        uint32_t* d_cnt = (uint32_t*)c->prep;
        uint64_t* d_base = (uint64_t*)(c->prep + b_cnt);
        uint64_t* d_total = (uint64_t*)(c->prep + b_cnt + b_base);
        uint64_t* h_total = reinterpret_cast<uint64_t*>(c->host_counters);
        k_text_count<<<(unsigned)nchunk, PREP_THREADS, 0, st>>>(d_text, size, d_cnt);
        k_text_scan<<<1, 1024, 0, st>>>(d_cnt, (uint32_t)nchunk, d_base, d_total);
        PSS_CUDA(cudaGetLastError());
        PSS_CUDA(cudaMemcpyAsync(h_total, d_total, 8, cudaMemcpyDeviceToHost, st));
        PSS_CUDA(cudaStreamSynchronize(st));
        total = *h_total;
    }
    *n_out = 1 + total;
    return PSSGPU_OK;
}

// The second step, after text_count on the same text: d_offs holds n entries.
static int text_write(Ctx* c, uint8_t* d_text, uint64_t size, int mode, uint64_t* d_offs,
                      cudaStream_t st)
{
    if (mode == PSSGPU_TEXT_SUFFIXES) {
        const uint64_t blocks = std::min<uint64_t>((size + 255) / 256, 148ull * 16);
        k_text_suffixes<<<(unsigned)blocks, 256, 0, st>>>(d_offs, size);
    } else {
        const uint64_t nchunk = (size - 1 + PREP_CHUNK - 1) / PREP_CHUNK;
        const uint64_t* d_base = (const uint64_t*)(c->prep + align256(4 * nchunk));
        PSS_CUDA(cudaMemsetAsync(d_offs, 0, 8, st));  // string 0 starts at 0
        if (nchunk) k_text_lines<<<(unsigned)nchunk, PREP_THREADS, 0, st>>>(d_text, size, d_base, d_offs);
    }
    PSS_CUDA(cudaGetLastError());
    PSS_CUDA(cudaMemsetAsync(d_text + size - 1, 0, 1, st));  // the last string ends there
    return PSSGPU_OK;
}

// Host text in, host results out (the body of pssgpu_sort_text_host; the
// suffix-pointer drop-ins use it too). Caller holds c->mu; size > 0.
static int sort_text_host_locked(Ctx* c, const uint8_t* text, uint64_t size, int mode,
                                 uint32_t* perm, uint32_t* lcp, uint64_t cap, uint64_t* n_out)
{
    PSS_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    const uint64_t b_text = align256(size + PSSGPU_ARENA_PAD);
    int rc;
    if ((rc = ensure_io(c, b_text))) return rc;
    uint8_t* d_text = c->io;
    PSS_CUDA(cudaMemcpyAsync(d_text, text, size, cudaMemcpyHostToDevice, st));
    PSS_CUDA(cudaMemsetAsync(d_text + size, 0, b_text - size, st));
    uint64_t n = 0;
    if ((rc = text_count(c, d_text, size, mode, &n, st))) return rc;
    *n_out = n;
    if (n > cap) return fail(PSSGPU_EINVAL, "result arrays too small");
    if ((rc = check_args(size, n))) return rc;
    const uint64_t b_offs = align256(8 * n), b_perm = align256(4 * n);
    const uint64_t b_lcp = lcp ? align256(4 * n) : 0;
    if ((rc = ensure_buf(&c->io2, &c->io2_bytes, b_offs + b_perm + b_lcp))) return rc;
    uint64_t* d_offs = (uint64_t*)c->io2;
    uint32_t* d_perm = (uint32_t*)(c->io2 + b_offs);
    uint32_t* d_lcp = lcp ? (uint32_t*)(c->io2 + b_offs + b_perm) : nullptr;
    if ((rc = text_write(c, d_text, size, mode, d_offs, st))) return rc;
    if ((rc = run_sort(c, d_text, size, d_offs, (uint32_t)n, d_perm, d_lcp, st))) return rc;
    PSS_CUDA(cudaMemcpyAsync(perm, d_perm, 4 * n, cudaMemcpyDeviceToHost, st));
    if (lcp && n > 1)
        PSS_CUDA(cudaMemcpyAsync(lcp + 1, d_lcp + 1, 4 * (n - 1), cudaMemcpyDeviceToHost, st));
    PSS_CUDA(cudaStreamSynchronize(st));
    return PSSGPU_OK;
}

// fn(part, lo, hi) over `parts` contiguous slices of [0, n), one host thread
// per slice, from OpenMP's pool (its threads outlive the call, so a call
// costs no thread start-up).
template <class F>
static void host_parts(size_t n, size_t parts, F fn)
{
    if (parts <= 1) {
        fn((size_t)0, (size_t)0, n);
        return;
    }
#pragma omp parallel for num_threads((int)parts) schedule(static, 1)
    for (long long p = 0; p < (long long)parts; ++p)
        fn((size_t)p, n * (size_t)p / parts, n * ((size_t)p + 1) / parts);
}

// Slices for host_parts: one per 64 Ki items, at most one per hardware thread
// (capped at 32).
static size_t host_slices(size_t n)
{
    const size_t hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    return std::max<size_t>(1, std::min(hw, n >> 16));
}

// Offset arrays of at least this many strings may cross PCIe as gaps.
constexpr uint64_t GAP_MIN_N = 1u << 20;

// Copy n host offsets to d_offs on stream st. When the offsets never
// decrease (strings laid out in order, as psstest's loader and the packing
// of pointer arrays leave them) and every gap is below 65536, host threads
// write the gaps in 1 or 2 bytes each to a pinned buffer while the copies
// already queued on st run, 1-2 bytes instead of 8 cross PCIe, and
// k_gap_sum / k_text_scan / k_gap_offsets rebuild the offsets in HBM.
// scratch (device, 256-byte aligned, free until the sort writes it) takes
// the gaps and the chunk sums; when it is too small, or n < GAP_MIN_N, or
// the offsets do not qualify, the offsets are copied as they are.
static int upload_offsets(Ctx* c, const uint64_t* offs, uint64_t n, uint64_t* d_offs,
                          unsigned char* scratch, uint64_t scratch_bytes, cudaStream_t st)
{
    const uint64_t nchunk = (n + GAP_CHUNK - 1) / GAP_CHUNK;
    const uint64_t padded = nchunk * GAP_CHUNK;
    auto need = [&](uint64_t w) {
        return align256(w * padded) + align256(4 * nchunk) + 8 * (nchunk + 1);
    };
    if (n < GAP_MIN_N || need(2) > scratch_bytes) {
        PSS_CUDA(cudaMemcpyAsync(d_offs, offs, 8 * n, cudaMemcpyHostToDevice, st));
        return PSSGPU_OK;
    }
    if (!c->gap_host || c->gap_host_bytes < 2 * n) {
        if (c->gap_host) cudaFreeHost(c->gap_host);
        c->gap_host = nullptr;
        c->gap_host_bytes = 0;
        if (cudaHostAlloc((void**)&c->gap_host, 2 * n, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            c->gap_host = nullptr;
            PSS_CUDA(cudaMemcpyAsync(d_offs, offs, 8 * n, cudaMemcpyHostToDevice, st));
            return PSSGPU_OK;
        }
        c->gap_host_bytes = 2 * n;
    }
    const size_t parts = host_slices(n);
    std::vector<uint8_t> ok(parts, 1);
    std::vector<uint64_t> mx(parts, 0);
    uint8_t* g8 = c->gap_host;
    host_parts(n, parts, [&](size_t p, size_t b, size_t e) {
        uint64_t prev = offs[b ? b - 1 : 0], m = 0;
        bool up = true;
        for (size_t i = b; i < e; ++i) {
            const uint64_t o = offs[i];
            up &= o >= prev;
            m = std::max(m, o - prev);
            g8[i] = (uint8_t)(o - prev);
            prev = o;
        }
        ok[p] = up;
        mx[p] = m;
    });
    uint64_t m = 0;
    for (size_t p = 0; p < parts; ++p) {
        if (!ok[p]) m = ~0ull;
        m = std::max(m, mx[p]);
    }
    if (m >= 65536) {
        PSS_CUDA(cudaMemcpyAsync(d_offs, offs, 8 * n, cudaMemcpyHostToDevice, st));
        return PSSGPU_OK;
    }
    const uint64_t w = m < 256 ? 1 : 2;
    if (w == 2) {
        uint16_t* g16 = reinterpret_cast<uint16_t*>(c->gap_host);
        host_parts(n, parts, [&](size_t, size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) g16[i] = (uint16_t)(i ? offs[i] - offs[i - 1] : 0);
        });
    }
    unsigned char* d_gaps = scratch;
    uint32_t* d_cnt = reinterpret_cast<uint32_t*>(scratch + align256(w * padded));
    uint64_t* d_base = reinterpret_cast<uint64_t*>(scratch + align256(w * padded) + align256(4 * nchunk));
    PSS_CUDA(cudaMemcpyAsync(d_gaps, c->gap_host, w * n, cudaMemcpyHostToDevice, st));
    PSS_CUDA(cudaMemsetAsync(d_gaps + w * n, 0, w * (padded - n), st));
    const unsigned nb = (unsigned)nchunk;
    if (w == 1) {
        k_gap_sum<uint8_t><<<nb, GAP_THREADS, 0, st>>>(d_gaps, d_cnt);
        k_text_scan<<<1, 1024, 0, st>>>(d_cnt, nb, d_base, d_base + nchunk);
        k_gap_offsets<uint8_t><<<nb, GAP_THREADS, 0, st>>>(d_gaps, n, offs[0], d_base, d_offs);
    } else {
        const uint16_t* g = reinterpret_cast<const uint16_t*>(d_gaps);
        k_gap_sum<uint16_t><<<nb, GAP_THREADS, 0, st>>>(g, d_cnt);
        k_text_scan<<<1, 1024, 0, st>>>(d_cnt, nb, d_base, d_base + nchunk);
        k_gap_offsets<uint16_t><<<nb, GAP_THREADS, 0, st>>>(g, n, offs[0], d_base, d_offs);
    }
    PSS_CUDA(cudaGetLastError());
    return PSSGPU_OK;
}

// Host buffers in, host buffers out. Caller holds c->mu.
static int sort_host_locked(Ctx* c, const uint8_t* chars, uint64_t nchars, const uint64_t* offs,
                            uint64_t n, uint32_t* perm, uint32_t* lcp)
{
    int rc = check_args(nchars, n);
    if (rc) return rc;
    if (n == 0) return PSSGPU_OK;
    if (chars[nchars - 1] != 0) return fail(PSSGPU_EINVAL, "arena does not end with NUL");
    PSS_CUDA(cudaSetDevice(c->device));
    const uint64_t b_chars = align256(nchars + PSSGPU_ARENA_PAD);
    const uint64_t b_offs = align256(8 * n);
    const uint64_t b_perm = align256(4 * n);
    const uint64_t b_lcp = lcp ? align256(4 * n) : 0;
    if ((rc = ensure_io(c, b_chars + b_offs + b_perm + b_lcp))) return rc;
    uint8_t* d_chars = c->io;
    uint64_t* d_offs = (uint64_t*)(c->io + b_chars);
    uint32_t* d_perm = (uint32_t*)(c->io + b_chars + b_offs);
    uint32_t* d_lcp = lcp ? (uint32_t*)(c->io + b_chars + b_offs + b_perm) : nullptr;
    cudaStream_t st = c->stream;
    PSS_CUDA(cudaMemcpyAsync(d_chars, chars, nchars, cudaMemcpyHostToDevice, st));
    PSS_CUDA(cudaMemsetAsync(d_chars + nchars, 0, b_chars - nchars, st));
    if ((rc = upload_offsets(c, offs, n, d_offs, (unsigned char*)d_perm, b_perm, st))) return rc;
    if ((rc = run_sort(c, d_chars, nchars, d_offs, (uint32_t)n, d_perm, d_lcp, st))) return rc;
    PSS_CUDA(cudaMemcpyAsync(perm, d_perm, 4 * n, cudaMemcpyDeviceToHost, st));
    if (lcp && n > 1)
        PSS_CUDA(cudaMemcpyAsync(lcp + 1, d_lcp + 1, 4 * (n - 1), cudaMemcpyDeviceToHost, st));
    PSS_CUDA(cudaStreamSynchronize(st));
    return PSSGPU_OK;
}

// Batch: check the instance boundaries and copy them to the device.
static int stage_instances(Ctx* c, const uint64_t* inst, uint32_t ninst, uint64_t n,
                           cudaStream_t st)
{
    if (!inst || ninst == 0) return fail(PSSGPU_EINVAL, "batch without instances");
    if (inst[0] != 0 || inst[ninst] != n)
        return fail(PSSGPU_EINVAL, "instance boundaries must start at 0 and end at n");
    for (uint32_t k = 0; k < ninst; ++k)
        if (inst[k + 1] < inst[k]) return fail(PSSGPU_EINVAL, "instance boundaries decrease");
    const uint64_t need = (uint64_t)ninst + 1;
    if (!c->inst_buf || c->inst_cap < need) {
        if (c->inst_buf) cudaFree(c->inst_buf);
        c->inst_buf = nullptr;
        PSS_CUDA(cudaMalloc(&c->inst_buf, 8 * need));
        c->inst_cap = need;
    }
    PSS_CUDA(cudaMemcpyAsync(c->inst_buf, inst, 8 * need, cudaMemcpyHostToDevice, st));
    return PSSGPU_OK;
}

static int sort_batch_host_locked(Ctx* c, const uint8_t* chars, uint64_t nchars,
                                  const uint64_t* offs, const uint64_t* inst, uint32_t ninst,
                                  uint32_t* perm, uint32_t* lcp)
{
    const uint64_t n = inst ? inst[ninst] : 0;
    int rc = check_args(nchars, n);
    if (rc) return rc;
    if (n == 0) return PSSGPU_OK;
    if (chars[nchars - 1] != 0) return fail(PSSGPU_EINVAL, "arena does not end with NUL");
    PSS_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    if ((rc = stage_instances(c, inst, ninst, n, st))) return rc;
    const uint64_t b_chars = align256(nchars + PSSGPU_ARENA_PAD);
    const uint64_t b_offs = align256(8 * n);
    const uint64_t b_perm = align256(4 * n);
    const uint64_t b_lcp = lcp ? align256(4 * n) : 0;
    if ((rc = ensure_io(c, b_chars + b_offs + b_perm + b_lcp))) return rc;
    uint8_t* d_chars = c->io;
    uint64_t* d_offs = (uint64_t*)(c->io + b_chars);
    uint32_t* d_perm = (uint32_t*)(c->io + b_chars + b_offs);
    uint32_t* d_lcp = lcp ? (uint32_t*)(c->io + b_chars + b_offs + b_perm) : nullptr;
    PSS_CUDA(cudaMemcpyAsync(d_chars, chars, nchars, cudaMemcpyHostToDevice, st));
    PSS_CUDA(cudaMemsetAsync(d_chars + nchars, 0, b_chars - nchars, st));
    if ((rc = upload_offsets(c, offs, n, d_offs, (unsigned char*)d_perm, b_perm, st))) return rc;
    if ((rc = run_sort(c, d_chars, nchars, d_offs, (uint32_t)n, d_perm, d_lcp, st, c->inst_buf,
                       ninst)))
        return rc;
    PSS_CUDA(cudaMemcpyAsync(perm, d_perm, 4 * n, cudaMemcpyDeviceToHost, st));
    if (lcp) PSS_CUDA(cudaMemcpyAsync(lcp, d_lcp, 4 * n, cudaMemcpyDeviceToHost, st));
    PSS_CUDA(cudaStreamSynchronize(st));
    return PSSGPU_OK;
}

// Default contexts for the pointer-array drop-ins, one per device.
static Ctx* default_ctx(int device, int* rc)
{
    static std::mutex mu;
    static std::vector<Ctx*> ctxs;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)ctxs.size() <= device) ctxs.resize(device + 1, nullptr);
    if (!ctxs[device]) {
        Ctx* c = nullptr;
        *rc = ctx_create(device, &c);
        if (*rc) return nullptr;
        ctxs[device] = c;
    }
    *rc = PSSGPU_OK;
    return ctxs[device];
}

// Pack a pointer array into (arena, offsets), sort it and write the sorted
// pointers to `out` (== strings: in place, as parallel_sample_sort_base;
// else a separate output array, as parallel_sample_sort_out_base,
// bingmann-parallel_sample_sort.hpp:1704-1714, with strings left unchanged).
// With arena_lo the caller vouches that every string, NUL included, lies in
// arena_lo[0, arena_size): the span from the lowest string pointer to the end
// of the highest string is copied as is (psstest's string data, suffix
// pointers). Without it every string is gathered by strlen / memcpy, so
// strings in separate allocations are fine and no byte between them is read.
static int sort_pointer_array(unsigned char** strings, unsigned char** out, uintptr_t* lcp_out,
                              uint8_t* cache, size_t n, const uint8_t* arena_lo,
                              uint64_t arena_size)
{
    if (n > PSSGPU_MAX_STRINGS) return fail(PSSGPU_EINVAL, "too many strings for one call");
    if (n == 0) return PSSGPU_OK;
    if (n == 1) {
        out[0] = strings[0];
        return PSSGPU_OK;
    }
    int rc;
    Ctx* c = default_ctx(0, &rc);
    if (!c) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    const size_t parts = host_slices(n);
    // offsets, permutation and LCPs in the context's pinned buffer (copies at
    // full PCIe speed, no page faults per call), or in ordinary host memory
    // when that much cannot be pinned
    const uint64_t need = 8ull * n + 4ull * n + (lcp_out ? 4ull * n : 0ull);
    std::vector<uint64_t> unpinned;
    unsigned char* hbuf = c->ptr_host;
    if (!c->ptr_host || c->ptr_host_bytes < need) {
        if (c->ptr_host) cudaFreeHost(c->ptr_host);
        c->ptr_host = nullptr;
        c->ptr_host_bytes = 0;
        if (cudaHostAlloc((void**)&c->ptr_host, need, cudaHostAllocDefault) == cudaSuccess) {
            c->ptr_host_bytes = need;
            hbuf = c->ptr_host;
        } else {
            cudaGetLastError();
            c->ptr_host = nullptr;
            unpinned.resize((need + 7) / 8);
            hbuf = reinterpret_cast<unsigned char*>(unpinned.data());
        }
    }
    uint64_t* const offs = reinterpret_cast<uint64_t*>(hbuf);
    uint32_t* const perm = reinterpret_cast<uint32_t*>(hbuf + 8ull * n);
    uint32_t* const lcp32 = lcp_out ? perm + n : nullptr;
    std::vector<uint8_t> packed;
    const uint8_t* arena;
    uint64_t nchars;
    if (arena_lo) {
        const uintptr_t A = (uintptr_t)arena_lo, E = A + arena_size;
        std::vector<uintptr_t> plo(parts, UINTPTR_MAX), phi(parts, 0);
        std::vector<char> bad(parts, 0), seq(parts, 1);
        const uintptr_t s0 = (uintptr_t)strings[0];
        host_parts(n, parts, [&](size_t p, size_t b, size_t e) {
            uintptr_t lo = UINTPTR_MAX, hi = 0;
            bool sq = true;  // strings[i] == strings[0] + i: every suffix of one text
            for (size_t i = b; i < e; ++i) {
                const uintptr_t s = (uintptr_t)strings[i];
                lo = std::min(lo, s);
                hi = std::max(hi, s);
                sq = sq && s == s0 + i;
            }
            plo[p] = lo;
            phi[p] = hi;
            bad[p] = lo < A || hi >= E;
            seq[p] = sq;
        });
        uintptr_t lo = UINTPTR_MAX, hi = 0;
        bool suffixes = true;
        for (size_t p = 0; p < parts; ++p) {
            if (bad[p]) return fail(PSSGPU_EINVAL, "a string pointer lies outside the arena");
            lo = std::min(lo, plo[p]);
            hi = std::max(hi, phi[p]);
            suffixes = suffixes && seq[p];
        }
        if (suffixes && ((const uint8_t*)lo)[n - 1] == 0) {
            // all suffixes of the text lo[0, n) (psstest --suffix): only the
            // text crosses to the device, which makes the offsets itself, and
            // the sorted pointers are lo + perm[i]
            uint64_t nn = 0;
            rc = sort_text_host_locked(c, (const uint8_t*)lo, n, PSSGPU_TEXT_SUFFIXES, perm, lcp32, n,
                                       &nn);
            if (rc) return rc;
            if (nn != n) return fail(PSSGPU_ECUDA, "suffix count differs");
            host_parts(n, parts, [&](size_t, size_t b, size_t e) {
                for (size_t i = b; i < e; ++i) out[i] = (unsigned char*)(lo + perm[i]);
                if (lcp_out)
                    for (size_t i = std::max<size_t>(b, 1); i < e; ++i) lcp_out[i] = lcp32[i];
                if (cache && lcp_out)
                    for (size_t i = std::max<size_t>(b, 1); i < e; ++i) cache[i] = out[i][lcp_out[i]];
            });
            return PSSGPU_OK;
        }
        const size_t tail = strnlen((const char*)hi, E - hi);
        if (tail == E - hi) return fail(PSSGPU_EINVAL, "a string is not terminated inside the arena");
        arena = (const uint8_t*)lo;
        nchars = hi + tail + 1 - lo;
        host_parts(n, parts, [&](size_t, size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) offs[i] = (uintptr_t)strings[i] - lo;
        });
    } else {
        // lengths per slice, slice bases, then offsets and copies
        std::vector<uint64_t> base(parts + 1, 0);
        host_parts(n, parts, [&](size_t p, size_t b, size_t e) {
            uint64_t t = 0;
            for (size_t i = b; i < e; ++i) {
                offs[i] = t;
                t += strlen((const char*)strings[i]) + 1;
            }
            base[p + 1] = t;
        });
        for (size_t p = 0; p < parts; ++p) base[p + 1] += base[p];
        nchars = base[parts];
        packed.resize(nchars);
        host_parts(n, parts, [&](size_t p, size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) {
                const uint64_t o = base[p] + offs[i];
                const uint64_t len = (i + 1 < e ? offs[i + 1] + base[p] : base[p + 1]) - o;
                memcpy(packed.data() + o, strings[i], len);
                offs[i] = o;
            }
        });
        arena = packed.data();
    }
    rc = sort_host_locked(c, arena, nchars, offs, n, perm, lcp32);
    if (rc) return rc;
    // sorted pointers: in the caller's buffer string id's pointer is
    // arena + offs[id]; gathered strings need the original array (a copy
    // of it when the output overwrites it)
    std::vector<unsigned char*> orig;
    unsigned char* const* src = strings;
    if (!arena_lo && out == strings) {
        orig.resize(n);
        host_parts(n, parts, [&](size_t, size_t b, size_t e) {
            memcpy(orig.data() + b, strings + b, (e - b) * sizeof(unsigned char*));
        });
        src = orig.data();
    }
    host_parts(n, parts, [&](size_t, size_t b, size_t e) {
        if (arena_lo)
            for (size_t i = b; i < e; ++i) out[i] = const_cast<unsigned char*>(arena) + offs[perm[i]];
        else
            for (size_t i = b; i < e; ++i) out[i] = src[perm[i]];
        if (lcp_out)
            for (size_t i = std::max<size_t>(b, 1); i < e; ++i) lcp_out[i] = lcp32[i];
        if (cache && lcp_out)
            for (size_t i = std::max<size_t>(b, 1); i < e; ++i) cache[i] = out[i][lcp_out[i]];
    });
    return PSSGPU_OK;
}

}  // namespace pssgpu

#include "server.cuh"

using namespace pssgpu;

extern "C" {

int pssgpu_server_create(int device, const pssgpu_server_config* cfg, pssgpu_server** out)
{
    if (!cfg || !out) return fail(PSSGPU_EINVAL, "null argument");
    if (cfg->workers < 1 || cfg->workers > 16) return fail(PSSGPU_EINVAL, "1..16 workers");
    if (cfg->max_batch_strings < 1024 || cfg->max_batch_strings > PSSGPU_MAX_STRINGS)
        return fail(PSSGPU_EINVAL, "max_batch_strings out of range");
    Server* s = new Server;
    s->device = device;
    s->budget = cfg->hbm_budget;
    s->max_batch_strings = cfg->max_batch_strings;
    s->max_batch_requests = cfg->max_batch_requests ? cfg->max_batch_requests : 4096;
    auto bail = [&](int rc) {
        pssgpu_server_destroy(reinterpret_cast<pssgpu_server*>(s));
        return rc;
    };
    // each worker reserves a workspace and batch buffers for its largest batch
    const uint64_t per_worker =
        workspace_bytes(sizes_for(cfg->max_batch_strings)) + 16 * cfg->max_batch_strings;
    const uint64_t reserve = per_worker * cfg->workers;
    if (cfg->hbm_budget <= reserve + (64ull << 20))
        return bail(fail(PSSGPU_EBUDGET, "budget below the workers' reserve"));
    s->slab_size = align256(cfg->hbm_budget - reserve) - 256;
    int rc;
    if (cudaSetDevice(device) != cudaSuccess) return bail(fail(PSSGPU_ENODEV, "no such device"));
    if (cudaMalloc(&s->slab, s->slab_size + 256) != cudaSuccess)
        return bail(fail(PSSGPU_ENOMEM, "slab allocation failed"));
    // the slab's tail stays zero: it ends the arena and pads the last reads
    cudaMemset(s->slab + s->slab_size - 256, 0, 512);
    s->alloc.init(s->slab_size - 256);
    if (cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(PSSGPU_ECUDA, "stream creation failed"));
    for (uint32_t i = 0; i < cfg->workers; ++i) {
        Worker* wk = new Worker;
        wk->srv = s;
        s->workers.push_back(wk);
        if ((rc = ctx_create(device, &wk->ctx))) return bail(rc);
        {
            std::lock_guard<std::mutex> lk(wk->ctx->mu);
            if ((rc = ensure_workspace(wk->ctx, cfg->max_batch_strings))) return bail(rc);
        }
        if ((rc = worker_grow(wk, cfg->max_batch_strings, 1024))) return bail(rc);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(PSSGPU_ECUDA, "set-up failed"));
    s->admitter = std::thread(admit_loop, s);
    for (Worker* wk : s->workers) wk->th = std::thread(worker_loop, wk);
    *out = reinterpret_cast<pssgpu_server*>(s);
    return PSSGPU_OK;
}

void pssgpu_server_destroy(pssgpu_server* srv)
{
    Server* s = reinterpret_cast<Server*>(srv);
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_pending.notify_all();
    s->cv_space.notify_all();
    if (s->admitter.joinable()) s->admitter.join();
    s->cv_ready.notify_all();
    for (Worker* wk : s->workers) {
        if (wk->th.joinable()) wk->th.join();
    }
    cudaSetDevice(s->device);
    for (Worker* wk : s->workers) {
        if (wk->d_offs) cudaFree(wk->d_offs);
        if (wk->d_perm) cudaFree(wk->d_perm);
        if (wk->d_lcp) cudaFree(wk->d_lcp);
        if (wk->d_parts) cudaFree(wk->d_parts);
        if (wk->h_parts) cudaFreeHost(wk->h_parts);
        ctx_destroy(wk->ctx);
        delete wk;
    }
    for (auto& kv : s->requests) {
        if (kv.second->uploaded) cudaEventDestroy(kv.second->uploaded);
        delete kv.second;
    }
    if (s->slab) cudaFree(s->slab);
    if (s->upload) cudaStreamDestroy(s->upload);
    delete s;
}

int pssgpu_server_submit(pssgpu_server* srv, const uint8_t* chars, uint64_t nchars,
                         const uint64_t* offs, uint64_t offs_base, uint64_t n, uint32_t* perm,
                         uint32_t* lcp, uint64_t* ticket)
{
    Server* s = reinterpret_cast<Server*>(srv);
    if (!s || !ticket) return fail(PSSGPU_EINVAL, "null argument");
    if (n && (!chars || !offs || !perm || nchars == 0)) return fail(PSSGPU_EINVAL, "null buffer");
    if (n > s->max_batch_strings) return fail(PSSGPU_EBUDGET, "request above max_batch_strings");
    if (n && chars[nchars - 1] != 0) return fail(PSSGPU_EINVAL, "arena does not end with NUL");
    for (uint64_t i = 0; i < n; ++i)
        if (offs[i] - offs_base >= nchars) return fail(PSSGPU_EINVAL, "offset outside the arena");
    Request* r = new Request;
    r->h_chars = chars;
    r->nchars = nchars;
    r->h_offs = offs;
    r->offs_base = offs_base;
    r->n = n;
    r->h_perm = perm;
    r->h_lcp = lcp;
    r->region_bytes = request_bytes(nchars, n);
    if (r->region_bytes > s->slab_size - 256) {
        delete r;
        return fail(PSSGPU_EBUDGET, "request larger than the serving budget");
    }
    if (cudaEventCreateWithFlags(&r->uploaded, cudaEventDisableTiming) != cudaSuccess) {
        delete r;
        return fail(PSSGPU_ECUDA, "event creation failed");
    }
    std::lock_guard<std::mutex> lk(s->mu);
    r->ticket = s->next_ticket++;
    r->t_submit = now_ns();
    s->requests[r->ticket] = r;
    if (n == 0) {
        r->t_admit = r->t_start = r->t_done = r->t_submit;
        r->done = true;
    } else {
        s->pending.push_back(r);
        s->cv_pending.notify_one();
    }
    *ticket = r->ticket;
    return PSSGPU_OK;
}

int pssgpu_server_wait(pssgpu_server* srv, uint64_t ticket, pssgpu_request_info* info)
{
    Server* s = reinterpret_cast<Server*>(srv);
    if (!s) return fail(PSSGPU_EINVAL, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return fail(PSSGPU_EINVAL, "unknown ticket");
    Request* r = it->second;
    s->cv_done.wait(lk, [&] { return r->done; });
    const int rc = r->status;
    if (info) {
        info->status = r->status;
        info->batch_requests = r->batch_requests;
        info->batch_strings = r->batch_strings;
        info->t_submit_ns = r->t_submit;
        info->t_admit_ns = r->t_admit;
        info->t_start_ns = r->t_start;
        info->t_done_ns = r->t_done;
    }
    s->requests.erase(it);
    lk.unlock();
    cudaEventDestroy(r->uploaded);
    delete r;
    return rc ? fail(rc, "request failed") : PSSGPU_OK;
}

int pssgpu_server_get_stats(pssgpu_server* srv, pssgpu_server_stats* out)
{
    Server* s = reinterpret_cast<Server*>(srv);
    if (!s || !out) return fail(PSSGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out->slab_bytes = s->slab_size;
    out->slab_peak_bytes = s->peak_used;
    out->batches = s->batches;
    out->batched_requests = s->batched_requests;
    out->pending = s->pending.size();
    out->ready = s->ready.size();
    return PSSGPU_OK;
}

const char* pssgpu_last_error(void) { return g_last_error.c_str(); }

const char* pssgpu_version(void) { return "pssgpu 0.1 sm_100a"; }

int pssgpu_ctx_create(int device, pssgpu_ctx** out)
{
    if (!out) return fail(PSSGPU_EINVAL, "null output pointer");
    Ctx* c = nullptr;
    int rc = ctx_create(device, &c);
    if (rc) return rc;
    *out = reinterpret_cast<pssgpu_ctx*>(c);
    return PSSGPU_OK;
}

void pssgpu_ctx_destroy(pssgpu_ctx* ctx) { ctx_destroy(reinterpret_cast<Ctx*>(ctx)); }

uint64_t pssgpu_workspace_bytes(uint64_t n)
{
    return workspace_bytes(sizes_for(std::max<uint64_t>(n, 1024)));
}

int pssgpu_ctx_stats(pssgpu_ctx* ctx, pssgpu_stats* out)
{
    if (!ctx || !out) return fail(PSSGPU_EINVAL, "null argument");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    *out = c->stats;
    return PSSGPU_OK;
}

int pssgpu_ctx_set_profile(pssgpu_ctx* ctx, int on)
{
    if (!ctx) return fail(PSSGPU_EINVAL, "null context");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    c->profile = on != 0;
    return PSSGPU_OK;
}

int pssgpu_ctx_set_option(pssgpu_ctx* ctx, int option, int64_t value)
{
    if (!ctx) return fail(PSSGPU_EINVAL, "null context");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    switch (option) {
    case PSSGPU_OPT_PROFILE: c->profile = value != 0; return PSSGPU_OK;
    case PSSGPU_OPT_INDIRECT_HANDLES: c->indirect_handles = value != 0; return PSSGPU_OK;
    case PSSGPU_OPT_SINGLE_LAUNCH: c->single_launch = value != 0; return PSSGPU_OK;
    case PSSGPU_OPT_SUFFIX_DOUBLING: c->suffix_doubling = value != 0; return PSSGPU_OK;
    case PSSGPU_OPT_MERGE_PIECE:
        if (value < 1 || value > (int64_t)MERGE_PIECE_MAX) return fail(PSSGPU_EINVAL, "merge piece out of range");
        c->merge_piece = (uint32_t)value;
        return PSSGPU_OK;
    case PSSGPU_OPT_WAIT_LIMIT:
        if (value < 1 || value > 0xFFFFFFFFll) return fail(PSSGPU_EINVAL, "wait limit out of range");
        c->wait_limit = (uint32_t)value;
        return PSSGPU_OK;
    default: return fail(PSSGPU_EINVAL, "unknown option");
    }
}

int pssgpu_ctx_kernel_stats(pssgpu_ctx* ctx, pssgpu_kernel_stats* out, int max)
{
    if (!ctx || (!out && max > 0)) return -fail(PSSGPU_EINVAL, "null argument");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    int k = 0;
    for (; k < K_NCLASS && k < max; ++k) {
        memset(&out[k], 0, sizeof(out[k]));
        strncpy(out[k].name, kclass_name[k], sizeof(out[k].name) - 1);
        out[k].launches = c->kstat[k].launches;
        out[k].strings = c->kstat[k].strings;
        out[k].alg_bytes = c->kstat[k].alg_bytes;
        out[k].ms = c->kstat[k].ms;
    }
    return k;
}

int pssgpu_sort_host(pssgpu_ctx* ctx, const uint8_t* chars, uint64_t nchars,
                     const uint64_t* offs, uint64_t n, uint32_t* perm, uint32_t* lcp)
{
    if (!ctx) return fail(PSSGPU_EINVAL, "null context");
    if (n && (!chars || !offs || !perm)) return fail(PSSGPU_EINVAL, "null buffer");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    return sort_host_locked(c, chars, nchars, offs, n, perm, lcp);
}

int pssgpu_prepare_text_device(pssgpu_ctx* ctx, uint8_t* d_text, uint64_t size, int mode,
                               uint64_t* d_offs, uint64_t offs_cap, uint64_t* n_out, void* stream)
{
    if (!ctx || !n_out) return fail(PSSGPU_EINVAL, "null context or count");
    *n_out = 0;
    if (mode != PSSGPU_TEXT_LINES && mode != PSSGPU_TEXT_SUFFIXES)
        return fail(PSSGPU_EINVAL, "unknown text mode");
    if (size == 0) return PSSGPU_OK;
    if (!d_text || !d_offs) return fail(PSSGPU_EINVAL, "null buffer");
    if (((uintptr_t)d_text & 7) != 0) return fail(PSSGPU_EINVAL, "text not 8-byte aligned");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    PSS_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    uint64_t n = 0;
    int rc = text_count(c, d_text, size, mode, &n, st);
    if (rc) return rc;
    *n_out = n;
    if (n > offs_cap) return fail(PSSGPU_EINVAL, "offset array too small");
    if ((rc = text_write(c, d_text, size, mode, d_offs, st))) return rc;
    PSS_CUDA(cudaStreamSynchronize(st));
    return PSSGPU_OK;
}

int pssgpu_sort_text_host(pssgpu_ctx* ctx, const uint8_t* text, uint64_t size, int mode,
                          uint32_t* perm, uint32_t* lcp, uint64_t cap, uint64_t* n_out)
{
    if (!ctx || !n_out) return fail(PSSGPU_EINVAL, "null context or count");
    *n_out = 0;
    if (mode != PSSGPU_TEXT_LINES && mode != PSSGPU_TEXT_SUFFIXES)
        return fail(PSSGPU_EINVAL, "unknown text mode");
    if (size == 0) return PSSGPU_OK;
    if (!text || !perm) return fail(PSSGPU_EINVAL, "null buffer");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    return sort_text_host_locked(c, text, size, mode, perm, lcp, cap, n_out);
}

// Outputs per piece of a merge of n strings when the caller set none: at
// most MERGE_PIECE, and as few waves of `wave` pieces (the piece-merge
// threads the GPU holds at once) as that allows, filled evenly, so that no
// wave runs part-empty; at least MERGE_PIECE_MIN (every piece costs a split).
static uint32_t merge_piece_for(uint64_t n, uint64_t wave)
{
    const uint64_t per_wave = (uint64_t)MERGE_PIECE * wave;
    const uint64_t waves = std::max<uint64_t>(1, (n + per_wave - 1) / per_wave);
    const uint64_t p = (n + waves * wave - 1) / (waves * wave);
    return (uint32_t)std::min<uint64_t>(MERGE_PIECE, std::max<uint64_t>(MERGE_PIECE_MIN, p));
}

int pssgpu_merge_lcp_device(pssgpu_ctx* ctx, const uint8_t* d_chars, uint64_t nchars,
                            const uint64_t* d_offs, const uint64_t* runs, uint32_t nruns,
                            const uint32_t* d_ids, const uint32_t* d_lcp, uint32_t* d_ids_out,
                            uint32_t* d_lcp_out, void* stream)
{
    if (!ctx || !runs) return fail(PSSGPU_EINVAL, "null context or runs");
    if (nruns == 0) return fail(PSSGPU_EINVAL, "no runs");
    if (runs[0] != 0) return fail(PSSGPU_EINVAL, "run boundaries must start at 0");
    for (uint32_t k = 0; k < nruns; ++k)
        if (runs[k + 1] < runs[k]) return fail(PSSGPU_EINVAL, "run boundaries decrease");
    const uint64_t n = runs[nruns];
    int rc = check_args(nchars, n);
    if (rc) return rc;
    if (n == 0) return PSSGPU_OK;
    if (!d_chars || !d_offs || !d_ids || !d_ids_out) return fail(PSSGPU_EINVAL, "null buffer");
    if (d_lcp_out && !d_lcp) return fail(PSSGPU_EINVAL, "LCP output needs the runs' LCP arrays");
    if (((uintptr_t)d_chars & 7) != 0) return fail(PSSGPU_EINVAL, "arena not 8-byte aligned");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    PSS_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    uint8_t last = 1;
    PSS_CUDA(cudaMemcpyAsync(&last, d_chars + nchars - 1, 1, cudaMemcpyDeviceToHost, st));
    PSS_CUDA(cudaStreamSynchronize(st));
    if (last != 0) return fail(PSSGPU_EINVAL, "arena does not end with NUL");
    if (nruns == 1) {
        PSS_CUDA(cudaMemcpyAsync(d_ids_out, d_ids, 4 * n, cudaMemcpyDeviceToDevice, st));
        if (d_lcp_out && n > 1)
            PSS_CUDA(cudaMemcpyAsync(d_lcp_out + 1, d_lcp + 1, 4 * (n - 1), cudaMemcpyDeviceToDevice, st));
        PSS_CUDA(cudaStreamSynchronize(st));
        return PSSGPU_OK;
    }
    // runs as handles (32-bit id << hbits | offset) when the offsets fit 32
    // bits: made once, then every round reads offsets in order with the
    // entries instead of gathering them; else as ids
    const uint32_t hbits = std::max<uint32_t>(1, bit_length(nchars - 1));
    const bool packed = hbits <= 32 && !c->indirect_handles;
    const bool with_lcp = d_lcp != nullptr;
    // the piece merge: MS_THREADS threads and their staging per block
    const uint32_t smem_h = sizeof(MergeStage<uint64_t>), smem_i = sizeof(MergeStage<uint32_t>);
    const void* piece_fn = packed ? (const void*)k_merge_lcp_seq<MergeByHandles>
                                  : (const void*)k_merge_lcp_seq<MergeByIds>;
    uint32_t pc = c->merge_piece;
    if (with_lcp) {  // per device: set on every call
        PSS_CUDA(cudaFuncSetAttribute(piece_fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(packed ? smem_h : smem_i)));
        if (!pc) {
            int sms = 0, per_sm = 0;
            PSS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
            PSS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, piece_fn, MS_THREADS,
                                                                   packed ? smem_h : smem_i));
            pc = merge_piece_for(n, (uint64_t)std::max(sms, 1) * std::max(per_sm, 1) * MS_THREADS);
        }
    }
    if (!pc) pc = MERGE_PIECE;
    // pairs and piece counts of every round, uploaded at once: round i
    // merges the runs of level i into those of level i + 1
    std::vector<std::vector<uint64_t>> level{std::vector<uint64_t>(runs, runs + nruns + 1)};
    while (level.back().size() > 2) {
        const std::vector<uint64_t>& a = level.back();
        const uint32_t K = (uint32_t)a.size() - 1, K2 = (K + 1) / 2;
        std::vector<uint64_t> b(K2 + 1);
        for (uint32_t p = 0; p < K2; ++p) b[p] = a[2 * p];
        b[K2] = n;
        level.push_back(std::move(b));
    }
    const size_t rounds = level.size() - 1;
    std::vector<uint64_t> flat;  // per round: pairs, piece starts, coarse-split starts
    std::vector<uint64_t> at_pairs, at_first, at_cfirst, npairs;
    uint64_t max_tasks = 0, max_coarse = 0;
    for (size_t i = 0; i < rounds; ++i) {
        const std::vector<uint64_t>& a = level[i];
        const uint32_t K = (uint32_t)a.size() - 1, np = (K + 1) / 2;
        at_pairs.push_back(flat.size());
        for (uint32_t p = 0; p < np; ++p) {
            const uint64_t a0 = a[2 * p], a1 = a[2 * p + 1];
            const uint64_t b1 = 2 * p + 2 <= K ? a[2 * p + 2] : a1;  // an unpaired last run
            flat.push_back(a0);
            flat.push_back(a1);
            flat.push_back(b1);
        }
        at_first.push_back(flat.size());
        uint64_t t = 0;
        for (uint32_t p = 0; p < np; ++p) {
            flat.push_back(t);
            const uint64_t m = flat[at_pairs.back() + 3 * p + 2] - flat[at_pairs.back() + 3 * p];
            t += (m + pc - 1) / pc;
        }
        flat.push_back(t);
        at_cfirst.push_back(flat.size());
        uint64_t tc = 0;
        for (uint32_t p = 0; p < np; ++p) {
            flat.push_back(tc);
            const uint64_t pieces = flat[at_first.back() + p + 1] - flat[at_first.back() + p];
            tc += (pieces + MERGE_SPLIT_COARSE - 1) / MERGE_SPLIT_COARSE;
        }
        flat.push_back(tc);
        npairs.push_back(np);
        max_tasks = std::max(max_tasks, t);
        max_coarse = std::max(max_coarse, tc);
    }
    // padded past the last entry: the piece merge stages whole chunks of
    // MS_CH entries
    const uint64_t b_v = align256(4 * n + 8 * MS_CH), b_h = align256(8 * n + 8 * MS_CH);
    const uint64_t b_runs = align256(8 * flat.size()), b_split = align256(8 * (max_tasks + 1));
    const uint64_t b_ck = with_lcp ? b_h : 0;
    if ((rc = ensure_buf(&c->mbuf, &c->mbuf_bytes, 2 * b_h + 2 * b_v + 2 * b_ck + b_runs + b_split + 256)))
        return rc;
    unsigned char* tv[2] = {c->mbuf, c->mbuf + b_h};  // ids or handles, by round parity
    uint32_t* tlcp[2] = {(uint32_t*)(c->mbuf + 2 * b_h), (uint32_t*)(c->mbuf + 2 * b_h + b_v)};
    unsigned char* const rest = c->mbuf + 2 * b_h + 2 * b_v;
    uint64_t* tck[2] = {(uint64_t*)rest, (uint64_t*)(rest + b_ck)};  // char caches
    uint64_t* d_flat = (uint64_t*)(rest + 2 * b_ck);
    uint64_t* split = (uint64_t*)(rest + 2 * b_ck + b_runs);
    uint32_t* d_err = (uint32_t*)(rest + 2 * b_ck + b_runs + b_split);
    PSS_CUDA(cudaMemcpyAsync(d_flat, flat.data(), 8 * flat.size(), cudaMemcpyHostToDevice, st));
    PSS_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
    const unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    // with the runs' LCP arrays every round is LCP-aware and carries the
    // merged LCP array and the char caches to the next one (the last round
    // writes d_lcp_out, if any). Its reads are staged in 16-byte copies from
    // the library's own buffers (aligned, padded): k_merge_prep copies the
    // caller's ids (as handles, or as they are) and LCPs in; round 0 writes
    // tv[0], tlcp[0] and tck[0].
    const unsigned char* in_v = (const unsigned char*)d_ids;
    const uint32_t* in_lcp = with_lcp ? tlcp[1] : nullptr;
    const uint64_t* in_ck = with_lcp ? tck[1] : nullptr;
    if (packed) {
        k_merge_prep<true><<<blocks, 256, 0, st>>>(d_offs, nchars, d_ids, d_lcp, n, hbits, tv[1], tlcp[1],
                                                   d_err);
        in_v = tv[1];
    } else {
        k_merge_prep<false><<<blocks, 256, 0, st>>>(d_offs, nchars, d_ids, d_lcp, n, hbits,
                                                    with_lcp ? tv[1] : nullptr, tlcp[1], d_err);
        if (with_lcp) in_v = tv[1];
    }
    const MergeByIds by_ids{d_offs};
    const MergeByHandles by_h{(1ull << hbits) - 1, hbits};
    if (with_lcp) {
        // round 0's caches on a side stream, beside round 0's splits (which
        // do not read them); round 0's piece merge waits for them
        PSS_CUDA(cudaEventRecord(c->fork_ev, st));
        PSS_CUDA(cudaStreamWaitEvent(c->side[0], c->fork_ev, 0));
        cudaStream_t s = c->side[0];
        if (packed)
            k_merge_caches<MergeByHandles><<<blocks, 256, 0, s>>>(d_chars, nchars, by_h, (const uint64_t*)in_v,
                                                                  tlcp[1], n, tck[1]);
        else
            k_merge_caches<MergeByIds><<<blocks, 256, 0, s>>>(d_chars, nchars, by_ids, (const uint32_t*)in_v,
                                                              tlcp[1], n, tck[1]);
        PSS_CUDA(cudaEventRecord(c->join_ev[0], c->side[0]));
    }
    const unsigned ms_blocks =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((max_tasks + MS_THREADS - 1) / MS_THREADS, 148 * 8));
    // coarse splits: one warp each, 8 per block
    const unsigned cs_blocks =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((max_coarse + 7) / 8, 148ull * 16));
    for (size_t i = 0; i < rounds; ++i) {
        const bool lastr = i + 1 == rounds;
        // the last round writes the caller's ids directly unless it merges
        // handles (then the piece merge writes them through ids_out, or
        // k_merge_unpack after a merge without LCPs)
        unsigned char* out_v = lastr && !packed ? (unsigned char*)d_ids_out : tv[i & 1];
        uint32_t* out_lcp = lastr ? d_lcp_out : tlcp[i & 1];
        uint64_t* out_ck = lastr || !with_lcp ? nullptr : tck[i & 1];
        const MergePair* pairs = reinterpret_cast<const MergePair*>(d_flat + at_pairs[i]);
        const uint64_t* first = d_flat + at_first[i];
        const uint64_t* cfirst = d_flat + at_cfirst[i];
        const uint32_t np = (uint32_t)npairs[i];
        // the last round of handles with LCPs writes the caller's ids itself
        uint32_t* ids_out = lastr && packed && with_lcp ? d_ids_out : nullptr;
        // the piece merge of round 0 reads the caches of the side stream
        const bool wait_caches = i == 0 && with_lcp;
        if (packed) {
            const uint64_t* in = (const uint64_t*)in_v;
            uint64_t* out = (uint64_t*)out_v;
            k_merge_split_coarse<MergeByHandles><<<cs_blocks, 256, 0, st>>>(
                d_chars, nchars, by_h, pairs, first, cfirst, np, in, split, pc);
            k_merge_split<MergeByHandles><<<blocks, 256, 0, st>>>(d_chars, nchars, by_h, pairs, first, np, in,
                                                                  split, pc);
            if (wait_caches) PSS_CUDA(cudaStreamWaitEvent(st, c->join_ev[0], 0));
            if (with_lcp)
                k_merge_lcp_seq<MergeByHandles><<<ms_blocks, MS_THREADS, smem_h, st>>>(
                    d_chars, nchars, by_h, pairs, first, np, split, in, in_lcp, in_ck, out, out_lcp, out_ck,
                    ids_out, pc);
            else
                k_merge_seq<MergeByHandles><<<blocks, 256, 0, st>>>(d_chars, nchars, by_h, pairs, first, np,
                                                                    split, in, out, pc);
        } else {
            const uint32_t* in = (const uint32_t*)in_v;
            uint32_t* out = (uint32_t*)out_v;
            k_merge_split_coarse<MergeByIds><<<cs_blocks, 256, 0, st>>>(
                d_chars, nchars, by_ids, pairs, first, cfirst, np, in, split, pc);
            k_merge_split<MergeByIds><<<blocks, 256, 0, st>>>(d_chars, nchars, by_ids, pairs, first, np, in,
                                                              split, pc);
            if (wait_caches) PSS_CUDA(cudaStreamWaitEvent(st, c->join_ev[0], 0));
            if (with_lcp)
                k_merge_lcp_seq<MergeByIds><<<ms_blocks, MS_THREADS, smem_i, st>>>(
                    d_chars, nchars, by_ids, pairs, first, np, split, in, in_lcp, in_ck, out, out_lcp, out_ck,
                    ids_out, pc);
            else
                k_merge_seq<MergeByIds><<<blocks, 256, 0, st>>>(d_chars, nchars, by_ids, pairs, first, np,
                                                                split, in, out, pc);
        }
        PSS_CUDA(cudaGetLastError());
        in_v = out_v;
        in_lcp = out_lcp;
        in_ck = out_ck;
    }
    if (packed && !with_lcp)
        k_merge_unpack<<<blocks, 256, 0, st>>>((const uint64_t*)in_v, n, hbits, d_ids_out);
    uint32_t err = 0;
    PSS_CUDA(cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, st));
    PSS_CUDA(cudaStreamSynchronize(st));
    if (err) return fail(PSSGPU_EINVAL, "a string offset lies outside the arena");
    return PSSGPU_OK;
}

int pssgpu_sort_device(pssgpu_ctx* ctx, const uint8_t* d_chars, uint64_t nchars,
                       const uint64_t* d_offs, uint64_t n, uint32_t* d_perm, uint32_t* d_lcp,
                       void* stream)
{
    if (!ctx) return fail(PSSGPU_EINVAL, "null context");
    int rc = check_args(nchars, n);
    if (rc) return rc;
    if (n == 0) return PSSGPU_OK;
    if (!d_chars || !d_offs || !d_perm) return fail(PSSGPU_EINVAL, "null buffer");
    if (((uintptr_t)d_chars & 7) != 0) return fail(PSSGPU_EINVAL, "arena not 8-byte aligned");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    PSS_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    // the arena's last char is checked on the device by the first kernel
    return run_sort(c, d_chars, nchars, d_offs, (uint32_t)n, d_perm, d_lcp, st);
}

int pssgpu_ctx_set_tree_bits(pssgpu_ctx* ctx, const uint8_t* tree_bits, int count)
{
    if (!ctx || (count > 0 && !tree_bits)) return fail(PSSGPU_EINVAL, "null argument");
    if (count < 0 || count > 33) return fail(PSSGPU_EINVAL, "at most 33 size classes");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    memset(c->tree_bits_by_size, 0, sizeof(c->tree_bits_by_size));
    for (int k = 0; k < count; ++k) {
        if (tree_bits[k] > MAX_TREE_BITS) return fail(PSSGPU_EINVAL, "at most 10 tree levels");
        c->tree_bits_by_size[k] = tree_bits[k];
    }
    return PSSGPU_OK;
}

int pssgpu_sort_batch_host(pssgpu_ctx* ctx, const uint8_t* chars, uint64_t nchars,
                           const uint64_t* offs, const uint64_t* inst, uint32_t ninst,
                           uint32_t* perm, uint32_t* lcp)
{
    if (!ctx) return fail(PSSGPU_EINVAL, "null context");
    if (!inst) return fail(PSSGPU_EINVAL, "null instance boundaries");
    if (inst[ninst] && (!chars || !offs || !perm)) return fail(PSSGPU_EINVAL, "null buffer");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    return sort_batch_host_locked(c, chars, nchars, offs, inst, ninst, perm, lcp);
}

int pssgpu_sort_batch_device(pssgpu_ctx* ctx, const uint8_t* d_chars, uint64_t nchars,
                             const uint64_t* d_offs, const uint64_t* inst, uint32_t ninst,
                             uint32_t* d_perm, uint32_t* d_lcp, void* stream)
{
    if (!ctx) return fail(PSSGPU_EINVAL, "null context");
    if (!inst) return fail(PSSGPU_EINVAL, "null instance boundaries");
    const uint64_t n = inst[ninst];
    int rc = check_args(nchars, n);
    if (rc) return rc;
    if (n == 0) return PSSGPU_OK;
    if (!d_chars || !d_offs || !d_perm) return fail(PSSGPU_EINVAL, "null buffer");
    if (((uintptr_t)d_chars & 7) != 0) return fail(PSSGPU_EINVAL, "arena not 8-byte aligned");
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    PSS_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    if ((rc = stage_instances(c, inst, ninst, n, st))) return rc;
    uint8_t last = 1;
    PSS_CUDA(cudaMemcpyAsync(&last, d_chars + nchars - 1, 1, cudaMemcpyDeviceToHost, st));
    PSS_CUDA(cudaStreamSynchronize(st));
    if (last != 0) return fail(PSSGPU_EINVAL, "arena does not end with NUL");
    return run_sort(c, d_chars, nchars, d_offs, (uint32_t)n, d_perm, d_lcp, st, c->inst_buf, ninst);
}

int pssgpu_sort_strings_status(unsigned char** strings, uintptr_t* lcp, uint8_t* cache, size_t n)
{
    if (n && !strings) return fail(PSSGPU_EINVAL, "null string array");
    return sort_pointer_array(strings, strings, lcp, cache, n, nullptr, 0);
}

int pssgpu_sort_strings_arena(const uint8_t* arena, uint64_t arena_size, unsigned char** strings,
                              unsigned char** output, uintptr_t* lcp, uint8_t* cache, size_t n)
{
    if (n && (!strings || !arena)) return fail(PSSGPU_EINVAL, "null string array or arena");
    if (output == strings) output = nullptr;
    if (output && n && output < strings + n && strings < output + n)
        return fail(PSSGPU_EINVAL, "output overlaps the input array");
    return sort_pointer_array(strings, output ? output : strings, lcp, cache, n, arena, arena_size);
}

int pssgpu_sort_strings_out_status(unsigned char** strings, unsigned char** output, size_t n)
{
    if (n && (!strings || !output)) return fail(PSSGPU_EINVAL, "null string array");
    if (output == strings) return sort_pointer_array(strings, strings, nullptr, nullptr, n, nullptr, 0);
    if (n && output < strings + n && strings < output + n)
        return fail(PSSGPU_EINVAL, "output overlaps the input array");
    return sort_pointer_array(strings, output, nullptr, nullptr, n, nullptr, 0);
}

static void die_on(int rc)
{
    if (rc) {
        fprintf(stderr, "pssgpu: sort failed (status %d): %s\n", rc, g_last_error.c_str());
        abort();
    }
}

void pssgpu_sort_strings(unsigned char** strings, size_t n)
{
    die_on(pssgpu_sort_strings_status(strings, nullptr, nullptr, n));
}

void pssgpu_sort_strings_lcp(unsigned char** strings, uintptr_t* lcp, size_t n)
{
    die_on(pssgpu_sort_strings_status(strings, lcp, nullptr, n));
}

void pssgpu_sort_strings_lcp_cache(uint8_t** strings, uintptr_t* lcp, uint8_t* cache, size_t n)
{
    die_on(pssgpu_sort_strings_status(strings, lcp, cache, n));
}

void pssgpu_sort_strings_out(unsigned char** strings, unsigned char** output, size_t n)
{
    die_on(pssgpu_sort_strings_out_status(strings, output, n));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// pssgpu_sort_device_noalloc sorts at most PSSGPU_NOALLOC_MAX_STRINGS strings
// with the small-segment kernel and allocates nothing. Its scratch -- the
// string-handle buffer, the one segment descriptor and the counters that
// kernel uses -- is the file-scope array below (16,528 bytes), which every
// device that loads this library holds until the process exits. In host code
// the array's name is only a host-side stand-in: kernels get the device
// address that cudaGetSymbolAddress returns, looked up once per device with
// that device current. Device code may name the array directly
// (k_noalloc_prep does).
namespace pssgpu {

struct NoAllocScratch {
    uint64_t hnd[PSSGPU_NOALLOC_MAX_STRINGS];
    Seg seg;
    uint32_t counters[C_COUNT];
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// One block: clear the counters (the array keeps the previous call's
// contents), write the initial handles and the single segment, check offsets.
__global__ void k_noalloc_prep(Work w)
{
    NoAllocScratch* s = reinterpret_cast<NoAllocScratch*>(g_noalloc_scratch);
    for (int i = threadIdx.x; i < C_COUNT; i += blockDim.x) s->counters[i] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < w.n; i += blockDim.x) {
        s->hnd[i] = h_make(w, i, w.offs[i]);
        if (w.offs[i] >= w.nchars) atomicOr(&s->counters[C_ERR], ERR_OFFSET);
    }
    if (threadIdx.x == 0) s->seg = Seg{0u, w.n, 0u, 0u};
}

constexpr int NOALLOC_MAX_DEVICES = 64;
static std::mutex g_noalloc_mu;
static NoAllocScratch* g_noalloc_addr[NOALLOC_MAX_DEVICES];

}  // namespace pssgpu

// Error messages of this entry point are at most 15 characters, so setting
// the thread's error string stays inside its inline buffer: failures do not
// allocate either.
extern "C" int pssgpu_sort_device_noalloc(const uint8_t* d_chars, uint64_t nchars,
                                          const uint64_t* d_offs, uint64_t n, uint32_t* d_perm,
                                          uint32_t* d_lcp, void* stream)
{
    if (n > PSSGPU_NOALLOC_MAX_STRINGS) return fail(PSSGPU_EINVAL, "n over max 2048");
    if (n == 0) return PSSGPU_OK;
    if (!d_chars || !d_offs || !d_perm) return fail(PSSGPU_EINVAL, "null buffer");
    if (nchars == 0) return fail(PSSGPU_EINVAL, "empty arena");
    if (((uintptr_t)d_chars & 7) != 0) return fail(PSSGPU_EINVAL, "unaligned arena");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return fail(PSSGPU_ENODEV, "no device");
    NoAllocScratch* scratch;
    {
        // set-up, once per device, with that device current
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
                return fail(PSSGPU_ECUDA, "symbol lookup");
            if (cudaFuncSetAttribute(K_BLOCK_NOALLOC, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(BlockSmem<2048>)) != cudaSuccess)
                return fail(PSSGPU_ECUDA, "smem limit");
            g_noalloc_addr[dev] = static_cast<NoAllocScratch*>(p);
        }
        scratch = g_noalloc_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint8_t last = 1;
    if (cudaMemcpyAsync(&last, d_chars + nchars - 1, 1, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(PSSGPU_ECUDA, "CUDA error");
    if (last != 0) return fail(PSSGPU_EINVAL, "no NUL at end");
    Work w{};
    w.chars = d_chars;
    w.nchars = nchars;
    w.offs = d_offs;
    w.n = (uint32_t)n;
    w.hnd[0] = w.hnd[1] = scratch->hnd;
    w.perm = d_perm;
    w.lcp = d_lcp;
    w.counters = scratch->counters;
    w.cur = 0;
    set_handle_format(w, false);
    k_noalloc_prep<<<1, SMALL_THREADS, 0, st>>>(w);
    K_BLOCK_NOALLOC<<<1, 256, sizeof(BlockSmem<2048>), st>>>(w, &scratch->seg);
    uint32_t err = 0;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(&err, scratch->counters + C_ERR, 4, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(PSSGPU_ECUDA, "CUDA error");
    if (err & ERR_OFFSET) return fail(PSSGPU_EINVAL, "bad offset");
    if (err) return fail(PSSGPU_ECUDA, "device error");
    return PSSGPU_OK;
}
