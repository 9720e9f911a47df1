// work.cuh -- the device-side state of one sort, passed by value to kernels.
#pragma once

#include "device_common.cuh"

namespace pssgpu {

constexpr int TILE = 8192;          // strings per classify / scatter tile
constexpr int TILE_THREADS = 512;   // 16 strings per thread
constexpr int MAX_TREE_BITS = 10;   // 1023 splitters, 2047 buckets (pS5's DefaultTreebits)
constexpr int MAX_BKT = 2056;       // bucket slots per big segment: 2047 + the two prefix buckets
constexpr int JMAX_CHUNKS = 32;     // common-prefix jump of one pass: at most 32 8-byte chunks
constexpr int SMALL_MAX = 1024;     // largest segment the block sorters take
constexpr int SMALL_THREADS = 256;
constexpr int WARP_GROUP_MAX = 32;  // groups this small are finished by one warp
constexpr int FINAL_INLINE = 64;    // equal-string buckets this small are copied inline
constexpr int CHUNK = 32;           // tiles per chunk of the destination scan
constexpr uint32_t DBL_MAX = 4096;  // largest group a suffix sort hands to rank doubling

// segment list classes
enum : int { L_BIG = 0, L_TINY = 1, L_SMALLA = 2, L_SMALLB = 3, L_NCLASS = 4 };

// counters[] layout
enum : int {
    C_PAR = 8,        // counters per parity block: [class] lengths, then tiles
    C_NTILES = 4,     // + C_PAR * parity: tiles of the big list
    C_NSTR = 4,       // + C_PAR * parity + class (1..3): strings in the small lists
    C_NBND = 16,      // boundary list length
    C_SPARE = 17,
    C_ERR = 18,       // error bits
    C_SMALLSEGS = 19, // statistics: segments finished by the block sorter
    // per-pass statistics, reset every pass
    C_P_BIG = 20,     // strings in big sample-sort segments
    C_P_STALE = 21,   // of those, strings whose key was gathered this pass
    C_P_FINAL = 22,   // strings copied out of big all-equal segments
    C_P_SCATTER = 23, // strings moved by the scatter
    C_P_TIE = 24,     // of the big strings, those classified behind a common-prefix jump
    C_P_JCHUNKS = 25, // their prefix chunks: sum over jump segments of size * jump / 8
    C_P_FIRST = C_P_BIG,
    C_P_LAST = C_P_JCHUNKS,
    C_MULTI = 26,     // + parity: big segments of more than CHUNK tiles in the list
    C_DEEP = 28,      // + parity: length of the deep-group list
    C_SFX = 30,       // suffix-set check: nonzero when the input is not all suffixes of a text
    C_DBL = 31,       // groups handed to rank doubling by the passes
    C_DBL_CNT = 32,   // + 3 * parity + class: rank-doubling round lists
    C_DBL_MEMB = 38,  // 64-bit (38, 39): members of the rank-doubling groups, summed over rounds
    C_COUNT = 40
};

struct Work {
    // input arena
    const uint8_t* chars;
    uint64_t nchars;
    const uint64_t* offs;
    uint32_t n;
    // String handles: (id << hbits) | arena offset when both fit in 64 bits
    // (packed), else the id alone and the offset is read from offs[id].
    // Carrying the offset saves the dependent offs[id] load of every gather.
    uint32_t hbits;
    uint64_t hmask;
    int packed;
    // handle / key ping-pong
    uint64_t* hnd[2];
    uint64_t* keys[2];
    uint16_t* bkt;
    // outputs
    uint32_t* perm;
    uint32_t* lcp;  // may be null
    // bookkeeping
    uint32_t* counters;
    uint2* bnd;  // (position, depth) of split boundaries
    uint32_t bnd_cap;
    // segment lists per class, double-buffered by pass parity
    Seg* list[L_NCLASS][2];
    uint32_t cap[L_NCLASS];
    // per big segment of the current pass
    uint32_t* tile_start;  // [cap[L_BIG] + 1]
    uint8_t* tree_bits;    // [cap[L_BIG]]; 0 = all-equal copy
    uint64_t* tree;        // [cap[L_BIG]][1024], level order, index 1..k
    uint64_t* spl;         // [cap[L_BIG]][1024], sorted splitters
    uint32_t* bcount;      // [cap[L_BIG]][MAX_BKT]
    uint32_t* bstart;      // [cap[L_BIG]][MAX_BKT]
    uint8_t* bflags;       // [cap[L_BIG]]: 1 = whole segment in one bucket
    // Common-prefix jump: when every sample shares more chars beyond the
    // segment depth, jump[s] = that many chars (a multiple of 8) and jpre holds
    // them as keys; the tree then splits at depth + jump, and strings that
    // leave the prefix earlier go to a first ('<' prefix) or last ('>' prefix)
    // bucket.
    uint32_t* jump;        // [cap[L_BIG]]
    uint64_t* jpre;        // [cap[L_BIG]][JMAX_CHUNKS]
    // Scatter destinations, pS5's count / count_finished over parts (hpp:1414-1460)
    // with tiles as parts: per tile and bucket the count, then (after the
    // bucket-major, tile-minor exclusive scan) the tile's first destination.
    // The scan runs in chunks of CHUNK tiles.
    uint32_t* chunk_start;  // [cap[L_BIG] + 1]: first chunk of each big segment
    uint32_t* tcount;       // [tile_cap][MAX_BKT]
    uint32_t* ccount;       // [tile_cap][MAX_BKT]: chunk sums, then chunk bases
    uint32_t tile_cap;
    int cur;               // parity of the lists read in this pass
    // Deep groups: groups of at most 32 strings that a block sorter's warp
    // window found stuck on a long common prefix, handed to k_deep (one warp
    // each) in the next pass; double-buffered by pass parity, null when not
    // allocated
    Seg* deep[2];
    uint32_t deep_cap;
    // splitter-tree levels for a big segment of 2^k..2^(k+1)-1 strings
    // (0: the default rule), set from a tuning table
    uint8_t tree_bits_by_size[33];
    // Suffix sets (every string is a suffix of one text: offs[i] = i, no NUL
    // before the last char): '=' groups of at most DBL_MAX strings below
    // depth 8 go to the rank-doubling list instead of deeper passes.
    int suffix;
    Seg* dbl;
    uint32_t dbl_cap;
};

// buckets of a classified big segment: the tree's 2^(L+1) - 1, plus the two
// prefix buckets of a jump segment
__device__ __forceinline__ uint32_t seg_buckets(const Work& w, int s)
{
    return (2u << w.tree_bits[s]) - 1 + (w.jump[s] ? 2u : 0u);
}

__device__ __forceinline__ uint64_t h_make(const Work& w, uint32_t id, uint64_t off)
{
    return w.packed ? (((uint64_t)id << w.hbits) | off) : (uint64_t)id;
}

__device__ __forceinline__ uint32_t h_id(const Work& w, uint64_t h)
{
    return w.packed ? (uint32_t)(h >> w.hbits) : (uint32_t)h;
}

__device__ __forceinline__ uint64_t h_off(const Work& w, uint64_t h)
{
    return w.packed ? (h & w.hmask) : __ldg(w.offs + h);
}

// key of the string behind handle h at depth d
__device__ __forceinline__ uint64_t h_key(const Work& w, uint64_t h, uint32_t d)
{
    return load_key(w.chars, w.nchars, h_off(w, h) + d);
}

}  // namespace pssgpu
