// work.cuh -- the device-side state of one sort, passed by value to kernels.
#pragma once

#include "device_common.cuh"

namespace pssgpu {

constexpr int TILE = 4096;          // strings per classify / scatter tile
constexpr int TILE_THREADS = 256;   // 16 strings per thread
constexpr int MAX_TREE_BITS = 10;   // 1023 splitters, 2047 buckets (pS5's DefaultTreebits)
constexpr int MAX_BKT = 2048;       // bucket slots per big segment
constexpr int SMALL_MAX = 2048;     // largest segment the small-sort kernel takes
constexpr int SMALL_THREADS = 256;
constexpr int WARP_GROUP_MAX = 32;  // groups this small are finished by one warp
constexpr int FINAL_INLINE = 64;    // equal-string buckets this small are copied inline
constexpr uint32_t SPIN_CAP = 1u << 20;  // look-back wait limit (polls, ~0.1 s)

// counters[] layout
enum : int {
    C_NBIG = 0,       // + 3 * parity
    C_NSMALL = 1,     // + 3 * parity
    C_NTILES = 2,     // + 3 * parity
    C_NBND = 6,       // boundary list length
    C_TICKET = 7,     // scatter tile ticket
    C_ERR = 8,        // error bits
    C_SMALLSEGS = 9,  // statistics: segments finished by the small sorter
    // per-pass statistics, reset every pass
    C_P_BIG = 10,      // strings in big sample-sort segments
    C_P_STALE = 11,    // of those, strings whose key was gathered this pass
    C_P_FINAL = 12,    // strings copied out of big all-equal segments
    C_P_SCATTER = 13,  // strings moved by the scatter
    C_P_SMALL = 14,    // strings finished by the small sorter
    C_COUNT = 16
};

struct Work {
    // input arena
    const uint8_t* chars;
    uint64_t nchars;
    const uint64_t* offs;
    uint32_t n;
    // permutation / key ping-pong
    uint32_t* ids[2];
    uint64_t* keys[2];
    uint16_t* bkt;
    // outputs
    uint32_t* perm;
    uint32_t* lcp;  // may be null
    // bookkeeping
    uint32_t* counters;
    uint2* bnd;  // (position, depth) of split boundaries
    uint32_t bnd_cap;
    // segment lists, double-buffered by pass parity
    Seg* big[2];
    Seg* small[2];
    uint32_t big_cap, small_cap;
    // per big segment of the current pass
    uint32_t* tile_start;  // [big_cap + 1]
    uint8_t* tree_bits;    // [big_cap]
    uint64_t* tree;        // [big_cap][1024], level order, index 1..k
    uint64_t* spl;         // [big_cap][1024], sorted splitters
    uint32_t* bcount;      // [big_cap][MAX_BKT]
    uint32_t* bstart;      // [big_cap][MAX_BKT]
    uint8_t* bflags;       // [big_cap]: 1 = whole segment in one bucket
    uint64_t* status;      // [tile_cap][MAX_BKT] decoupled look-back words
    uint32_t tile_cap;
    uint32_t epoch;        // look-back epoch of this pass (1..65535)
    int cur;               // parity of the lists read in this pass
};

}  // namespace pssgpu
