/*
 * oracle/pss_oracle.c -- TEST INFRASTRUCTURE, not part of the product.
 *
 * Plain-C restatement of the pS5 path of bingmann/parallel-string-sorting as
 * it runs below the sequential threshold: multikey quicksort on 8-byte
 * character caches with the LCP computed from key XORs, and an insertion-sort
 * base case. Used only as a checker (tests/, the smoke check, the CPU-baseline
 * leg of bench.py). Each function cites the reference lines it restates; the
 * file shares no code with the reference.
 */
#include "pss_oracle.h"

#include <stdlib.h>
#include <string.h>

/* get_char_uint64_simple (src/tools/stringset.hpp:201-231) via get_uint64
 * (stringset.hpp:251-255): up to 8 chars packed big-endian, stopping at the
 * terminating NUL (UCharStringSet::is_end is *i == 0). */
uint64_t pso_get_uint64(const uint8_t* s, size_t depth)
{
    const uint8_t* p = s + depth;
    uint64_t v = 0;
    for (int k = 0; k < 8; ++k) {
        if (p[k] == 0) return v;
        v |= (uint64_t)p[k] << (56 - 8 * k);
    }
    return v;
}

/* lcpKeyType (src/parallel/bingmann-parallel_sample_sort.hpp:225-230). */
unsigned pso_lcp_key_type(uint64_t a, uint64_t b)
{
    uint64_t x = a ^ b;
    return x ? (unsigned)(__builtin_clzll(x) / 8) : 8u;
}

/* lcpKeyDepth (bingmann-parallel_sample_sort.hpp:232-237). */
unsigned pso_lcp_key_depth(uint64_t a)
{
    return a ? 8u - (unsigned)(__builtin_ctzll(a) / 8) : 0u;
}

/* ------------------------------------------------------------------------ */

typedef struct {
    const uint8_t* chars;
    const uint64_t* offs;
} sset;

static inline const uint8_t* sptr(const sset* ss, uint32_t id)
{
    return ss->chars + ss->offs[id];
}

/* calc_lcp from depth on: chars shared beyond the common prefix `depth`. */
static size_t lcp_from(const sset* ss, uint32_t a, uint32_t b, size_t depth)
{
    const uint8_t* x = sptr(ss, a);
    const uint8_t* y = sptr(ss, b);
    size_t h = depth;
    while (x[h] != 0 && x[h] == y[h]) ++h;
    return h;
}

static int cmp_from(const sset* ss, uint32_t a, uint32_t b, size_t depth)
{
    const uint8_t* x = sptr(ss, a) + depth;
    const uint8_t* y = sptr(ss, b) + depth;
    while (*x != 0 && *x == *y) { ++x; ++y; }
    return (int)*x - (int)*y;
}

/* inssort_generic (src/sequential/inssort.hpp:63-95): insertion sort of
 * strings sharing `depth` chars, comparing characters from depth on; the LCPs
 * inside the range are written afterwards (lcp_insertion_sort emits the same
 * values, src/sequential/bingmann-lcp_inssort.hpp:38-189). */
static void inssort_generic(const sset* ss, uint32_t* ids, size_t n,
                            size_t depth, uint64_t* lcp)
{
    for (size_t j = 1; j < n; ++j) {
        uint32_t t = ids[j];
        size_t i = j;
        while (i > 0 && cmp_from(ss, ids[i - 1], t, depth) > 0) {
            ids[i] = ids[i - 1];
            --i;
        }
        ids[i] = t;
    }
    if (lcp)
        for (size_t j = 1; j < n; ++j)
            lcp[j] = lcp_from(ss, ids[j - 1], ids[j], depth);
}

static inline void swap2(uint32_t* ids, uint64_t* cache, size_t a, size_t b)
{
    uint32_t t = ids[a]; ids[a] = ids[b]; ids[b] = t;
    uint64_t c = cache[a]; cache[a] = cache[b]; cache[b] = c;
}

/* insertion_sort_cache (bingmann-parallel_sample_sort.hpp:805-861): sort by
 * cached key, then groups of equal keys either are finished (key holds the
 * NUL: all strings equal, LCP = depth + lcpKeyDepth) or are sorted deeper by
 * characters from depth + 8. */
static void inssort_cache(const sset* ss, uint32_t* ids, uint64_t* cache,
                          size_t n, size_t depth, uint64_t* lcp)
{
    for (size_t j = 1; j < n; ++j) {
        uint32_t ti = ids[j];
        uint64_t tc = cache[j];
        size_t i = j;
        while (i > 0 && cache[i - 1] > tc) {
            ids[i] = ids[i - 1];
            cache[i] = cache[i - 1];
            --i;
        }
        ids[i] = ti;
        cache[i] = tc;
    }
    size_t start = 0;
    for (size_t i = 1; i <= n; ++i) {
        if (i < n && cache[i] == cache[start]) continue;
        size_t len = i - start;
        if (start != 0 && lcp)
            lcp[start] = depth + pso_lcp_key_type(cache[start - 1], cache[start]);
        if (len > 1) {
            if (cache[start] & 0xFF) {
                inssort_generic(ss, ids + start, len, depth + 8,
                                lcp ? lcp + start : NULL);
            } else if (lcp) {
                uint64_t v = depth + pso_lcp_key_depth(cache[start]);
                for (size_t k = start + 1; k < i; ++k) lcp[k] = v;
            }
        }
        start = i;
    }
}

static size_t med3(const uint64_t* c, size_t a, size_t b, size_t d)
{
    /* med3 (bingmann-parallel_sample_sort.hpp:767-781) */
    if (c[a] == c[b]) return a;
    if (c[d] == c[a] || c[d] == c[b]) return d;
    if (c[a] < c[b]) {
        if (c[b] < c[d]) return b;
        return (c[a] < c[d]) ? d : a;
    }
    if (c[b] > c[d]) return b;
    return (c[a] < c[d]) ? a : d;
}

/* MKQSStep + sort_mkqs_cache (bingmann-parallel_sample_sort.hpp:863-1178):
 * ternary partition on 8-byte caches around a median-of-9 pivot. The '<' and
 * '>' parts recurse at the same depth with valid caches; the '=' part
 * recurses at depth + 8 only when the pivot holds no NUL (hpp:984). The LCPs
 * at the part boundaries come from max_lt / min_gt (hpp:986-1008). */
static void mkqs(const sset* ss, uint32_t* ids, uint64_t* cache, size_t n,
                 size_t depth, int dirty, uint64_t* lcp)
{
    while (1) {
        if (dirty)
            for (size_t i = 0; i < n; ++i)
                cache[i] = pso_get_uint64(sptr(ss, ids[i]), depth);
        if (n < 32) {  /* g_inssort_threshold (hpp:104) */
            inssort_cache(ss, ids, cache, n, depth, lcp);
            return;
        }
        size_t p = med3(cache,
                        med3(cache, 0, n / 8, n / 4),
                        med3(cache, n / 2 - n / 8, n / 2, n / 2 + n / 8),
                        med3(cache, n - 1 - n / 4, n - 1 - n / 8, n - 3));
        uint64_t pivot = cache[p];
        /* three-way partition [< | = | >] */
        size_t lt = 0, i = 0, gt = n;
        uint64_t max_lt = 0, min_gt = ~(uint64_t)0;
        while (i < gt) {
            uint64_t c = cache[i];
            if (c < pivot) {
                if (c > max_lt) max_lt = c;
                swap2(ids, cache, lt++, i++);
            } else if (c > pivot) {
                if (c < min_gt) min_gt = c;
                swap2(ids, cache, i, --gt);
            } else {
                ++i;
            }
        }
        size_t num_lt = lt, num_eq = gt - lt, num_gt = n - gt;
        if (lcp) {
            if (num_lt > 0) lcp[lt] = depth + pso_lcp_key_type(max_lt, pivot);
            if (num_gt > 0) lcp[gt] = depth + pso_lcp_key_type(pivot, min_gt);
        }
        if (num_lt > 1) mkqs(ss, ids, cache, num_lt, depth, 0, lcp);
        if (num_gt > 1)
            mkqs(ss, ids + gt, cache + gt, num_gt, depth, 0, lcp ? lcp + gt : NULL);
        if (num_eq <= 1) return;
        if (!(pivot & 0xFF)) {
            if (lcp) {
                uint64_t v = depth + pso_lcp_key_depth(pivot);
                for (size_t k = lt + 1; k < gt; ++k) lcp[k] = v;
            }
            return;
        }
        /* iterate on the '=' part at depth + 8 */
        ids += lt;
        cache += lt;
        if (lcp) lcp += lt;
        n = num_eq;
        depth += 8;
        dirty = 1;
    }
}

void pso_sort_lcp(const uint8_t* chars, const uint64_t* offs, uint32_t* ids,
                  size_t n, uint64_t* lcp)
{
    if (n <= 1) return;
    sset ss = { chars, offs };
    uint64_t* cache = (uint64_t*)malloc(n * sizeof(uint64_t));
    if (!cache) abort();
    mkqs(&ss, ids, cache, n, 0, 1, lcp);
    free(cache);
}

/* ClassifyTreeSimple::find_bkt (src/sequential/bingmann-sample_sortBTC.hpp:
 * 45-72) restated as a lower-bound search on the sorted splitters. */
void pso_classify(const uint64_t* splitters, size_t k, const uint64_t* keys,
                  size_t n, uint16_t* out)
{
    for (size_t i = 0; i < n; ++i) {
        uint64_t key = keys[i];
        size_t lo = 0, hi = k;
        while (lo < hi) {
            size_t mid = lo + (hi - lo) / 2;
            if (splitters[mid] < key) lo = mid + 1; else hi = mid;
        }
        size_t b = 2 * lo;
        if (lo < k && splitters[lo] == key) b += 1;
        out[i] = (uint16_t)b;
    }
}

/* ------------------------------------------------------------------------ */
/* Checkers: check_sorted_order (src/tools/checker.hpp:131-153), verify_lcp
 * (src/tools/stringptr.hpp:977-1046), calc_distinguishing_prefix
 * (checker.hpp:155-180). */

int64_t pso_check_order(const uint8_t* chars, const uint64_t* offs,
                        const uint32_t* ids, size_t n)
{
    sset ss = { chars, offs };
    int64_t first = INT64_MAX;
#pragma omp parallel for schedule(static) reduction(min : first)
    for (size_t i = 1; i < n; ++i)
        if (cmp_from(&ss, ids[i - 1], ids[i], 0) > 0 && (int64_t)i < first)
            first = (int64_t)i;
    return first == INT64_MAX ? -1 : first;
}

int pso_check_permutation(const uint32_t* ids, size_t n)
{
    uint8_t* seen = (uint8_t*)calloc(n ? n : 1, 1);
    if (!seen) abort();
    int ok = 1;
    for (size_t i = 0; i < n && ok; ++i) {
        if (ids[i] >= n || seen[ids[i]]) ok = 0;
        else seen[ids[i]] = 1;
    }
    free(seen);
    return ok;
}

void pso_lcp_array(const uint8_t* chars, const uint64_t* offs,
                   const uint32_t* ids, size_t n, uint64_t* lcp)
{
    sset ss = { chars, offs };
#pragma omp parallel for schedule(static)
    for (size_t i = 1; i < n; ++i)
        lcp[i] = lcp_from(&ss, ids[i - 1], ids[i], 0);
}

int64_t pso_check_lcp32(const uint8_t* chars, const uint64_t* offs,
                        const uint32_t* ids, size_t n, const uint32_t* lcp)
{
    sset ss = { chars, offs };
    int64_t first = INT64_MAX;
#pragma omp parallel for schedule(static) reduction(min : first)
    for (size_t i = 1; i < n; ++i)
        if ((uint64_t)lcp[i] != (uint64_t)lcp_from(&ss, ids[i - 1], ids[i], 0) &&
            (int64_t)i < first)
            first = (int64_t)i;
    return first == INT64_MAX ? -1 : first;
}

uint64_t pso_dprefix(const uint8_t* chars, const uint64_t* offs,
                     const uint32_t* ids, size_t n, uint64_t* lcpsum)
{
    sset ss = { chars, offs };
    uint64_t D = 0, sum = 0, pdepth = 0;
    for (size_t i = 1; i < n; ++i) {
        uint64_t depth = lcp_from(&ss, ids[i - 1], ids[i], 0);
        sum += depth;
        depth++;
        if (pdepth < depth) D += depth - pdepth;
        D += depth;
        pdepth = depth;
    }
    if (lcpsum) *lcpsum = sum;
    return D;
}
