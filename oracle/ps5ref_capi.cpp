/*
 * oracle/ps5ref_capi.cpp -- TEST INFRASTRUCTURE, not part of the product.
 *
 * A thin C ABI over the reference's own pS5 engine, compiled from the
 * reference sources where they lie (see oracle/Makefile) into
 * oracle/_ref/libps5ref.so. Only tests/, the smoke check and bench.py's CPU
 * baseline leg load it, as the checker or as the timed reference; the GPU
 * product never links it.
 *
 * Every function below calls the reference code path unchanged:
 *   ps5ref_sort       -> parallel_sample_sortBTCUI
 *                        (src/parallel/bingmann-parallel_sample_sort.cpp:31-37)
 *   ps5ref_sort_lcp   -> parallel_sample_sort_lcp_base<ClassifyTreeUnrollInterleaveX>
 *                        (src/parallel/bingmann-parallel_sample_sort.hpp:1733-1748)
 *   ps5ref_get_uint64 -> StringSetBase::get_uint64 / get_char_uint64_simple
 *                        (src/tools/stringset.hpp:201-231, 251-255)
 *   ps5ref_find_bkt   -> ClassifyTreeSimple::find_bkt
 *                        (src/sequential/bingmann-sample_sortBTC.hpp:45-72)
 *   ps5ref_verify_lcp -> stringtools::verify_lcp (src/tools/stringptr.hpp:1035-1046)
 */
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

#include "parallel/bingmann-parallel_sample_sort.hpp"

size_t g_small_sort = 0;

namespace bingmann_parallel_sample_sort {

extern "C" {

int ps5ref_set_threads(int threads)
{
    if (threads > 0) omp_set_num_threads(threads);
    return omp_get_max_threads();
}

void ps5ref_sort(unsigned char** strings, size_t n)
{
    parallel_sample_sort_base<
        bingmann_sample_sort::ClassifyTreeUnrollInterleaveX>(
        UCharStringSet(strings, strings + n), 0);
}

void ps5ref_sort_lcp(unsigned char** strings, uintptr_t* lcp, size_t n)
{
    parallel_sample_sort_lcp_base<
        bingmann_sample_sort::ClassifyTreeUnrollInterleaveX>(
        UCharStringSet(strings, strings + n), lcp, 0);
}

uint64_t ps5ref_get_uint64(const unsigned char* s, size_t depth)
{
    unsigned char* p = const_cast<unsigned char*>(s);
    UCharStringSet ss(&p, &p + 1);
    return ss.get_uint64(p, depth);
}

static void fill_levelorder(const uint64_t* sorted, size_t lo, size_t hi,
                            size_t node, uint64_t* tree)
{
    if (lo >= hi) return;
    size_t mid = lo + (hi - lo) / 2;
    tree[node] = sorted[mid];
    fill_levelorder(sorted, lo, mid, 2 * node, tree);
    fill_levelorder(sorted, mid + 1, hi, 2 * node + 1, tree);
}

/* Classify keys with the reference's 1023-splitter tree given 1023 sorted
 * splitters; bucket ids in [0, 2046]. */
void ps5ref_find_bkt(const uint64_t* sorted_splitters, const uint64_t* keys,
                     size_t n, uint16_t* out)
{
    typedef bingmann_sample_sort::ClassifyTreeSimple<10> Classify;
    Classify* c = new Classify;
    for (size_t i = 0; i < Classify::numsplitters; ++i)
        c->splitter[i] = sorted_splitters[i];
    fill_levelorder(sorted_splitters, 0, Classify::numsplitters, 1,
                    c->splitter_tree);
    for (size_t i = 0; i < n; ++i) out[i] = (uint16_t)c->find_bkt(keys[i]);
    delete c;
}

int ps5ref_verify_lcp(unsigned char** strings, const uintptr_t* lcp, size_t n,
                      uintptr_t expected_first)
{
    return stringtools::verify_lcp(strings, lcp, n, expected_first) ? 1 : 0;
}

} // extern "C"

} // namespace bingmann_parallel_sample_sort
