// gpu_contestant.cpp -- psstest contestants backed by libpssgpu.so.
//
// Compiled into the reference's psstest (with -DPSS_CONTEST=1, as its own
// contestants are, src/CMakeLists.txt:77-78) and linked against
// libpssgpu.so, this registers the B200 sorter under the Contest plugin API
// (src/tools/contest.hpp:146-179) with the three contestant signatures
// (contest.hpp:88-91), so `psstest -A gpu/sample_sort` selects it beside
// `-A bingmann/parallel_sample_sortBTCUI`. Registered as sequential
// contestants: the thread sweep of PSS_CONTESTANT_PARALLEL
// (src/psstest.cpp:716-779) would re-run the same device sort per thread
// count. Failures abort(), which psstest -F reports as status=aborted.
//
// psstest keeps every string inside its string data, g_string_data[0,
// g_string_datasize) (src/psstest.cpp:87-88, filled by
// src/tools/input.hpp:129-180); the reference's own contestants reach it the
// same way (src/sinha-copy-burstsort/glue.cpp:33-34). The contestants pass
// that buffer to pssgpu_sort_strings_arena, which then copies one span to the
// device instead of gathering every string on the host.
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "pssgpu.h"
#include "tools/contest.hpp"

extern const char* g_string_data;
extern size_t g_string_datasize;

namespace pss_b200 {

static void sort_in_arena(unsigned char** strings, unsigned char** output, uintptr_t* lcp,
                          uint8_t* cache, size_t n)
{
    const int rc = pssgpu_sort_strings_arena(reinterpret_cast<const uint8_t*>(g_string_data),
                                             g_string_datasize, strings, output, lcp, cache, n);
    if (rc) {
        std::fprintf(stderr, "pssgpu: sort failed (status %d): %s\n", rc, pssgpu_last_error());
        std::abort();
    }
}

static void gpu_sample_sort(unsigned char** strings, size_t n)
{
    sort_in_arena(strings, nullptr, nullptr, nullptr, n);
}

static void gpu_sample_sort_lcp(unsigned char** strings, uintptr_t* lcp, size_t n)
{
    sort_in_arena(strings, nullptr, lcp, nullptr, n);
}

static void gpu_sample_sort_lcp_cache(uint8_t** strings, uintptr_t* lcp, uint8_t* cache,
                                      size_t n)
{
    sort_in_arena(strings, nullptr, lcp, cache, n);
}

// The separate-output contestant, as parallel_sample_sortBTCUI_out
// (src/parallel/bingmann-parallel_sample_sort.cpp:44-62): sort into a new
// array, then copy it back for psstest's check.
static void gpu_sample_sort_out(unsigned char** strings, size_t n)
{
    unsigned char** output = new unsigned char*[n];
    sort_in_arena(strings, output, nullptr, nullptr, n);
    std::memcpy(strings, output, n * sizeof(unsigned char*));
    delete[] output;
}

PSS_CONTESTANT(gpu_sample_sort, "gpu/sample_sort",
               "B200 string sample sort (pS5 method, sm_100a kernels)")
PSS_CONTESTANT(gpu_sample_sort_lcp, "gpu/sample_sort_lcp",
               "B200 string sample sort with LCP output")
PSS_CONTESTANT(gpu_sample_sort_lcp_cache, "gpu/sample_sort_lcp_cache",
               "B200 string sample sort with LCP and distinguishing-char output")
PSS_CONTESTANT(gpu_sample_sort_out, "gpu/sample_sort_out",
               "B200 string sample sort, separate output")

}  // namespace pss_b200
