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
#include <cstddef>
#include <cstdint>

#include "pssgpu.h"
#include "tools/contest.hpp"

namespace pss_b200 {

static void gpu_sample_sort(unsigned char** strings, size_t n)
{
    pssgpu_sort_strings(strings, n);
}

static void gpu_sample_sort_lcp(unsigned char** strings, uintptr_t* lcp, size_t n)
{
    pssgpu_sort_strings_lcp(strings, lcp, n);
}

static void gpu_sample_sort_lcp_cache(uint8_t** strings, uintptr_t* lcp, uint8_t* cache,
                                      size_t n)
{
    pssgpu_sort_strings_lcp_cache(strings, lcp, cache, n);
}

PSS_CONTESTANT(gpu_sample_sort, "gpu/sample_sort",
               "B200 string sample sort (pS5 method, sm_100a kernels)")
PSS_CONTESTANT(gpu_sample_sort_lcp, "gpu/sample_sort_lcp",
               "B200 string sample sort with LCP output")
PSS_CONTESTANT(gpu_sample_sort_lcp_cache, "gpu/sample_sort_lcp_cache",
               "B200 string sample sort with LCP and distinguishing-char output")

}  // namespace pss_b200
