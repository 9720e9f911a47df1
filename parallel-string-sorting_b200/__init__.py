"""B200-native string sample sort: a drop-in for pS5 of
bingmann/parallel-string-sorting behind psstest's Contest API.

The product is the C ABI library ``lib/libpssgpu.so`` (include/pssgpu.h,
sm_100a kernels in ``csrc/``); this package is its Python host API.
"""
from .api import (Context, SortError, default_context, pack_strings, parallel_sample_sort,
                  parallel_sample_sort_lcp, sort_pointer_array, sort_pointer_array_arena,
                  sort_pointer_array_out)
from . import workloads

__all__ = ["Context", "SortError", "default_context", "pack_strings", "parallel_sample_sort",
           "parallel_sample_sort_lcp", "sort_pointer_array", "sort_pointer_array_arena",
           "sort_pointer_array_out", "workloads"]
