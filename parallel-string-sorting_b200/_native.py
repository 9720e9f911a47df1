"""ctypes bindings of libpssgpu.so (the C ABI declared in include/pssgpu.h)
and of libpsswork.so (seeded workloads, algorithmic-byte model).

Loading fails loudly when a library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"

PSSGPU_OK = 0
STATUS_NAMES = {
    0: "PSSGPU_OK", 1: "PSSGPU_EINVAL", 2: "PSSGPU_ENOMEM", 3: "PSSGPU_ECUDA",
    4: "PSSGPU_ETIMEOUT", 5: "PSSGPU_ENODEV", 6: "PSSGPU_EBUDGET",
}

# Every symbol include/pssgpu.h declares, with its ctypes signature.
GPU_SIGNATURES = {
    "pssgpu_last_error": (C.c_char_p, []),
    "pssgpu_version": (C.c_char_p, []),
    "pssgpu_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "pssgpu_ctx_destroy": (None, [C.c_void_p]),
    "pssgpu_workspace_bytes": (C.c_uint64, [C.c_uint64]),
    "pssgpu_ctx_stats": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pssgpu_ctx_set_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "pssgpu_ctx_kernel_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "pssgpu_ctx_set_option": (C.c_int, [C.c_void_p, C.c_int, C.c_int64]),
    "pssgpu_sort_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                   C.c_void_p, C.c_void_p]),
    "pssgpu_sort_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    "pssgpu_prepare_text_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int,
                                             C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
                                             C.c_void_p]),
    "pssgpu_sort_text_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_void_p,
                                        C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "pssgpu_merge_lcp_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                          C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]),
    "pssgpu_sort_batch_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                         C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "pssgpu_sort_batch_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                           C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                           C.c_void_p]),
    "pssgpu_ctx_set_tree_bits": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "pssgpu_server_create": (C.c_int, [C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "pssgpu_server_destroy": (None, [C.c_void_p]),
    "pssgpu_server_submit": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                       C.c_uint64, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_uint64)]),
    "pssgpu_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    "pssgpu_server_get_stats": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pssgpu_sort_strings": (None, [C.c_void_p, C.c_size_t]),
    "pssgpu_sort_strings_lcp": (None, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "pssgpu_sort_strings_lcp_cache": (None, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]),
    "pssgpu_sort_strings_status": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]),
    "pssgpu_sort_strings_out": (None, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "pssgpu_sort_strings_out_status": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "pssgpu_sort_strings_arena": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_size_t]),
    "pssgpu_sort_device_noalloc": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                             C.c_void_p, C.c_void_p, C.c_void_p]),
}

WORK_SIGNATURES = {
    "pssw_random_offsets": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_void_p]),
    "pssw_random_fill": (None, [C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p,
                                C.c_uint32, C.c_void_p]),
    "pssw_digits_count": (C.c_uint64, [C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]),
    "pssw_digits_fill": (None, [C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p]),
    "pssw_prefix_offsets": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_void_p]),
    "pssw_prefix_fill": (None, [C.c_uint64, C.c_uint64, C.c_void_p, C.c_double, C.c_void_p,
                                C.c_void_p]),
    "pssw_dna_text": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_double, C.c_void_p]),
    "pssw_lognormal_offsets": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_double, C.c_double,
                                            C.c_uint32, C.c_uint32, C.c_void_p]),
    "pssw_alg_bytes": (None, [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(C.c_uint64),
                              C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                              C.POINTER(C.c_uint32)]),
    "pssw_check_sorted": (C.c_int64, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                      C.c_uint64]),
    "pssw_check_permutation": (C.c_int, [C.c_void_p, C.c_uint64]),
}


class PssStats(C.Structure):
    _fields_ = [
        ("passes", C.c_uint32),
        ("kernel_launches", C.c_uint32),
        ("big_elements", C.c_uint64),
        ("small_segments", C.c_uint64),
        ("boundaries", C.c_uint64),
        ("device_ms", C.c_float),
    ]


class PssKernelStats(C.Structure):
    _fields_ = [
        ("name", C.c_char * 16),
        ("launches", C.c_uint32),
        ("strings", C.c_uint64),
        ("alg_bytes", C.c_uint64),
        ("ms", C.c_double),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("hbm_budget", C.c_uint64),
        ("max_batch_strings", C.c_uint64),
        ("workers", C.c_uint32),
        ("max_batch_requests", C.c_uint32),
    ]


class RequestInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int),
        ("batch_requests", C.c_uint32),
        ("batch_strings", C.c_uint64),
        ("t_submit_ns", C.c_uint64),
        ("t_admit_ns", C.c_uint64),
        ("t_start_ns", C.c_uint64),
        ("t_done_ns", C.c_uint64),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("slab_bytes", C.c_uint64),
        ("slab_peak_bytes", C.c_uint64),
        ("batches", C.c_uint64),
        ("batched_requests", C.c_uint64),
        ("pending", C.c_uint64),
        ("ready", C.c_uint64),
    ]


def _load(name: str, sigs: dict) -> C.CDLL:
    path = LIB_DIR / name
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build the native libraries first "
            "(python -c 'import __graft_entry__ as g; g.build()')")
    lib = C.CDLL(str(path))
    for sym, (res, args) in sigs.items():
        fn = getattr(lib, sym)
        fn.restype = res
        fn.argtypes = args
    return lib


_gpu = None
_work = None


def gpu() -> C.CDLL:
    global _gpu
    if _gpu is None:
        _gpu = _load("libpssgpu.so", GPU_SIGNATURES)
    return _gpu


def work() -> C.CDLL:
    global _work
    if _work is None:
        _work = _load("libpsswork.so", WORK_SIGNATURES)
    return _work
