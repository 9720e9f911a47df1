"""CPU tests of the drop-in boundary: the C-ABI library loads without a GPU,
exports every function include/pssgpu.h declares, reports the absence of a
device as a status code, and the Python bindings cover the header."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "pssgpu.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(pssgpu_\w+)\s*\(", text))


def test_header_declares_contestant_signatures():
    names = declared_functions()
    for f in ("pssgpu_sort_strings", "pssgpu_sort_strings_lcp", "pssgpu_sort_strings_lcp_cache",
              "pssgpu_sort_host", "pssgpu_sort_device"):
        assert f in names


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg._native.gpu()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_bindings_cover_header(pkg):
    assert set(pkg._native.GPU_SIGNATURES) == declared_functions()


def test_version_string(pkg):
    assert b"sm_100a" in pkg._native.gpu().pssgpu_version()


def test_workspace_bytes_monotone(pkg):
    f = pkg._native.gpu().pssgpu_workspace_bytes
    assert 0 < f(1000) <= f(10**6) <= f(64 * 2**20)


def test_no_device_is_a_status_not_a_crash(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = pkg._native.gpu().pssgpu_ctx_create(0, C.byref(h))
    assert rc == 5  # PSSGPU_ENODEV
    assert b"device" in pkg._native.gpu().pssgpu_last_error()
    with pytest.raises(pkg.SortError):
        pkg.Context(0)


def test_build_tracks_every_cuda_source():
    """Every CUDA source of the package is a dependency of the library build,
    so that editing any of them rebuilds it."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "pss_build", ROOT / "parallel-string-sorting_b200" / "build.py")
    build = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(build)
    sources = {p.name for p in (ROOT / "parallel-string-sorting_b200" / "csrc").iterdir()
               if p.suffix in (".cu", ".cuh")}
    assert sources <= set(build.CUDA_DEPS)


def test_text_and_merge_arguments_checked_before_device_use(pkg):
    """The text and merge entry points refuse bad arguments with
    PSSGPU_EINVAL (and accept empty inputs) before they touch the context or
    any device buffer, so these checks run without a GPU. The context handle
    is a placeholder that the checked paths never dereference."""
    lib = pkg._native.gpu()
    fake = C.c_void_p(64)
    n = C.c_uint64(99)
    assert lib.pssgpu_prepare_text_device(None, None, 5, 0, None, 0, C.byref(n), None) == 1
    assert lib.pssgpu_prepare_text_device(fake, None, 5, 7, None, 0, C.byref(n), None) == 1
    assert lib.pssgpu_prepare_text_device(fake, None, 0, 0, None, 0, C.byref(n), None) == 0
    assert n.value == 0
    assert lib.pssgpu_prepare_text_device(fake, None, 5, 0, None, 9, C.byref(n), None) == 1
    assert lib.pssgpu_prepare_text_device(fake, 9, 5, 0, 64, 9, C.byref(n), None) == 1  # unaligned
    assert b"aligned" in lib.pssgpu_last_error()
    assert lib.pssgpu_sort_text_host(fake, None, 5, 2, None, None, 0, C.byref(n)) == 1
    assert lib.pssgpu_sort_text_host(fake, None, 0, 0, None, None, 0, C.byref(n)) == 0
    assert lib.pssgpu_sort_text_host(fake, None, 5, 0, None, None, 5, C.byref(n)) == 1

    def runs(*b):
        return (C.c_uint64 * len(b))(*b)
    merge = lib.pssgpu_merge_lcp_device
    assert merge(fake, 64, 10, 64, runs(0), 0, 64, 64, 64, 64, None) == 1           # no runs
    assert merge(fake, 64, 10, 64, runs(1, 2), 1, 64, 64, 64, 64, None) == 1        # not from 0
    assert merge(fake, 64, 10, 64, runs(0, 5, 3), 2, 64, 64, 64, 64, None) == 1     # decreasing
    assert merge(fake, 64, 0, 64, runs(0, 5), 1, 64, 64, 64, 64, None) == 1         # empty arena
    assert merge(fake, None, 10, 64, runs(0, 5), 1, 64, 64, 64, 64, None) == 1      # null arena
    assert merge(fake, 64, 10, 64, runs(0, 5), 1, 64, None, 64, 64, None) == 1      # LCP out, none in
    assert merge(fake, 68, 10, 64, runs(0, 5), 1, 64, 64, 64, 64, None) == 1        # unaligned arena
    assert merge(fake, 64, 10, 64, runs(0, 0, 0), 2, None, None, None, None, None) == 0  # nothing to merge
