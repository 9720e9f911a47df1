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
