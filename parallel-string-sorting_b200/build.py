"""Native build of the package: the sm_100a CUDA library and the host
workload library, compiled in-tree into ``lib/`` so they travel with the
repository snapshot.

``build_all()`` is what ``__graft_entry__.build()`` runs; ``python build.py``
does the same from the command line.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
INCLUDE = PKG.parent / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = ["pssgpu.cu"]
CUDA_DEPS = ["device_common.cuh", "work.cuh", "block_util.cuh", "kernels_big.cuh",
             "kernels_small.cuh", "kernels_block.cuh", "kernels_wave.cuh", "kernels_suffix.cuh",
             "server.cuh", "prepare.cuh",
             "merge.cuh",
             "pssgpu.cu"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_cuda(force: bool = False) -> Path:
    out = LIB / "libpssgpu.so"
    deps = [CSRC / d for d in CUDA_DEPS] + [INCLUDE / "pssgpu.h"]
    if force or _stale(out, deps):
        LIB.mkdir(exist_ok=True)
        _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fopenmp", "-shared", "-o", str(out),
              *[str(CSRC / s) for s in CUDA_SOURCES], "-lgomp"])
    return out


def build_host(force: bool = False) -> Path:
    out = LIB / "libpsswork.so"
    src = CSRC / "workgen.cpp"
    if force or _stale(out, [src]):
        LIB.mkdir(exist_ok=True)
        _run(["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-Wall",
              "-o", str(out), str(src)])
    return out


def build_all(force: bool = False) -> None:
    build_host(force)
    build_cuda(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
