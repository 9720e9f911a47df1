"""Seeded synthetic workloads with the shapes of the reference's benchmark
configurations (no public dataset is available offline; every generator is
deterministic and documented).

* ``digits(seed=1)``            -- strings of length U[1,40] over '0'..'9',
  packed to 10 MiB of chars (a psstest ``random10``-style plain sort).
* ``prefixes(n=64 Mi, seed=2)``  -- one of 4096 random 48-char prefixes
  ('a'..'z', Zipf s=1.1 by rank) + a suffix of length U[8,24]; mean LCP ~50.
* ``dna_suffixes(seed=3)``       -- a 32 MiB ACGT text with 5% overwritten by
  copies of earlier 1-10 KiB blocks; all 33,554,433 suffixes.
* ``random_strings(...)``        -- generic test inputs.

Arenas are (chars u8[nchars + 16], offs u64[n], nchars): NUL-terminated
strings, 16 zero bytes of padding after the last char. ``out`` allocators let
callers place the arena in pinned host memory.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional

import numpy as np

from . import _native

PAD = 16


def _alloc_np(nbytes: int, dtype) -> np.ndarray:
    return np.empty(nbytes // np.dtype(dtype).itemsize, dtype=dtype)


def random_strings(n: int, lmin: int, lmax: int, alphabet: bytes, seed: int,
                   alloc: Callable = _alloc_np):
    w = _native.work()
    offs = alloc(8 * n, np.uint64) if n else np.zeros(0, np.uint64)
    nchars = w.pssw_random_offsets(seed, n, lmin, lmax, offs.ctypes.data if n else None)
    chars = alloc(nchars + PAD, np.uint8)
    chars[nchars:] = 0
    alpha = np.frombuffer(alphabet, dtype=np.uint8).copy()
    if n:
        w.pssw_random_fill(seed, n, offs.ctypes.data, nchars, alpha.ctypes.data, len(alpha),
                           chars.ctypes.data)
    return chars, offs, int(nchars)


def digits(seed: int = 1, budget: int = 10 * 1024 * 1024, alloc: Callable = _alloc_np):
    w = _native.work()
    nch = C.c_uint64()
    n = w.pssw_digits_count(seed, budget, C.byref(nch))
    offs = alloc(8 * n, np.uint64)
    chars = alloc(nch.value + PAD, np.uint8)
    chars[nch.value:] = 0
    w.pssw_digits_fill(seed, n, offs.ctypes.data, chars.ctypes.data)
    return chars, offs, int(nch.value)


def prefixes(n: int = 64 * 1024 * 1024, seed: int = 2, zipf_s: float = 1.1,
             alloc: Callable = _alloc_np, with_ids: bool = False):
    w = _native.work()
    offs = alloc(8 * n, np.uint64)
    nchars = w.pssw_prefix_offsets(seed, n, offs.ctypes.data)
    chars = alloc(nchars + PAD, np.uint8)
    chars[nchars:] = 0
    ids = np.empty(n, np.uint16) if with_ids else None
    w.pssw_prefix_fill(seed, n, offs.ctypes.data, zipf_s, chars.ctypes.data,
                       ids.ctypes.data if with_ids else None)
    if with_ids:
        return chars, offs, int(nchars), ids
    return chars, offs, int(nchars)


def dna_text(length: int = 32 * 1024 * 1024, seed: int = 3, copy_frac: float = 0.05,
             alloc: Callable = _alloc_np):
    """The text plus its terminating NUL and padding: chars[length] == 0."""
    chars = alloc(length + 1 + PAD, np.uint8)
    chars[length:] = 0
    _native.work().pssw_dna_text(seed, length, copy_frac, chars.ctypes.data)
    return chars


def dna_suffixes(length: int = 32 * 1024 * 1024, seed: int = 3, copy_frac: float = 0.05,
                 alloc: Callable = _alloc_np):
    """All length + 1 suffixes of the text (the last one is empty), as the
    reference's psstest --suffix builds them (src/psstest.cpp:502-518)."""
    chars = dna_text(length, seed, copy_frac, alloc)
    offs = alloc(8 * (length + 1), np.uint64)
    offs[:] = np.arange(length + 1, dtype=np.uint64)
    return chars, offs, length + 1


PRINTABLE = bytes(range(32, 127))


def batch_sizes(ninst: int = 100_000, smin: int = 16, smax: int = 1 << 20,
                budget_chars: int = 1 << 30, mean_chars: float = 23.8, seed: int = 4):
    """Instance sizes of the batched workload: log-uniform in [smin, smax],
    then all scaled by one common factor f (with a floor of smin) so that the
    expected total chars (sizes x mean_chars per string incl. terminator)
    stay within budget_chars. Returns (sizes, f)."""
    rng = np.random.default_rng(seed)
    raw = np.exp(rng.uniform(np.log(smin), np.log(smax), ninst))

    def total(f):
        return np.maximum(smin, np.floor(raw * f)).sum() * mean_chars

    f = 1.0
    if total(1.0) > budget_chars:
        lo, hi = 0.0, 1.0
        for _ in range(60):
            mid = (lo + hi) / 2
            if total(mid) <= budget_chars:
                lo = mid
            else:
                hi = mid
        f = lo
    sizes = np.maximum(smin, np.floor(raw * f)).astype(np.uint64)
    return sizes, f


def batched(ninst: int = 100_000, seed: int = 4, budget_chars: int = 1 << 30,
            smin: int = 16, smax: int = 1 << 20, alloc: Callable = _alloc_np):
    """The batched workload: ninst independent instances (batch_sizes), string
    lengths lognormal(mu=3, sigma=0.5) clipped to [1, 256], chars uniform over
    printable ASCII 32..126, all packed into one arena. Returns (chars, offs,
    nchars, inst) with inst the ninst + 1 instance boundaries."""
    sizes, _ = batch_sizes(ninst, smin, smax, budget_chars, seed=seed)
    inst = np.zeros(ninst + 1, dtype=np.uint64)
    np.cumsum(sizes, out=inst[1:])
    n = int(inst[-1])
    w = _native.work()
    offs = alloc(8 * n, np.uint64)
    nchars = w.pssw_lognormal_offsets(seed, n, 3.0, 0.5, 1, 256, offs.ctypes.data)
    chars = alloc(nchars + PAD, np.uint8)
    chars[nchars:] = 0
    alpha = np.frombuffer(PRINTABLE, dtype=np.uint8).copy()
    w.pssw_random_fill(seed, n, offs.ctypes.data, nchars, alpha.ctypes.data, len(alpha),
                       chars.ctypes.data)
    return chars, offs, int(nchars), inst


def alg_bytes(lcp: np.ndarray, T: int = 32) -> dict:
    """Algorithmic bytes of the sample-sort method for a sorted LCP array."""
    lcp = np.ascontiguousarray(lcp, dtype=np.uint32)
    tot, rb, bb = C.c_uint64(), C.c_uint64(), C.c_uint64()
    mr = C.c_uint32()
    _native.work().pssw_alg_bytes(lcp.ctypes.data, lcp.shape[0], T, C.byref(tot), C.byref(rb),
                                  C.byref(bb), C.byref(mr))
    return {"total": tot.value, "rounds": rb.value, "base": bb.value, "max_round": mr.value}


def check_sorted(chars: np.ndarray, nchars: int, offs: np.ndarray, perm: np.ndarray) -> int:
    """First position whose string sorts before its predecessor (or whose id
    is out of range); -1 when perm lists the strings in order."""
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    perm = np.ascontiguousarray(perm, dtype=np.uint32)
    return int(_native.work().pssw_check_sorted(chars.ctypes.data, nchars, offs.ctypes.data,
                                                perm.ctypes.data, perm.shape[0]))


def check_permutation(perm: np.ndarray) -> bool:
    """True when perm holds every id 0..n-1 exactly once."""
    perm = np.ascontiguousarray(perm, dtype=np.uint32)
    return bool(_native.work().pssw_check_permutation(perm.ctypes.data, perm.shape[0]))


def string_lengths(chars: np.ndarray, offs: np.ndarray) -> np.ndarray:
    """strlen of every string of the arena."""
    zeros = np.flatnonzero(np.asarray(chars) == 0).astype(np.uint64)
    pos = np.searchsorted(zeros, np.asarray(offs, dtype=np.uint64))
    return (zeros[pos] - np.asarray(offs, dtype=np.uint64)).astype(np.uint64)


def canonical_ids(chars, offs, ids, lcp, lengths=None) -> np.ndarray:
    """Sorted ids with every run of equal strings in increasing id order: two
    correct sorts of the same input (which may order equal strings
    differently) have the same canonical ids. `lengths` (the strlen of every
    string of offs) may be passed to skip scanning the arena."""
    ids = np.asarray(ids, dtype=np.uint32)
    n = ids.shape[0]
    if n == 0:
        return ids.copy()
    lens = (string_lengths(chars, offs) if lengths is None else np.asarray(lengths))[ids]
    lcp = np.asarray(lcp, dtype=np.uint64)
    eq = np.zeros(n, dtype=bool)
    eq[1:] = (lcp[1:] == lens[1:]) & (lens[1:] == lens[:-1])
    run = np.cumsum(~eq)
    return ids[np.lexsort((ids, run))]


def strings_of(chars: np.ndarray, offs: np.ndarray, ids: Optional[np.ndarray] = None) -> list:
    """Python bytes of the strings (small inputs only)."""
    raw = chars.tobytes()
    idx = range(len(offs)) if ids is None else ids
    out = []
    for i in idx:
        o = int(offs[i])
        out.append(raw[o:raw.index(b"\0", o)])
    return out
