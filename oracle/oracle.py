"""TEST INFRASTRUCTURE, not part of the product: ctypes bindings of the two
checkers built by oracle/Makefile, and small restatements in numpy / Python.

* ``build/libpssoracle.so`` -- the plain-C restatement (pss_oracle.c).
* ``_ref/libps5ref.so``     -- the reference pS5 compiled from its sources.
* ``split_text`` / ``sorted_output`` -- psstest's text loading and its -o
  output, pinned to the reference psstest's outputs (tests/golden/text/).
* ``lcp_merge2`` -- the reference loser tree's LCP rule for two runs.

Only tests/, the smoke check and the CPU-baseline leg of bench.py use this
module, always as the checker or as the timed reference.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "build" / "libpssoracle.so"
REF_SO = HERE / "_ref" / "libps5ref.so"

_orc = None
_ref = None


def oracle_lib() -> C.CDLL:
    global _orc
    if _orc is None:
        lib = C.CDLL(str(ORACLE_SO))
        lib.pso_get_uint64.restype = C.c_uint64
        lib.pso_get_uint64.argtypes = [C.c_void_p, C.c_size_t]
        lib.pso_lcp_key_type.restype = C.c_uint
        lib.pso_lcp_key_type.argtypes = [C.c_uint64, C.c_uint64]
        lib.pso_lcp_key_depth.restype = C.c_uint
        lib.pso_lcp_key_depth.argtypes = [C.c_uint64]
        lib.pso_sort_lcp.restype = None
        lib.pso_sort_lcp.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
        lib.pso_classify.restype = None
        lib.pso_classify.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p]
        lib.pso_check_order.restype = C.c_int64
        lib.pso_check_order.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]
        lib.pso_check_permutation.restype = C.c_int
        lib.pso_check_permutation.argtypes = [C.c_void_p, C.c_size_t]
        lib.pso_lcp_array.restype = None
        lib.pso_lcp_array.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
        lib.pso_check_lcp32.restype = C.c_int64
        lib.pso_check_lcp32.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
        lib.pso_dprefix.restype = C.c_uint64
        lib.pso_dprefix.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                    C.POINTER(C.c_uint64)]
        _orc = lib
    return _orc


def ref_available() -> bool:
    return REF_SO.exists()


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REF_SO))
        lib.ps5ref_set_threads.restype = C.c_int
        lib.ps5ref_set_threads.argtypes = [C.c_int]
        lib.ps5ref_sort.restype = None
        lib.ps5ref_sort.argtypes = [C.c_void_p, C.c_size_t]
        lib.ps5ref_sort_lcp.restype = None
        lib.ps5ref_sort_lcp.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        lib.ps5ref_get_uint64.restype = C.c_uint64
        lib.ps5ref_get_uint64.argtypes = [C.c_void_p, C.c_size_t]
        lib.ps5ref_find_bkt.restype = None
        lib.ps5ref_find_bkt.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
        lib.ps5ref_verify_lcp.restype = C.c_int
        lib.ps5ref_verify_lcp.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t]
        _ref = lib
    return _ref


def _u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


# ---- restatement ----------------------------------------------------------

def sort_ids(chars, offs) -> np.ndarray:
    chars, offs = _u8(chars), _u64(offs)
    ids = np.arange(offs.shape[0], dtype=np.uint32)
    oracle_lib().pso_sort_lcp(chars.ctypes.data, offs.ctypes.data, ids.ctypes.data,
                              offs.shape[0], None)
    return ids


def sort_ids_lcp(chars, offs):
    chars, offs = _u8(chars), _u64(offs)
    n = offs.shape[0]
    ids = np.arange(n, dtype=np.uint32)
    lcp = np.zeros(n, dtype=np.uint64)
    oracle_lib().pso_sort_lcp(chars.ctypes.data, offs.ctypes.data, ids.ctypes.data, n,
                              lcp.ctypes.data)
    return ids, lcp


def lcp_array(chars, offs, ids) -> np.ndarray:
    chars, offs = _u8(chars), _u64(offs)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    lcp = np.zeros(ids.shape[0], dtype=np.uint64)
    oracle_lib().pso_lcp_array(chars.ctypes.data, offs.ctypes.data, ids.ctypes.data,
                               ids.shape[0], lcp.ctypes.data)
    return lcp


def check_order(chars, offs, ids) -> int:
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    return oracle_lib().pso_check_order(_u8(chars).ctypes.data, _u64(offs).ctypes.data,
                                        ids.ctypes.data, ids.shape[0])


def check_permutation(ids) -> bool:
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    return bool(oracle_lib().pso_check_permutation(ids.ctypes.data, ids.shape[0]))


def check_lcp32(chars, offs, ids, lcp) -> int:
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    lcp = np.ascontiguousarray(lcp, dtype=np.uint32)
    return oracle_lib().pso_check_lcp32(_u8(chars).ctypes.data, _u64(offs).ctypes.data,
                                        ids.ctypes.data, ids.shape[0], lcp.ctypes.data)


def dprefix(chars, offs, ids):
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    s = C.c_uint64()
    d = oracle_lib().pso_dprefix(_u8(chars).ctypes.data, _u64(offs).ctypes.data,
                                 ids.ctypes.data, ids.shape[0], C.byref(s))
    return d, s.value


def get_uint64(chars, off, depth) -> int:
    chars = _u8(chars)
    return oracle_lib().pso_get_uint64(chars.ctypes.data + int(off), depth)


def classify(splitters, keys) -> np.ndarray:
    splitters, keys = _u64(splitters), _u64(keys)
    out = np.zeros(keys.shape[0], dtype=np.uint16)
    oracle_lib().pso_classify(splitters.ctypes.data, splitters.shape[0], keys.ctypes.data,
                              keys.shape[0], out.ctypes.data)
    return out


def sorted_strings(chars, offs, ids) -> bytes:
    """Concatenation of the sorted strings with their NULs (byte-compare form
    of a sorted sequence)."""
    raw = _u8(chars).tobytes()
    parts = []
    for i in ids:
        o = int(offs[i])
        parts.append(raw[o:raw.index(b"\0", o) + 1])
    return b"".join(parts)


# ---- reference pS5 ---------------------------------------------------------

def ref_pointer_array(chars, offs):
    """unsigned char* array into `chars` (kept alive by the caller)."""
    base = chars.ctypes.data
    ptrs = (np.asarray(offs, dtype=np.uint64) + np.uint64(base)).astype(np.uint64)
    return ptrs


def ref_sort(chars, offs, threads: int = 0, lcp: bool = False):
    """Run the reference pS5 (parallel_sample_sortBTCUI or
    parallel_sample_sort_lcp_base) on the arena; returns (ids, lcp or None).
    lcp[0] keeps the sentinel 42 the reference tests use."""
    chars = _u8(chars)
    lib = ref_lib()
    lib.ps5ref_set_threads(threads)
    ptrs = ref_pointer_array(chars, offs)
    n = ptrs.shape[0]
    lcp_a = None
    if lcp:
        lcp_a = np.full(n, np.uint64(2**64 - 1), dtype=np.uint64)
        if n:
            lcp_a[0] = 42
        lib.ps5ref_sort_lcp(ptrs.ctypes.data, lcp_a.ctypes.data, n)
    else:
        lib.ps5ref_sort(ptrs.ctypes.data, n)
    order = np.argsort(np.asarray(offs, dtype=np.uint64), kind="stable")
    sorted_offs = np.asarray(offs, dtype=np.uint64)[order]
    pos = np.searchsorted(sorted_offs, ptrs - np.uint64(chars.ctypes.data))
    ids = order[pos].astype(np.uint32)
    return ids, lcp_a


def ref_get_uint64(chars, off, depth) -> int:
    chars = _u8(chars)
    return ref_lib().ps5ref_get_uint64(chars.ctypes.data + int(off), depth)


def ref_find_bkt(splitters_1023, keys) -> np.ndarray:
    s, keys = _u64(splitters_1023), _u64(keys)
    assert s.shape[0] == 1023
    out = np.zeros(keys.shape[0], dtype=np.uint16)
    ref_lib().ps5ref_find_bkt(s.ctypes.data, keys.ctypes.data, keys.shape[0], out.ctypes.data)
    return out


def split_text(text, suffix: bool = False):
    """psstest's plain-file loading and string pointer array, restated for
    the device-side text preparation: src/tools/input.hpp:255-297 (every
    '\\n' or NUL byte becomes NUL and, unless it is the last byte, starts a
    new string; the last byte is forced to NUL; suffix mode leaves the bytes
    and counts every position) and src/psstest.cpp:479-518 (strings start at
    0 and behind every NUL; suffix mode: at every position).

    Returns (arena: u8[size + 16], the text after the rewrite plus zero pad;
    offsets: u64[n])."""
    t = np.frombuffer(bytes(text), dtype=np.uint8).copy() if not isinstance(text, np.ndarray) \
        else np.ascontiguousarray(text, dtype=np.uint8).copy()
    size = t.shape[0]
    if size == 0:
        return np.zeros(16, np.uint8), np.zeros(0, np.uint64)
    if suffix:
        starts = np.arange(size, dtype=np.uint64)
    else:
        sep = (t == 10) | (t == 0)
        t[sep] = 0
        starts = np.concatenate([np.zeros(1, np.uint64),
                                 np.flatnonzero(sep[: size - 1]).astype(np.uint64) + 1])
    t[size - 1] = 0
    return np.concatenate([t, np.zeros(16, np.uint8)]), starts


def sorted_output(chars, offs, ids) -> bytes:
    """psstest's -o output (src/psstest.cpp:696-703): every string of the
    sorted order followed by a newline."""
    raw = bytes(chars)
    out = []
    for i in np.asarray(ids):
        o = int(offs[int(i)])
        e = raw.index(b"\0", o)
        out.append(raw[o:e] + b"\n")
    return b"".join(out)


def lcp_merge2(chars, offs, a_ids, a_lcp, b_ids, b_lcp):
    """Two-way LCP merge, restated from the reference's LCP loser tree
    (src/sequential/bingmann-lcp_losertree.hpp:61-105 for the compare rule,
    :156-185 for the output and the winner's successor): every head carries
    its LCP with the last output; the head with the larger LCP is the smaller
    string without reading a char; on equal LCPs the two compare from that
    depth, and the loser keeps the LCP found. The winner's successor takes its
    LCP from its run's LCP array; the output LCP is the winner's LCP. Ties go
    to the first run.

    Pure Python, for small inputs. Returns (ids, lcp, chars_read): lcp[0] = 0,
    chars_read counts the char pairs compared."""
    raw = bytes(chars)

    def char_at(i, d):
        o = int(offs[int(i)]) + d
        return raw[o] if o < len(raw) else 0

    runs = [(list(a_ids), list(a_lcp)), (list(b_ids), list(b_lcp))]
    pos = [0, 0]
    h = [0, 0]  # LCP of each head with the last output (0 before the first)
    out_ids, out_lcp = [], []
    reads = 0
    while pos[0] < len(runs[0][0]) or pos[1] < len(runs[1][0]):
        if pos[0] >= len(runs[0][0]):
            w = 1
        elif pos[1] >= len(runs[1][0]):
            w = 0
        elif h[0] != h[1]:
            w = 0 if h[0] > h[1] else 1
        else:
            a, b = runs[0][0][pos[0]], runs[1][0][pos[1]]
            d = h[0]
            while True:
                ca, cb = char_at(a, d), char_at(b, d)
                reads += 1
                if ca != cb or ca == 0:
                    break
                d += 1
            w = 0 if ca <= cb else 1  # equal strings: the first run
            h[1 - w] = d              # the loser's LCP with the new last output
        out_ids.append(runs[w][0][pos[w]])
        out_lcp.append(h[w] if out_ids[1:] else 0)
        pos[w] += 1
        if pos[w] < len(runs[w][0]):
            h[w] = int(runs[w][1][pos[w]])  # against its predecessor, the last output
    return np.array(out_ids, np.uint32), np.array(out_lcp, np.uint64), reads
