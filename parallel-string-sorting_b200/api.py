"""Python host API of the B200 string sample sort.

It mirrors the reference's entry points for this path
(src/parallel/bingmann-parallel_sample_sort.hpp:1685-1757 and the psstest
contestant signatures of src/tools/contest.hpp:88-91):

* ``parallel_sample_sort(strings)`` sorts a list of byte strings
  (the role of ``parallel_sample_sort_base``),
* ``parallel_sample_sort_lcp(strings)`` also returns the LCP array
  (``parallel_sample_sort_lcp_base``; ``lcp[0]`` is reported as 0),
* ``Context.sort_host`` / ``Context.sort_device`` sort an arena
  (chars + offsets) from host or device memory,
* ``sort_pointer_array`` calls the C drop-in ``pssgpu_sort_strings*`` on a
  raw ``unsigned char**`` array, exactly as psstest would.

Errors raise ``SortError`` carrying the library's status code. Nothing here
falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _native
from ._native import PssKernelStats, PssStats, STATUS_NAMES


class SortError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _check(rc: int) -> None:
    if rc != 0:
        msg = _native.gpu().pssgpu_last_error()
        raise SortError(rc, msg.decode() if msg else "")


def _ptr(a) -> Optional[int]:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


class Context:
    """A device context: one CUDA stream and a reusable workspace."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(_native.gpu().pssgpu_ctx_create(device, C.byref(h)))
        self._h = h
        self.device = device

    def close(self) -> None:
        if self._h:
            _native.gpu().pssgpu_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self) -> dict:
        s = PssStats()
        _check(_native.gpu().pssgpu_ctx_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in PssStats._fields_}

    def set_profile(self, on: bool) -> None:
        """Time every kernel class with CUDA events (per-class totals in
        kernel_stats())."""
        _check(_native.gpu().pssgpu_ctx_set_profile(self._h, 1 if on else 0))

    OPT_PROFILE = 1
    OPT_INDIRECT_HANDLES = 2
    OPT_SINGLE_LAUNCH = 3
    OPT_WAIT_LIMIT = 4
    OPT_MERGE_PIECE = 5
    OPT_SUFFIX_DOUBLING = 6

    def set_option(self, option: int, value: int) -> None:
        _check(_native.gpu().pssgpu_ctx_set_option(self._h, option, value))

    def kernel_stats(self) -> list:
        arr = (PssKernelStats * 16)()
        k = _native.gpu().pssgpu_ctx_kernel_stats(self._h, arr, 16)
        if k < 0:
            _check(-k)
        return [{"name": arr[i].name.decode(), "launches": arr[i].launches,
                 "strings": arr[i].strings, "alg_bytes": arr[i].alg_bytes, "ms": arr[i].ms}
                for i in range(k)]

    def sort_host(self, chars: np.ndarray, offs: np.ndarray, lcp: bool = True,
                  out_perm: Optional[np.ndarray] = None, out_lcp: Optional[np.ndarray] = None):
        """Sort the arena strings; returns (perm u32[n], lcp u32[n] or None).
        out_perm / out_lcp may supply (pinned) result buffers."""
        chars = np.ascontiguousarray(chars, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        n = offs.shape[0]
        perm = np.empty(n, dtype=np.uint32) if out_perm is None else out_perm
        if not lcp:
            lcp_a = None
        else:
            lcp_a = np.zeros(n, dtype=np.uint32) if out_lcp is None else out_lcp
        assert perm.dtype == np.uint32 and perm.shape[0] >= n and perm.flags.c_contiguous
        _check(_native.gpu().pssgpu_sort_host(self._h, _ptr(chars), chars.shape[0], _ptr(offs), n,
                                              _ptr(perm), _ptr(lcp_a)))
        return perm, lcp_a

    def set_tree_bits(self, table) -> None:
        """Splitter-tree levels per size class (index k: segments of 2^k..2^(k+1)-1
        strings; 0 = default rule)."""
        t = np.ascontiguousarray(np.asarray(table, dtype=np.uint8))
        _check(_native.gpu().pssgpu_ctx_set_tree_bits(self._h, t.ctypes.data, t.shape[0]))

    def sort_batch_host(self, chars: np.ndarray, offs: np.ndarray, inst: np.ndarray,
                        lcp: bool = True, out_perm=None, out_lcp=None):
        """Sort independent instances (inst: ninst+1 boundaries into offs);
        returns per-instance permutations and LCP arrays, concatenated."""
        chars = np.ascontiguousarray(chars, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        inst = np.ascontiguousarray(inst, dtype=np.uint64)
        n = offs.shape[0]
        perm = np.empty(n, dtype=np.uint32) if out_perm is None else out_perm
        lcp_a = (np.zeros(n, dtype=np.uint32) if out_lcp is None else out_lcp) if lcp else None
        _check(_native.gpu().pssgpu_sort_batch_host(self._h, _ptr(chars), chars.shape[0],
                                                    _ptr(offs), inst.ctypes.data,
                                                    inst.shape[0] - 1, _ptr(perm), _ptr(lcp_a)))
        return perm, lcp_a

    def sort_batch_device(self, chars, nchars: int, offs, inst: np.ndarray, perm, lcp=None,
                          stream=None) -> None:
        inst = np.ascontiguousarray(inst, dtype=np.uint64)
        s = None if stream is None else (stream if isinstance(stream, int) else stream.cuda_stream)
        _check(_native.gpu().pssgpu_sort_batch_device(
            self._h, chars.data_ptr(), nchars, offs.data_ptr(), inst.ctypes.data,
            inst.shape[0] - 1, perm.data_ptr(), None if lcp is None else lcp.data_ptr(), s))

    def sort_device(self, chars, nchars: int, offs, perm, lcp=None, stream=None) -> None:
        """Sort an arena resident on this context's device (torch tensors or
        raw device pointers). ``chars`` must hold nchars + 16 bytes."""
        def addr(t):
            if t is None:
                return None
            return t if isinstance(t, int) else t.data_ptr()
        n = offs.shape[0] if hasattr(offs, "shape") else int(perm)
        s = None if stream is None else (stream if isinstance(stream, int) else stream.cuda_stream)
        _check(_native.gpu().pssgpu_sort_device(self._h, addr(chars), nchars, addr(offs), n,
                                                addr(perm), addr(lcp), s))


    TEXT_LINES = 0
    TEXT_SUFFIXES = 1

    def sort_text_host(self, text, mode: int = 0, lcp: bool = True):
        """Sort the lines (mode TEXT_LINES) or suffixes (TEXT_SUFFIXES) of a
        host text, split on the device as psstest's loader splits a file;
        returns (perm u32[n], lcp u32[n] or None), ids in text order."""
        t = np.ascontiguousarray(np.frombuffer(text, dtype=np.uint8) if isinstance(text, (bytes, bytearray))
                                 else text, dtype=np.uint8)
        size = t.shape[0]
        n = C.c_uint64(0)
        cap = size  # n <= size in both modes
        perm = np.empty(max(cap, 1), dtype=np.uint32)
        lcp_a = np.zeros(max(cap, 1), dtype=np.uint32) if lcp else None
        _check(_native.gpu().pssgpu_sort_text_host(self._h, _ptr(t), size, mode, _ptr(perm),
                                                   _ptr(lcp_a), cap, C.byref(n)))
        k = n.value
        return perm[:k], (lcp_a[:k] if lcp else None)

    def prepare_text_device(self, text, size: int, mode: int, offs, stream=None) -> int:
        """In place on device buffers (torch tensors or raw pointers): the
        text becomes an arena, offs receives the string offsets; returns n."""
        def addr(t):
            return t if isinstance(t, int) else t.data_ptr()
        cap = offs.numel() if hasattr(offs, "numel") else 0
        n = C.c_uint64(0)
        s = None if stream is None else (stream if isinstance(stream, int) else stream.cuda_stream)
        _check(_native.gpu().pssgpu_prepare_text_device(self._h, addr(text), size, mode,
                                                        addr(offs), cap, C.byref(n), s))
        return n.value


    def merge_lcp_device(self, chars, nchars: int, offs, runs, ids, lcp, ids_out, lcp_out=None,
                         stream=None) -> None:
        """Merge sorted runs (runs: nruns + 1 boundaries into ids / lcp) into
        ids_out and, if given, its LCP array lcp_out (device tensors)."""
        runs = np.ascontiguousarray(runs, dtype=np.uint64)

        def addr(t):
            if t is None:
                return None
            return t if isinstance(t, int) else t.data_ptr()
        s = None if stream is None else (stream if isinstance(stream, int) else stream.cuda_stream)
        _check(_native.gpu().pssgpu_merge_lcp_device(
            self._h, addr(chars), nchars, addr(offs), runs.ctypes.data, runs.shape[0] - 1,
            addr(ids), addr(lcp), addr(ids_out), addr(lcp_out), s))


_default: Optional[Context] = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


def pack_strings(strings: Sequence[bytes]):
    """Pack byte strings (no NULs inside) into a NUL-terminated arena."""
    lens = np.fromiter((len(s) for s in strings), dtype=np.uint64, count=len(strings))
    offs = np.zeros(len(strings), dtype=np.uint64)
    if len(strings):
        np.cumsum(lens[:-1] + 1, out=offs[1:])
    chars = np.frombuffer(b"".join(s + b"\0" for s in strings), dtype=np.uint8).copy()
    return chars, offs


def parallel_sample_sort(strings: Sequence[bytes]) -> list:
    chars, offs = pack_strings(strings)
    if len(strings) == 0:
        return []
    perm, _ = default_context().sort_host(chars, offs, lcp=False)
    return [strings[i] for i in perm]


def parallel_sample_sort_lcp(strings: Sequence[bytes]):
    chars, offs = pack_strings(strings)
    if len(strings) == 0:
        return [], np.zeros(0, dtype=np.uint32)
    perm, lcp = default_context().sort_host(chars, offs, lcp=True)
    lcp[0] = 0
    return [strings[i] for i in perm], lcp


def sort_pointer_array(ptrs, n: int, lcp=None, cache=None) -> int:
    """Call the contestant drop-in on a ctypes ``unsigned char*`` array.
    Returns the status code (the void drop-ins abort on failure instead)."""
    return _native.gpu().pssgpu_sort_strings_status(ptrs, lcp, cache, n)


def sort_pointer_array_out(ptrs, output, n: int) -> int:
    """The separate-output drop-in: sorted pointers into ``output``, ``ptrs``
    unchanged. Returns the status code."""
    return _native.gpu().pssgpu_sort_strings_out_status(ptrs, output, n)


def sort_pointer_array_arena(arena: int, arena_size: int, ptrs, n: int, output=None, lcp=None,
                             cache=None) -> int:
    """The pointer-array sort for strings that all lie in one buffer of
    ``arena_size`` bytes at address ``arena`` (psstest's string data).
    ``output`` None sorts in place. Returns the status code."""
    return _native.gpu().pssgpu_sort_strings_arena(arena, arena_size, ptrs, output, lcp, cache, n)
