"""Serving: a sort-request server with continuous batching (pssgpu_server_*
in include/pssgpu.h) and the synthetic request stream that drives it.

The stream follows the serving workload: Poisson arrivals (2,000 requests/s
for 60 s by default), request sizes log-uniform in [1 KB, 64 MB] of chars,
an alphabet of 4, 10, 26 or 95 symbols drawn per request, string lengths
uniform in [1, 64]. Request bodies are contiguous runs of strings cut from
one pre-generated pool per alphabet (generating hundreds of GB of fresh
random text per minute on the host is not possible); the runs start at
random strings, so requests differ.
"""
from __future__ import annotations

import ctypes as C
import queue
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import _native, workloads
from .api import SortError, _check
from ._native import RequestInfo, ServerConfig, ServerStats

ALPHABETS = {4: b"ACGT", 10: b"0123456789", 26: b"abcdefghijklmnopqrstuvwxyz",
             95: bytes(range(32, 127))}


class Server:
    def __init__(self, device: int = 0, budget: int = 40 << 30, workers: int = 3,
                 max_batch_strings: int = 8 << 20, max_batch_requests: int = 0):
        cfg = ServerConfig(budget, max_batch_strings, workers, max_batch_requests)
        h = C.c_void_p()
        _check(_native.gpu().pssgpu_server_create(device, C.byref(cfg), C.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h:
            _native.gpu().pssgpu_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, chars_ptr: int, nchars: int, offs: np.ndarray, offs_base: int,
               perm: np.ndarray, lcp: Optional[np.ndarray] = None) -> int:
        """Queue one request; the caller keeps every buffer alive until wait()."""
        t = C.c_uint64()
        _check(_native.gpu().pssgpu_server_submit(
            self._h, chars_ptr, nchars, offs.ctypes.data, offs_base, offs.shape[0],
            perm.ctypes.data, None if lcp is None else lcp.ctypes.data, C.byref(t)))
        return t.value

    def wait(self, ticket: int) -> dict:
        info = RequestInfo()
        rc = _native.gpu().pssgpu_server_wait(self._h, ticket, C.byref(info))
        if rc:
            raise SortError(rc, _native.gpu().pssgpu_last_error().decode())
        return {f: getattr(info, f) for f, _ in RequestInfo._fields_}

    def stats(self) -> dict:
        s = ServerStats()
        _check(_native.gpu().pssgpu_server_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}


@dataclass
class Pool:
    chars: np.ndarray
    offs: np.ndarray
    nchars: int


def make_pools(bytes_per_pool: int = 256 << 20, seed: int = 5, alloc: Callable = workloads._alloc_np):
    """One string pool per alphabet: lengths U[1, 64], uniform chars."""
    pools = {}
    for i, (a, alpha) in enumerate(sorted(ALPHABETS.items())):
        n = bytes_per_pool // 34  # mean string + terminator is 33.5 bytes
        c, o, nch = workloads.random_strings(n, 1, 64, alpha, seed + i, alloc=alloc)
        pools[a] = Pool(c, o, nch)
    return pools


@dataclass
class Req:
    t_arrive: float
    alphabet: int
    i0: int
    i1: int
    start: int
    nchars: int
    perm: np.ndarray = None
    lcp: np.ndarray = None
    ticket: int = 0
    info: dict = field(default_factory=dict)


def make_stream(pools, rate: float = 2000.0, duration: float = 60.0, min_bytes: int = 1 << 10,
                max_bytes: int = 64 << 20, seed: int = 6) -> List[Req]:
    """Poisson arrivals; sizes log-uniform in [min_bytes, max_bytes]."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    alphas = sorted(pools)
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        a = alphas[rng.integers(len(alphas))]
        pool = pools[a]
        size = int(np.exp(rng.uniform(np.log(min_bytes), np.log(max_bytes))))
        size = min(size, pool.nchars // 2)
        n = pool.offs.shape[0]
        i0 = int(rng.integers(0, n - 1))
        start = int(pool.offs[i0])
        end_target = start + size
        # search with a uint64 scalar: a Python int would make numpy convert
        # the whole offset array to float64 on every call
        i1 = int(np.searchsorted(pool.offs, np.uint64(end_target), side="right"))
        i1 = max(i0 + 1, min(i1, n))
        end = int(pool.offs[i1]) if i1 < n else pool.nchars
        out.append(Req(t, a, i0, i1, start, end - start))
    return out


class ResultRing:
    """Result buffers carved from one reused host buffer (pinned when alloc
    pins), as a serving client with a fixed result area hands them out: a
    request's slot is overwritten once `entries` more results have been
    handed out, so the results must be read before then."""

    def __init__(self, entries: int, alloc: Callable = workloads._alloc_np):
        self.buf = alloc(4 * entries, np.uint32)
        self.buf.fill(0)  # resident before the first copy lands in it
        self.pos = 0

    def take(self, n: int) -> np.ndarray:
        if n > self.buf.shape[0]:
            raise ValueError("request larger than the result ring")
        if self.pos + n > self.buf.shape[0]:
            self.pos = 0
        out = self.buf[self.pos:self.pos + n]
        self.pos += n
        return out


def run_stream(server: Server, pools, reqs: List[Req], want_lcp: bool = False,
               results: ResultRing = None) -> dict:
    """Submit every request at its arrival time (relative to now); a second
    thread waits for completions in order. Returns latency figures. Results
    go to fresh arrays, or to slots of `results` (perm only)."""
    if results is not None and want_lcp:
        raise ValueError("a result ring holds permutations only")
    submitted: "queue.Queue[Req]" = queue.Queue()

    def waiter():
        for _ in range(len(reqs)):
            r = submitted.get()
            r.info = server.wait(r.ticket)

    t0 = time.perf_counter()
    th = threading.Thread(target=waiter)
    th.start()
    for r in reqs:
        delay = t0 + r.t_arrive - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        pool = pools[r.alphabet]
        n = r.i1 - r.i0
        r.perm = results.take(n) if results is not None else np.empty(n, dtype=np.uint32)
        r.lcp = np.zeros(n, dtype=np.uint32) if want_lcp else None
        r.ticket = server.submit(pool.chars.ctypes.data + r.start, r.nchars,
                                 pool.offs[r.i0:r.i1], r.start, r.perm, r.lcp)
        submitted.put(r)
    th.join()
    wall = time.perf_counter() - t0
    lat = np.array([(r.info["t_done_ns"] - r.info["t_submit_ns"]) / 1e6 for r in reqs])
    qwait = np.array([(r.info["t_start_ns"] - r.info["t_submit_ns"]) / 1e6 for r in reqs])
    chars = sum(r.nchars for r in reqs)
    first = min(r.info["t_submit_ns"] for r in reqs)
    last = max(r.info["t_done_ns"] for r in reqs)
    return {"requests": len(reqs), "chars": chars, "strings": sum(r.i1 - r.i0 for r in reqs),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "queue_p50_ms": float(np.percentile(qwait, 50)),
            "queue_p99_ms": float(np.percentile(qwait, 99)),
            "sustained_char_gb_s": chars / ((last - first) / 1e9) / 1e9,
            "wall_s": wall,
            "mean_batch_requests": float(np.mean([r.info["batch_requests"] for r in reqs]))}
