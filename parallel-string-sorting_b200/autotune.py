"""Autotuner for the batched sort: per size class of big segments
(2^k .. 2^(k+1)-1 strings), the splitter-tree depth L (2^L - 1 splitters,
2^(L+1) - 1 buckets) that sorts fastest.

For every class k it builds a batch of instances of that class from the
batched workload's string distribution (lognormal lengths, printable ASCII),
times pssgpu_sort_batch_device for each candidate L with CUDA events (median
of a few runs, inputs resident on the device) and keeps the best. The table
is saved as JSON (tuning_b200.json next to this file) and loaded with
load_table(); Context.set_tree_bits applies it.

Run on the GPU: python -m pss_b200.autotune (or tune() from Python).
"""
from __future__ import annotations

import json
import time
from pathlib import Path

import numpy as np

from . import workloads
from .api import Context

TABLE_PATH = Path(__file__).resolve().parent / "tuning_b200.json"
CLASSES = range(10, 21)  # big segments: more than 1024 strings


def _class_batch(k: int, strings: int, seed: int):
    """Instances of 2^k..2^(k+1)-1 strings, about `strings` in total."""
    rng = np.random.default_rng(seed + k)
    sizes = []
    total = 0
    while total < strings:
        s = int(rng.integers(1 << k, 1 << (k + 1)))
        sizes.append(s)
        total += s
    inst = np.zeros(len(sizes) + 1, dtype=np.uint64)
    np.cumsum(np.asarray(sizes, dtype=np.uint64), out=inst[1:])
    n = int(inst[-1])
    w = workloads._native.work()
    offs = np.empty(n, dtype=np.uint64)
    nchars = w.pssw_lognormal_offsets(seed + k, n, 3.0, 0.5, 1, 256, offs.ctypes.data)
    chars = np.zeros(nchars + workloads.PAD, dtype=np.uint8)
    alpha = np.frombuffer(workloads.PRINTABLE, dtype=np.uint8).copy()
    w.pssw_random_fill(seed + k, n, offs.ctypes.data, nchars, alpha.ctypes.data, len(alpha),
                       chars.ctypes.data)
    return chars, offs, int(nchars), inst


def tune(ctx: Context = None, strings_per_class: int = 4 << 20, reps: int = 3, seed: int = 11,
         classes=CLASSES, verbose: bool = True) -> dict:
    import torch
    own = ctx is None
    ctx = ctx or Context(0)
    table = [0] * 33
    timings = {}
    stream = torch.cuda.current_stream()
    try:
        for k in classes:
            chars, offs, nchars, inst = _class_batch(k, strings_per_class, seed)
            dc = torch.from_numpy(chars).cuda()
            do = torch.from_numpy(offs.view(np.int64)).cuda()
            dp = torch.empty(len(offs), dtype=torch.int32, device="cuda")
            best = None
            timings[k] = {}
            for L in range(3, min(10, k - 1) + 1):
                t = list(table)
                t[k] = L
                ctx.set_tree_bits(t)
                ctx.sort_batch_device(dc, nchars, do, inst, dp, stream=stream)  # warm
                ms = []
                for _ in range(reps):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    ctx.sort_batch_device(dc, nchars, do, inst, dp, stream=stream)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    ms.append(e0.elapsed_time(e1))
                m = float(np.median(ms))
                timings[k][L] = m
                if best is None or m < best[1]:
                    best = (L, m)
            table[k] = best[0]
            if verbose:
                print(f"class 2^{k}: best L={best[0]} ({best[1]:.3f} ms) of {timings[k]}",
                      flush=True)
            del dc, do, dp
        ctx.set_tree_bits(table)
    finally:
        if own:
            ctx.close()
    return {"table": table, "timings_ms": {str(k): v for k, v in timings.items()},
            "strings_per_class": strings_per_class, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}


def save_table(result: dict, path: Path = TABLE_PATH) -> None:
    path.write_text(json.dumps(result, indent=1, sort_keys=True) + "\n")


def load_table(path: Path = TABLE_PATH):
    """The tuned tree-bits table, or None when no table has been written."""
    if not path.exists():
        return None
    return json.loads(path.read_text())["table"]


if __name__ == "__main__":
    save_table(tune())
