#!/usr/bin/env python
"""Benchmark of the B200 string sample sort.

Workload: 64 Mi strings, each one of 4096 random 48-char prefixes ('a'..'z',
picked Zipf s=1.1 by rank) followed by a suffix of uniform length 8..24 over
'a'..'z' (about 4.36 GB of chars, mean LCP ~50), generated seeded on the host.
One step = one full plain sort (the pS5-Unroll contestant's job) of that
instance.

  value      sorted char GB/s with the arena resident in HBM (CUDA events on
             the launching stream, max over ranks; inputs are 4.4 GB > L2)
  e2e        the same metric through the C ABI with host buffers: the H2D copy
             of arena + offsets from pinned memory and the D2H copy of the
             permutation are inside every timed step
  e2e_text   the same through the text entry point: only the text (NUL ->
             newline, or the DNA text for suffixes) is copied; lines and
             offsets are made on the device
  roofline   the kernel class with the largest device time: its algorithmic
             bytes / its summed event time against the measured HBM copy
             bandwidth; roofline_sort does the same for the whole sort with
             the method's algorithmic bytes computed from the LCP array
  cpu_baseline  the reference pS5 (compiled from the reference sources) on
             the same instance, all host threads, best of 3
  verified   the last timed sort's permutation checked on the host (every id
             once, neighbouring strings in strcmp order)
  batched    the 100k-instance batched workload: one batched call (median and
             p99 over steps) against one call per instance (sampled)
  serving    a shortened Poisson request stream (--serving-duration seconds at
             --rate) through the continuous-batching server: p50 / p99 latency

--impl reference times the reference pS5 alone on the host cores (rank 0) on
the same instance, with the same warm-up and step counts.
With N GPUs (torchrun) every rank sorts its own instance (weak scaling; no
collective is needed by the sort).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "sorted char GB/s"
N_DEFAULT = 64 * 1024 * 1024
SEED = 2


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=N_DEFAULT, help="strings per instance (prefixes)")
    p.add_argument("--workload", choices=["prefixes", "digits", "dna"], default="prefixes",
                   help="sort mode: prefixes = 64 Mi high-LCP strings (the headline), "
                        "digits = the 10 MiB random-digit strings, dna = all suffixes of a "
                        "32 MiB repetitive DNA text")
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-extras", action="store_true",
                   help="sort mode: leave out the batched and serving records")
    p.add_argument("--serving-duration", type=float, default=10.0,
                   help="sort mode: seconds of arrivals of the serving record")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--mode", choices=["sort", "batched", "serving", "autotune", "merge"],
                   default="sort",
                   help="sort: the headline line; batched: the 100k-instance batch "
                        "against one call per instance; serving: the request stream "
                        "through the server; autotune: write the tuning table; merge: "
                        "the device merge of sorted shards (--shards of --n prefixes)")
    p.add_argument("--shards", type=int, default=8, help="merge mode: sorted runs to merge")
    p.add_argument("--merge-piece", type=int, default=0,
                   help="merge mode: outputs per thread of a merge round (0: library default)")
    p.add_argument("--duration", type=float, default=60.0, help="serving: seconds of arrivals")
    p.add_argument("--rate", type=float, default=2000.0, help="serving: requests per second")
    p.add_argument("--budget-gb", type=float, default=40.0, help="serving: HBM budget")
    p.add_argument("--sample-instances", type=int, default=1000,
                   help="batched mode: instances timed one call each")
    return p.parse_args()


def workload_config(n: int, nchars, workload: str = "prefixes") -> dict:
    if workload == "digits":
        return {"workload": "digits-10MiB", "strings": n, "chars": nchars,
                "lengths": "U[1,40]", "alphabet": "0-9", "seed": 1,
                "l2": "256 MB written between timed steps (inputs fit in L2)",
                "lcp_output": False}
    if workload == "dna":
        return {"workload": "dna-suffixes-32MiB", "strings": n, "chars": nchars,
                "text": "32 MiB uniform ACGT, 5% overwritten by copies of earlier 1-10 KiB blocks",
                "seed": 3, "l2": "256 MB written between timed steps",
                "lcp_output": False}
    return {"workload": "prefixes-64Mi" if n == N_DEFAULT else f"prefixes-{n}",
            "strings": n, "chars": nchars, "prefixes": 4096, "prefix_len": 48,
            "zipf_s": 1.1, "suffix_len": "U[8,24]", "alphabet": "a-z", "seed": SEED,
            "l2": "inputs larger than L2 (126 MB)", "lcp_output": False}


def make_workload(pkg, workload: str, n: int, seed_offset: int = 0, alloc=None):
    """(chars, offs, nchars) of a sort-mode workload; n applies to prefixes."""
    kw = {} if alloc is None else {"alloc": alloc}
    if workload == "digits":
        return pkg.workloads.digits(seed=1 + seed_offset, **kw)
    if workload == "dna":
        return pkg.workloads.dna_suffixes(seed=3 + seed_offset, **kw)
    return pkg.workloads.prefixes(n=n, seed=SEED + seed_offset, **kw)


def profiled_traffic(kernel: str, workload: str, n: int):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/classify_prefixes.md), for the prefix workload at its
    bench size; None otherwise."""
    if kernel != "classify" or workload != "prefixes" or n != N_DEFAULT:
        return None
    f = ROOT / "profiles" / "classify_prefixes.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch_64Mi:"):
            return int(line.split(":")[1])
    return None


def measured_peak() -> tuple:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of one GPU during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                maxs.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sms) if sms else None,
                "sm_max_mhz": max(maxs) if maxs else None,
                "samples": len(sms), "reasons": sorted(reasons)}


class Ranks:
    """The replicas of a multi-GPU run: one process per GPU, each sorting its
    own instance. The only collectives are the timing ones: a barrier around
    the timed region, the maximum of the per-rank step times and the sum of
    the ranks' chars. device is "cuda" under NCCL, "cpu" under gloo."""

    def __init__(self, dist, world: int, device: str = "cuda"):
        self.dist, self.world, self.device = dist, world, device

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def allmax(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.MAX)

    def allsum(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.SUM)


def replica_value(ranks: Ranks, chars: int, ms: float) -> tuple:
    """Whole-job char GB/s of a replica run: every rank's chars over the
    slowest rank's step time. Returns (value, ms_max, total_chars)."""
    ms_max = ranks.allmax(ms)
    total = ranks.allsum(float(chars))
    return total / (ms_max / 1e3) / 1e9, ms_max, total


def offset_wire_bytes(offs) -> int:
    """Bytes of an offset array that cross PCIe in pssgpu_sort_host: 1- or
    2-byte gaps for 2^20 or more offsets that never decrease with every gap
    below 65536 (the library rebuilds them on the device), else 8 each."""
    n = len(offs)
    if n < (1 << 20):
        return 8 * n
    o = offs.view(np.int64)
    top = 0
    for i in range(0, n - 1, 1 << 24):
        d = np.diff(o[i:min(i + (1 << 24) + 1, n)])
        if d.size and d.min() < 0:
            return 8 * n
        top = max(top, int(d.max()) if d.size else 0)
    return n if top < 256 else 2 * n if top < 65536 else 8 * n


def pinned_alloc(torch):
    def alloc(nbytes, dtype):
        t = torch.empty(int(nbytes), dtype=torch.uint8, pin_memory=True)
        return t.numpy().view(dtype)
    return alloc


def ref_time(chars, offs, nchars: int, reps: int, warmup: int = 0):
    """The reference pS5 (parallel_sample_sortBTCUI, built from the reference
    sources into oracle/_ref) on the given arena with every host thread:
    `warmup` untimed sorts, then `reps` timed ones (each on a fresh copy of
    the unsorted pointer array, copied outside the timer). Returns (list of
    seconds, threads), or None when the library is not built."""
    from oracle import oracle as orc
    if not orc.ref_available():
        return None
    threads = os.cpu_count()
    lib = orc.ref_lib()
    lib.ps5ref_set_threads(threads)
    base = orc.ref_pointer_array(chars, offs)
    n = base.shape[0]
    ptrs = np.empty_like(base)
    times = []
    for i in range(warmup + reps):
        np.copyto(ptrs, base)
        t0 = time.perf_counter()
        lib.ps5ref_sort(ptrs.ctypes.data, n)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    return times, threads


def cpu_baseline(chars, offs, nchars: int) -> dict:
    """Reference pS5 on the same input the GPU arm sorts (the whole instance),
    every host thread, best of 3."""
    r = ref_time(chars, offs, nchars, reps=3)
    if r is None:
        return {"value": None, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "oracle/_ref/libps5ref.so not built"}
    times, threads = r
    t = min(times)
    n = offs.shape[0]
    return {"value": nchars / t / 1e9, "unit": "GB/s", "cores": threads, "kind": "reference",
            "sample": f"the whole instance: {n} strings, {nchars} chars; pS5-Unroll "
                      f"(parallel_sample_sortBTCUI) best of 3: {t * 1e3:.1f} ms",
            "strings_per_s": n / t}


def run_reference(args):
    """The reference arm: pS5 from the reference sources on the host cores,
    on the same workload and config as the GPU arm, the same warm-up and step
    counts, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as orc
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    if not orc.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libps5ref.so (reference pS5 built from its sources) missing"}))
        return
    chars, offs, nchars = make_workload(pkg, args.workload, args.n)
    n = offs.shape[0]
    times, threads = ref_time(chars, offs, nchars, reps=args.steps, warmup=args.warmup)
    t = sum(times) / len(times)
    value = nchars / t / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic", "config": workload_config(n, nchars, args.workload),
        "impl": "reference",
        "strings_per_s": n / t,
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "reference",
                         "sample": f"the whole instance ({n} strings, {nchars} chars) every "
                                   "step; pS5-Unroll (parallel_sample_sortBTCUI) from the "
                                   "reference sources, every host thread"},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_autotune():
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    from importlib import import_module
    at = import_module("pss_b200.autotune")
    res = at.tune()
    at.save_table(res)
    print(json.dumps({"mode": "autotune", "table": res["table"]}))


def run_merge(args):
    """The reference's top-level composition, sorted shards merged into one
    sorted sequence with its LCP array (eberle-ps5-parallel-toplevel-merge),
    on one GPU: --shards contiguous shards of the prefix workload are sorted
    with LCP output, then each timed step merges them on the device."""
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    n_req = args.n if args.n != N_DEFAULT else 16 * 1024 * 1024
    chars, offs, nchars = pkg.workloads.prefixes(n=n_req, seed=SEED)
    n = offs.shape[0]
    ctx = pkg.Context(0)
    dc = torch.from_numpy(chars).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    bounds = np.linspace(0, n, args.shards + 1).astype(np.uint64)
    ids = torch.empty(n, dtype=torch.int32, device="cuda")
    lcp = torch.zeros(n, dtype=torch.int32, device="cuda")
    for k in range(args.shards):
        b, e = int(bounds[k]), int(bounds[k + 1])
        ctx.sort_device(dc, nchars, do[b:e], ids[b:e], lcp[b:e])
        ids[b:e] += b
    out = torch.empty_like(ids)
    out_lcp = torch.zeros_like(lcp)
    # a stream of its own (not the legacy default stream, which the library
    # reads as "the context's stream"): the merges and the events share it
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    if args.merge_piece:
        ctx.set_option(ctx.OPT_MERGE_PIECE, args.merge_piece)

    def step():
        ctx.merge_lcp_device(dc, nchars, do, bounds, ids, lcp, out, out_lcp, stream=stream)

    def sort_all():  # the same strings sorted outright, with their LCP array
        ctx.sort_device(dc, nchars, do, sort_ids, sort_lcp, stream=stream)

    def timed(fn):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps
    ms = timed(step)
    sort_ids, sort_lcp = torch.empty_like(ids), torch.zeros_like(lcp)
    sort_ms = timed(sort_all)
    print(json.dumps({
        "mode": "merge", "metric": "merged char GB/s", "value": nchars / (ms / 1e3) / 1e9,
        "unit": "GB/s", "ms_per_step": ms, "steps": args.steps, "warmup": max(args.warmup, 3),
        "higher_is_better": True, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"prefixes-{n}", "strings": n, "chars": nchars,
                   "shards": args.shards, "lcp_output": True,
                   "merge_piece": args.merge_piece or "default"},
        "strings_per_s": n / (ms / 1e3),
        "sort_with_lcp_ms": sort_ms, "merge_over_sort": ms / sort_ms}))
    ctx.close()


def run_batched(args, emit: bool = True) -> dict:
    """The batched workload (100k instances, <= 1 GiB of chars) sorted by one
    batched call, against one pssgpu_sort_device call per instance timed on a
    random sample of instances and scaled to all instances. The batched
    output is checked against the single-instance sorts of the sample."""
    import torch
    import __graft_entry__
    from importlib import import_module
    pkg = __graft_entry__.load_package()
    at = import_module("pss_b200.autotune")
    canonical_ids = pkg.workloads.canonical_ids
    alloc = pinned_alloc(torch)
    t0 = time.perf_counter()
    h_chars, h_offs, nchars, inst = pkg.workloads.batched(alloc=alloc)
    gen_s = time.perf_counter() - t0
    n = len(h_offs)
    ninst = len(inst) - 1
    ctx = pkg.Context(0)
    table = at.load_table()
    # the sorts and the events on one stream of their own
    stream = torch.cuda.Stream()
    dc = torch.from_numpy(h_chars).cuda()
    do = torch.from_numpy(h_offs.view(np.int64)).cuda()
    dp = torch.empty(n, dtype=torch.int32, device="cuda")
    dl = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()

    def timed(fn, reps):
        ms = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms

    def batch():
        ctx.sort_batch_device(dc, nchars, do, inst, dp, dl, stream=stream)

    res = {}
    for name, tb in (("default", None), ("tuned", table)):
        if name == "tuned" and tb is None:
            continue
        ctx.set_tree_bits(tb if tb is not None else [0] * 33)
        for _ in range(max(args.warmup, 3)):
            batch()
        ms = timed(batch, args.steps)
        res[name] = {"ms": statistics.median(ms), "ms_all": ms,
                     "launches": ctx.stats()["kernel_launches"]}
    best_name = min(res, key=lambda k: res[k]["ms"])
    best = res[best_name]
    ctx.set_tree_bits(table if best_name == "tuned" else [0] * 33)
    clocks = Clocks(0)
    clocks.start()
    time.sleep(0.2)
    ms_best = timed(batch, max(args.steps, 10))
    clk = clocks.stop()
    batch()  # output of the best configuration for the comparison
    perm_b = dp.cpu().numpy().view(np.uint32)
    lcp_b = dl.cpu().numpy().view(np.uint32)

    # one call per instance on a random sample of instances
    lens_all = pkg.workloads.string_lengths(h_chars[: nchars + 1], h_offs)
    rng = np.random.default_rng(0)
    sample = rng.choice(ninst, min(args.sample_instances, ninst), replace=False)
    p1 = torch.empty(int((inst[1:] - inst[:-1]).max()), dtype=torch.int32, device="cuda")
    l1 = torch.empty_like(p1)
    single_ms = 0.0
    identical = True
    for k in sample:
        b, e = int(inst[k]), int(inst[k + 1])
        ms = timed(lambda: ctx.sort_device(dc, nchars, do[b:e], p1, l1, stream=stream), 1)[0]
        single_ms += ms
        pp = p1[: e - b].cpu().numpy().view(np.uint32)
        ll = l1[: e - b].cpu().numpy().view(np.uint32)
        offs_k = h_offs[b:e]
        lens_k = lens_all[b:e]
        if not (np.array_equal(ll[1:], lcp_b[b + 1:e]) and np.array_equal(
                canonical_ids(h_chars, offs_k, pp, ll, lens_k),
                canonical_ids(h_chars, offs_k, perm_b[b:e], lcp_b[b:e], lens_k))):
            identical = False
    per_instance_ms = single_ms * ninst / len(sample)
    med = statistics.median(ms_best)
    line = {"mode": "batched", "metric": "batched sort time", "unit": "ms",
            "config": {"workload": "batched-100k", "instances": ninst, "strings": n,
                       "chars": nchars, "sizes": "log-uniform 16..1Mi, scaled to <= 1 GiB",
                       "lengths": "lognormal(3, 0.5) clipped 1..256", "alphabet": "32..126",
                       "inputs": "resident in HBM (1 GiB of chars > L2)",
                       "lcp_output": True},
            "batched_ms": med, "batched_ms_p99": float(np.percentile(ms_best, 99)),
            "batched_steps": len(ms_best), "tree_bits": best_name, "configs": res,
            "char_gb_s": nchars / (med / 1e3) / 1e9,
            "per_instance_ms_est": per_instance_ms,
            "per_instance_sample": len(sample),
            "speedup_vs_per_instance": per_instance_ms / med,
            "identical_output_on_sample": identical, "generate_s": gen_s, "clocks": clk}
    if emit:
        print(json.dumps(line))
    ctx.close()
    return line


def run_serving(args, duration=None, emit: bool = True) -> dict:
    """The serving stream: Poisson arrivals at --rate for --duration seconds,
    sizes log-uniform 1 KB..64 MB, alphabets {4, 10, 26, 95}, lengths
    U[1, 64], through the continuous-batching server under --budget-gb."""
    duration = args.duration if duration is None else duration
    import torch
    import __graft_entry__
    from importlib import import_module
    __graft_entry__.load_package()
    serving = import_module("pss_b200.serving")
    alloc = pinned_alloc(torch)
    t0 = time.perf_counter()
    pools = serving.make_pools(bytes_per_pool=512 << 20, alloc=alloc)
    t1 = time.perf_counter()
    reqs = serving.make_stream(pools, rate=args.rate, duration=duration)
    t2 = time.perf_counter()
    srv = serving.Server(budget=int(args.budget_gb * (1 << 30)), workers=3,
                         max_batch_strings=8 << 20)
    # results land in slots of one pinned, reused buffer, as the inputs come
    # from pinned pools (a fresh pageable array per request makes every
    # device-to-host copy fault in untouched pages: p50 4.5 ms, p99 13.7 ms
    # instead of 1.1 / 5.5 on the same stream)
    ring = serving.ResultRing(64 << 20, alloc=alloc)
    # warm the workers' kernels with a short burst
    serving.run_stream(srv, pools, serving.make_stream(pools, rate=2000, duration=0.05, seed=1),
                       results=ring)
    t3 = time.perf_counter()
    print(json.dumps({"pools_s": t1 - t0, "stream_s": t2 - t1, "server_warm_s": t3 - t2,
                      "requests": len(reqs)}), file=sys.stderr, flush=True)
    clocks = Clocks(0)
    clocks.start()
    res = serving.run_stream(srv, pools, reqs, results=ring)
    clk = clocks.stop()
    st = srv.stats()
    srv.close()
    line = {"mode": "serving", "metric": "request latency and sustained char GB/s",
            "config": {"workload": "serving-poisson", "rate_per_s": args.rate,
                       "duration_s": duration, "request_bytes": "log-uniform 1 KB..64 MB",
                       "alphabets": [4, 10, 26, 95], "lengths": "U[1,64]",
                       "hbm_budget_gb": args.budget_gb, "workers": 3,
                       "max_batch_strings": 8 << 20,
                       "result_buffers": "slots of one pinned 64 Mi-entry ring, reused"},
            **res, "batches": st["batches"], "slab_gb": st["slab_bytes"] / 2**30,
            "slab_peak_gb": st["slab_peak_bytes"] / 2**30, "clocks": clk}
    if emit:
        print(json.dumps(line))
    return line


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.mode == "serving":
        run_serving(args)
        return
    if args.mode == "autotune":
        run_autotune()
        return
    if args.mode == "batched":
        run_batched(args)
        return
    if args.mode == "merge":
        run_merge(args)
        return
    import torch
    import torch.distributed as dist
    import __graft_entry__
    pkg = __graft_entry__.load_package()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    ranks = Ranks(dist, world, "cuda")
    barrier = ranks.barrier
    allmax = ranks.allmax

    alloc = pinned_alloc(torch)
    h_chars, h_offs, nchars = make_workload(pkg, args.workload, args.n, rank, alloc)
    n = h_offs.shape[0]
    # inputs that fit in L2 are evicted between timed steps by writing a
    # buffer twice the L2 size (outside the timed events)
    flush = None if args.workload == "prefixes" else torch.empty(256 << 20, dtype=torch.uint8,
                                                                  device="cuda")
    ctx = pkg.Context(local)
    # the sorts, the L2 flush and the timing events on one stream of their
    # own (the legacy default stream reads as "the context's stream" in the
    # library, which would put the sort on another stream than the events)
    stream = torch.cuda.Stream(device=local)
    d_chars = torch.from_numpy(h_chars).cuda(non_blocking=True)
    d_offs = torch.from_numpy(h_offs.view(np.int64)).cuda(non_blocking=True)
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    d_lcp = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()

    def step(lcp=None):
        ctx.sort_device(d_chars, nchars, d_offs, d_perm, lcp, stream=stream)

    for _ in range(max(args.warmup, 3)):
        step()
    # untimed: one LCP-emitting sort for the method's algorithmic bytes
    step(d_lcp)
    lcp_host = d_lcp.cpu().numpy().view(np.uint32)
    model = pkg.workloads.alg_bytes(lcp_host)

    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    launches = 0
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if flush is None:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
            launches += ctx.stats()["kernel_launches"]
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
    else:
        tot = 0.0
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            ev0.record(stream)
            step()
            ev1.record(stream)
            torch.cuda.synchronize()
            tot += ev0.elapsed_time(ev1)
            launches += ctx.stats()["kernel_launches"]
        ms = tot / args.steps
    barrier()
    clk = clocks.stop()

    # the last timed sort's output, checked once on the host (outside the
    # timed region): a permutation of the ids in strcmp order of the strings
    t_v = time.perf_counter()
    h_check = d_perm.cpu().numpy().view(np.uint32)
    verified = bool(pkg.workloads.check_permutation(h_check)) and \
        pkg.workloads.check_sorted(h_chars, nchars, h_offs, h_check) == -1
    verify_s = time.perf_counter() - t_v
    del h_check

    # per-kernel-class split (profile mode: classes run one after another on
    # the stream, each between CUDA events), outside the timed region
    ctx.set_profile(True)
    kstats = {}
    for _ in range(args.steps):
        step()
        for k in ctx.kernel_stats():
            a = kstats.setdefault(k["name"], {"launches": 0, "strings": 0, "alg_bytes": 0, "ms": 0.0})
            for f in ("launches", "strings", "alg_bytes", "ms"):
                a[f] += k[f]
    torch.cuda.synchronize()
    ctx.set_profile(False)
    value, ms_max, total_chars = replica_value(ranks, nchars, ms)

    # end to end through the C ABI: host arena in, host permutation out
    h_perm = alloc(4 * n, np.uint32)
    ctx.sort_host(h_chars[:nchars], h_offs, lcp=False, out_perm=h_perm)  # warm
    e2e_times = []
    for _ in range(args.e2e_steps):
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.sort_host(h_chars[:nchars], h_offs, lcp=False, out_perm=h_perm)
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = allmax(sum(e2e_times) / max(len(e2e_times), 1))
    e2e_value = total_chars / e2e_s / 1e9 if e2e_s > 0 else None
    del h_perm

    peak, peak_kind = measured_peak()
    dom = max(kstats.items(), key=lambda kv: kv[1]["ms"])
    dom_name, d = dom
    achieved = d["alg_bytes"] / (d["ms"] / 1e3) / 1e9 if d["ms"] > 0 else 0.0
    sort_achieved = model["total"] / (ms / 1e3) / 1e9
    tot_ms = sum(v["ms"] for v in kstats.values())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(h_chars, h_offs, nchars)

    # the same end to end through the text entry point: only the text goes to
    # the device (no offset array) and is split there, as psstest's loader
    # splits a file (lines; suffixes for the DNA workload). The host arena
    # becomes that text in place (NUL -> newline), after every other use.
    e2e_text = None
    if args.e2e_steps > 0:
        import ctypes
        mode = 1 if args.workload == "dna" else 0
        if mode == 0:
            for i in range(0, nchars, 1 << 28):
                seg = h_chars[i:min(i + (1 << 28), nchars)]
                seg[seg == 0] = 10
        h_perm = alloc(4 * n, np.uint32)
        nout = ctypes.c_uint64(0)
        lib = pkg._native.gpu()

        def text_step():
            rc = lib.pssgpu_sort_text_host(ctx._h, h_chars.ctypes.data, nchars, mode,
                                           h_perm.ctypes.data, None, n, ctypes.byref(nout))
            if rc or nout.value != n:
                raise RuntimeError(f"pssgpu_sort_text_host: status {rc}, {nout.value} strings")
        text_step()  # warm
        t_times = []
        for _ in range(args.e2e_steps):
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            text_step()
            t_times.append(time.perf_counter() - t0)
        t_s = allmax(sum(t_times) / len(t_times))
        e2e_text = {"value": total_chars / t_s / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nchars,
                    "d2h_bytes_per_step": 4 * n, "ms_per_step": t_s * 1e3,
                    "entry": "pssgpu_sort_text_host, " + ("suffixes" if mode else "lines")}
        del h_perm

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic", "config": workload_config(n, nchars, args.workload),
            "strings_per_s": world * n / (ms_max / 1e3),
            "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": nchars + 8 * n,
                    "d2h_bytes_per_step": 4 * n, "ms_per_step": e2e_s * 1e3,
                    "h2d_wire_bytes_per_step": nchars + offset_wire_bytes(h_offs)},
            "e2e_text": e2e_text,
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profiled_traffic(dom_name, args.workload, n),
                         "peak_kind": peak_kind,
                         "alg_bytes_per_launch": d["alg_bytes"] / max(d["launches"], 1),
                         "ms_per_launch": d["ms"] / max(d["launches"], 1),
                         "share_of_device_time": d["ms"] / tot_ms if tot_ms else None},
            "roofline_sort": {"alg_bytes": model["total"], "achieved": sort_achieved,
                              "frac": sort_achieved / peak, "max_round": model["max_round"]},
            "kernels_serial_ms_per_step": tot_ms / args.steps,
            "kernels": {k: {"ms_per_step": v["ms"] / args.steps,
                            "launches_per_step": v["launches"] / args.steps,
                            "gb_s": v["alg_bytes"] / (v["ms"] / 1e3) / 1e9 if v["ms"] else None}
                        for k, v in kstats.items()},
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
            "verified": verified,
            "verified_how": "permutation of the last timed sort's ids and strcmp order of "
                            f"every neighbouring pair, on the host ({verify_s:.1f} s)",
        }
    ctx.close()
    del d_chars, d_offs, d_perm, d_lcp
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and args.workload == "prefixes" and not args.no_extras:
        # the other two patterns of the metric, on the same GPU after the
        # headline's buffers are freed: the 100k-instance batched sort and a
        # shortened serving stream (p50 / p99 request latency)
        del h_chars, h_offs
        b = run_batched(args, emit=False)
        line["batched"] = {k: b[k] for k in (
            "batched_ms", "batched_ms_p99", "batched_steps", "char_gb_s", "per_instance_ms_est",
            "per_instance_sample", "speedup_vs_per_instance", "identical_output_on_sample",
            "tree_bits", "config", "clocks")}
        torch.cuda.empty_cache()
        sv = run_serving(args, duration=args.serving_duration, emit=False)
        line["serving"] = {k: sv[k] for k in sv if k not in ("mode", "metric")}
        line["serving_p99_ms"] = sv.get("p99_ms")
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
