"""CPU test of bench.py's multi-GPU path with two gloo ranks: each rank is
a replica that sorts its own instance (seed + rank), and the job's value is
all ranks' chars over the slowest rank's time, with no other collective."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys
    from pathlib import Path
    import torch.distributed as dist
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import __graft_entry__
        pkg = __graft_entry__.load_package()
        ranks = bench.Ranks(dist, world, "cpu")
        # each replica generates its own instance (seed + rank)
        chars, offs, nchars = bench.make_workload(pkg, "prefixes", 20000, rank)
        ms = [3.0, 5.0][rank]  # per-rank step times
        ranks.barrier()
        value, ms_max, total = bench.replica_value(ranks, nchars, ms)
        out.put((rank, nchars, int(chars[: 64].sum()), value, ms_max, total))
    finally:
        dist.destroy_process_group()


def test_two_replicas_over_gloo(pkg):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, n0, h0, v0, m0, t0), (r1, n1, h1, v1, m1, t1) = res
    assert h0 != h1  # different instances
    assert m0 == m1 == 5.0  # the slowest rank's time
    assert t0 == t1 == float(n0 + n1)
    assert v0 == pytest.approx((n0 + n1) / 5e-3 / 1e9)
    assert v0 == v1
