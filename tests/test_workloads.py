"""CPU tests of the host logic: the seeded workload generators have the
documented shapes and are deterministic, and the algorithmic-byte model
matches a hand count."""
import numpy as np

from golden_util import string_lengths


def test_digits_shape(pkg):
    chars, offs, nchars = pkg.workloads.digits(seed=1)
    n = len(offs)
    assert 480_000 < n < 495_000
    assert nchars <= 10 * 1024 * 1024
    lens = string_lengths(chars[:nchars + 1], offs)
    assert lens.min() >= 1 and lens.max() <= 40
    body = chars[:nchars]
    assert set(np.unique(body).tolist()) <= set(range(48, 58)) | {0}
    c2, o2, n2 = pkg.workloads.digits(seed=1)
    assert n2 == nchars and np.array_equal(c2, chars) and np.array_equal(o2, offs)


def test_prefix_shape(pkg):
    chars, offs, nchars, ids = pkg.workloads.prefixes(n=200000, seed=2, with_ids=True)
    lens = string_lengths(chars, offs)
    assert lens.min() >= 56 and lens.max() <= 72
    counts = np.bincount(ids, minlength=4096)
    h = np.sum(np.arange(1, 4097, dtype=np.float64) ** -1.1)
    assert abs(counts[0] / len(ids) - 1 / h) < 0.01
    assert len(np.unique(ids)) > 3000


def test_dna_text(pkg):
    t = pkg.workloads.dna_text(length=1 << 20, seed=3)
    assert t[1 << 20] == 0
    assert set(np.unique(t[: 1 << 20]).tolist()) == {65, 67, 71, 84}
    t2 = pkg.workloads.dna_text(length=1 << 20, seed=3)
    assert np.array_equal(t, t2)


def test_random_strings_deterministic(pkg):
    a = pkg.workloads.random_strings(1000, 0, 9, b"xyz", seed=1)
    b = pkg.workloads.random_strings(1000, 0, 9, b"xyz", seed=1)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_batch_sizes_cap(pkg):
    sizes, f = pkg.workloads.batch_sizes()
    assert len(sizes) == 100_000
    assert sizes.min() == 16
    assert 0 < f < 1  # the 1 GiB cap binds: about 200 GB uncapped
    assert sizes.sum() * 23.8 <= (1 << 30)
    assert sizes.sum() * 23.8 > 0.95 * (1 << 30)


def test_batched_small(pkg):
    chars, offs, nchars, inst = pkg.workloads.batched(ninst=100, budget_chars=1 << 20, seed=1)
    assert len(inst) == 101 and inst[0] == 0 and inst[-1] == len(offs)
    lens = string_lengths(chars, offs)
    assert lens.min() >= 1 and lens.max() <= 256
    body = chars[:nchars]
    assert set(np.unique(body).tolist()) <= set(range(32, 127)) | {0}


def test_serving_stream_and_driver_with_a_fake_server(pkg):
    """Host logic of the serving driver (arrivals, request cutting, the
    submit / wait hand-off, latency figures) against a server stand-in."""
    from importlib import import_module
    serving = import_module("pss_b200.serving")
    pools = serving.make_pools(bytes_per_pool=1 << 20, seed=1)
    reqs = serving.make_stream(pools, rate=2000, duration=0.05, min_bytes=1 << 10,
                               max_bytes=64 << 10, seed=2)
    assert len(reqs) > 40
    for r in reqs:
        p = pools[r.alphabet]
        assert r.i1 > r.i0
        assert p.chars[r.start + r.nchars - 1] == 0  # the request ends with a NUL
        assert int(p.offs[r.i0]) == r.start

    class FakeServer:
        def __init__(self):
            self.t = {}

        def submit(self, ptr, nchars, offs, base, perm, lcp):
            k = len(self.t) + 1
            perm[:] = np.arange(perm.shape[0], dtype=np.uint32)
            self.t[k] = 1000 * k
            return k

        def wait(self, ticket):
            t = self.t[ticket]
            return {"status": 0, "batch_requests": 1, "batch_strings": 1,
                    "t_submit_ns": t, "t_admit_ns": t, "t_start_ns": t + 10,
                    "t_done_ns": t + 2_000_000}

    res = serving.run_stream(FakeServer(), pools, reqs, want_lcp=True)
    assert res["requests"] == len(reqs)
    assert abs(res["p50_ms"] - 2.0) < 1e-9 and abs(res["p99_ms"] - 2.0) < 1e-9


def test_alg_bytes_hand_count(pkg):
    # 40 strings tied at depth 0 (one group > 32) splitting into singletons
    lcp = np.zeros(40, np.uint32)
    r = pkg.workloads.alg_bytes(lcp, T=32)
    assert r["rounds"] == 52 * 40
    # every string enters the base case at depth 8 and needs 1 char: none left
    assert r["base"] == 40 * 12
    assert r["total"] == 52 * 40 + 40 * 12 + 8 * 40
    # a group of 10 enters the base case at depth 0 and needs lcp+1 chars
    lcp = np.array([0, 3, 3, 5, 0, 0, 0, 0, 0, 0], np.uint32)
    r = pkg.workloads.alg_bytes(lcp, T=32)
    need = [4, 4, 6, 6, 1, 1, 1, 1, 1, 1]
    assert r["rounds"] == 0
    assert r["base"] == sum(12 + x for x in need)


def test_bench_output_checks_catch_planted_mistakes(pkg, orc):
    """The checks bench.py runs on its timed output: a correct sort passes; a
    swapped pair, a duplicated id and an out-of-range id are caught."""
    w = pkg.workloads
    chars, offs, nchars = w.random_strings(5000, 0, 9, b"abc", 31)
    ids = orc.sort_ids(chars[:nchars], offs)
    assert w.check_permutation(ids) and w.check_sorted(chars, nchars, offs, ids) == -1
    # a swap of two different neighbours (the first pair that differs)
    lcp = orc.lcp_array(chars, offs, ids)
    lens = w.string_lengths(chars[:nchars + 1], offs)[ids]
    p = next(i for i in range(1, len(ids)) if not (lcp[i] == lens[i] == lens[i - 1]))
    bad = ids.copy()
    bad[p - 1], bad[p] = bad[p], bad[p - 1]
    assert w.check_permutation(bad) and w.check_sorted(chars, nchars, offs, bad) == p
    dup = ids.copy()
    dup[7] = dup[8]
    assert not w.check_permutation(dup)
    oob = ids.copy()
    oob[11] = len(ids)
    assert not w.check_permutation(oob)
    assert w.check_sorted(chars, nchars, offs, oob) == 11
