"""GPU tests of the request server (continuous batching under an HBM budget):
every sampled request's result equals the oracle's sort of that request and
the same request sorted alone, admission waits for slab space instead of
failing, and impossible requests are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def serving(pkg):
    from importlib import import_module
    return import_module("pss_b200.serving")


@pytest.fixture(scope="module")
def pools(serving):
    return serving.make_pools(bytes_per_pool=24 << 20, seed=9)


def alone(pkg, ctx, pool, r):
    chars = pool.chars[r.start:r.start + r.nchars]
    offs = pool.offs[r.i0:r.i1] - np.uint64(r.start)
    return ctx.sort_host(chars, offs, lcp=True), chars, offs


def oracle_ids(orc, chars, offs):
    """The oracle's canonical ids and LCP array of one request."""
    ids, rlcp = orc.sort_ids_lcp(chars, offs)
    from golden_util import canonical_ids
    return canonical_ids(chars, offs, ids, rlcp), rlcp


def test_results_same_alone_and_in_mix(pkg, orc, serving, pools, ctx):
    reqs = serving.make_stream(pools, rate=4000, duration=0.1, min_bytes=1 << 10,
                               max_bytes=2 << 20, seed=3)
    assert len(reqs) > 200
    srv = serving.Server(budget=3 << 30, workers=3, max_batch_strings=1 << 20)
    try:
        res = serving.run_stream(srv, pools, reqs, want_lcp=True)
        st = srv.stats()
    finally:
        srv.close()
    assert res["requests"] == len(reqs)
    assert st["batches"] < len(reqs)  # requests were batched together
    rng = np.random.default_rng(0)
    for k in rng.choice(len(reqs), 40, replace=False):
        r = reqs[k]
        (p1, l1), chars, offs = alone(pkg, ctx, pools[r.alphabet], r)
        assert r.info["status"] == 0
        cw = pkg.workloads.canonical_ids
        want, rlcp = oracle_ids(orc, chars, offs)
        # in the mix: equal to the oracle
        assert np.array_equal(r.lcp[1:].astype(np.uint64), rlcp[1:])
        assert np.array_equal(cw(chars, offs, r.perm, r.lcp), want)
        # alone: equal to the oracle, hence to the result in the mix
        assert np.array_equal(l1[1:].astype(np.uint64), rlcp[1:])
        assert np.array_equal(cw(chars, offs, p1, l1), want)


def test_admission_waits_for_space(pkg, orc, serving, pools, ctx):
    # a budget whose slab holds only a few requests at a time
    srv = serving.Server(budget=160 << 20, workers=2, max_batch_strings=1 << 16)
    try:
        slab = srv.stats()["slab_bytes"]
        reqs = serving.make_stream(pools, rate=20000, duration=0.05, min_bytes=64 << 10,
                                   max_bytes=1 << 20, seed=4)
        reqs = [r for r in reqs if (r.i1 - r.i0) <= (1 << 16)]
        total = sum(r.nchars + 8 * (r.i1 - r.i0) for r in reqs)
        assert total > slab  # more than fits at once
        serving.run_stream(srv, pools, reqs, want_lcp=False)
        st = srv.stats()
        assert st["slab_peak_bytes"] <= slab
    finally:
        srv.close()
    for r in reqs[:20]:
        pool = pools[r.alphabet]
        chars = pool.chars[r.start:r.start + r.nchars]
        offs = pool.offs[r.i0:r.i1] - np.uint64(r.start)
        # equal strings may come in another order: compare the sorted bytes
        # with the oracle's
        ids = orc.sort_ids(chars, offs)
        assert orc.check_permutation(r.perm)
        assert orc.sorted_strings(chars, offs, r.perm) == orc.sorted_strings(chars, offs, ids)


def test_refuses_requests_beyond_the_budget(pkg, serving):
    srv = serving.Server(budget=160 << 20, workers=1, max_batch_strings=1 << 16)
    try:
        n = (1 << 16) + 1
        chars = np.zeros(2 * n, dtype=np.uint8)
        chars[0::2] = 97
        offs = np.arange(0, 2 * n, 2, dtype=np.uint64)
        perm = np.empty(n, dtype=np.uint32)
        with pytest.raises(pkg.SortError) as e:
            srv.submit(chars.ctypes.data, chars.shape[0], offs, 0, perm)
        assert e.value.status == 6  # PSSGPU_EBUDGET
    finally:
        srv.close()

