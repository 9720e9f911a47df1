"""GPU tests of the batched entry point: many independent instances in one
call give, per instance, the same sorted sequence and LCP array as the
oracle and as a separate single-instance sort."""
import numpy as np
import pytest

from golden_util import canonical_ids

pytestmark = pytest.mark.gpu


def split_instance(chars, offs, inst, k):
    b, e = int(inst[k]), int(inst[k + 1])
    return offs[b:e]


def check_instance(orc, chars, offs_k, perm_k, lcp_k):
    ids, rlcp = orc.sort_ids_lcp(chars, offs_k)
    assert orc.check_permutation(perm_k)
    assert np.array_equal(canonical_ids(chars, offs_k, perm_k, lcp_k),
                          canonical_ids(chars, offs_k, ids, rlcp))
    if len(offs_k) > 1:
        assert np.array_equal(lcp_k[1:].astype(np.uint64), rlcp[1:])
    if len(offs_k):
        assert lcp_k[0] == 0


def mixed_batch(pkg, sizes, seed):
    chars, offs, nchars = pkg.workloads.random_strings(int(sum(sizes)), 0, 20, b"abcd", seed)
    inst = np.zeros(len(sizes) + 1, dtype=np.uint64)
    np.cumsum(np.asarray(sizes, dtype=np.uint64), out=inst[1:])
    return chars, offs, nchars, inst


def test_batch_mixed_sizes_vs_oracle(pkg, orc, ctx):
    sizes = [0, 1, 2, 5, 33, 300, 2049, 5000, 40000, 0, 17]
    chars, offs, nchars, inst = mixed_batch(pkg, sizes, 41)
    perm, lcp = ctx.sort_batch_host(chars, offs, inst, lcp=True)
    for k in range(len(sizes)):
        b, e = int(inst[k]), int(inst[k + 1])
        check_instance(orc, chars, offs[b:e], perm[b:e], lcp[b:e])


def test_batch_equals_single_sorts(pkg, ctx):
    sizes = [3, 700, 64, 2500, 1, 9000, 31, 32, 256, 257]
    chars, offs, nchars, inst = mixed_batch(pkg, sizes, 42)
    perm, lcp = ctx.sort_batch_host(chars, offs, inst, lcp=True)
    for k in range(len(sizes)):
        b, e = int(inst[k]), int(inst[k + 1])
        p1, l1 = ctx.sort_host(chars, offs[b:e], lcp=True)
        assert np.array_equal(canonical_ids(chars, offs[b:e], perm[b:e], lcp[b:e]),
                              canonical_ids(chars, offs[b:e], p1, l1))
        if e - b > 1:
            assert np.array_equal(lcp[b + 1:e], l1[1:])


def test_batched_workload_sample(pkg, orc, ctx):
    chars, offs, nchars, inst = pkg.workloads.batched(ninst=3000, budget_chars=8 << 20, seed=5)
    perm, lcp = ctx.sort_batch_host(chars[:nchars], offs, inst, lcp=True)
    rng = np.random.default_rng(0)
    for k in rng.choice(len(inst) - 1, 60, replace=False):
        b, e = int(inst[k]), int(inst[k + 1])
        check_instance(orc, chars, offs[b:e], perm[b:e], lcp[b:e])


def test_batch_tuning_table_keeps_output(pkg, ctx):
    sizes = [5000, 20000, 3000]
    chars, offs, nchars, inst = mixed_batch(pkg, sizes, 43)
    p0, l0 = ctx.sort_batch_host(chars, offs, inst, lcp=True)
    c2 = pkg.Context(0)
    try:
        c2.set_tree_bits([0] * 11 + [3, 9, 5, 10, 2] + [0] * 17)
        p1, l1 = c2.sort_batch_host(chars, offs, inst, lcp=True)
    finally:
        c2.close()
    assert np.array_equal(l0, l1)
    for k in range(len(sizes)):
        b, e = int(inst[k]), int(inst[k + 1])
        assert np.array_equal(canonical_ids(chars, offs[b:e], p0[b:e], l0[b:e]),
                              canonical_ids(chars, offs[b:e], p1[b:e], l1[b:e]))


def test_batch_rejects_bad_boundaries(pkg, ctx):
    chars, offs, nchars, inst = mixed_batch(pkg, [4, 4], 44)
    bad = inst.copy()
    bad[1] = 9  # beyond n
    with pytest.raises(pkg.SortError):
        ctx.sort_batch_host(chars, offs, bad)
