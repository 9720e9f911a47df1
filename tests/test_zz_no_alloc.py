"""GPU test of the allocation-free entry point pssgpu_sort_device_noalloc.

That entry point serves callers that cannot allocate device memory (a plugin
whose host application owns every byte of device memory through its own pool,
a latency-critical path that cannot take cudaMalloc's implicit device
synchronisation, a process whose device memory is fully reserved). It sorts up
to 2048 strings using a fixed scratch array inside the library instead of a
workspace. This test calls it through the C ABI twice in a row on every case
and checks each result bit-exactly against the oracle and against the
context-based pssgpu_sort_device on the same device buffers, then checks that
a size above the limit is rejected. The cases include 1, 2 and 33 strings and
a 40-string group that shares a 600-char prefix (the sorter's common-prefix
jump, with no deep-group list behind it).

The file name makes pytest collect it last, so a run that stops at the first
failure has already run every other test.
"""
import numpy as np
import pytest

from golden_util import canonical_ids

pytestmark = pytest.mark.gpu


def _dev(torch, a, dtype):
    return torch.from_numpy(a.view(dtype)).cuda()


def _long_prefix_case(pkg):
    """40 strings behind one 600-char prefix among 1000 random ones."""
    rnd = np.random.default_rng(24)
    strings = [b"q" * 600 + bytes(rnd.integers(97, 100, rnd.integers(0, 6)).astype(np.uint8))
               for _ in range(40)]
    strings += [bytes(rnd.integers(97, 100, rnd.integers(0, 20)).astype(np.uint8))
                for _ in range(1000)]
    order = rnd.permutation(len(strings))
    chars, offs = pkg.pack_strings([strings[i] for i in order])
    nchars = chars.shape[0]
    return np.concatenate([chars, np.zeros(16, np.uint8)]), offs, nchars


def _cases(pkg):
    for seed, n, alpha, lmax in ((21, 2048, b"abc", 24), (22, 1500, b"ab", 24),
                                 (25, 1, b"ab", 5), (26, 2, b"ab", 3), (27, 33, b"ab", 9)):
        yield f"random-{n}", pkg.workloads.random_strings(n, 0, lmax, alpha, seed)
    yield "prefix600-x40", _long_prefix_case(pkg)


def test_noalloc_matches_oracle_and_sort_device_twice(pkg, orc):
    import torch
    lib = pkg._native.gpu()
    ctx = pkg.Context(0)
    try:
        for name, (chars, offs, nchars) in _cases(pkg):
            n = len(offs)
            ids, rlcp = orc.sort_ids_lcp(chars[:nchars], offs)
            want = canonical_ids(chars, offs, ids, rlcp)
            dc = _dev(torch, chars, np.uint8)
            do = _dev(torch, offs, np.int64)
            p_ref = torch.empty(n, dtype=torch.int32, device="cuda")
            l_ref = torch.zeros(n, dtype=torch.int32, device="cuda")
            ctx.sort_device(dc, nchars, do, p_ref, l_ref)
            perm_ref = p_ref.cpu().numpy().view(np.uint32)
            lcp_ref = l_ref.cpu().numpy().view(np.uint32)
            for call in range(2):
                p_new = torch.full((n,), -1, dtype=torch.int32, device="cuda")
                l_new = torch.zeros(n, dtype=torch.int32, device="cuda")
                rc = lib.pssgpu_sort_device_noalloc(dc.data_ptr(), nchars, do.data_ptr(), n,
                                                    p_new.data_ptr(), l_new.data_ptr(), None)
                assert rc == 0, (name, call, lib.pssgpu_last_error())
                torch.cuda.synchronize()
                perm_new = p_new.cpu().numpy().view(np.uint32)
                lcp_new = l_new.cpu().numpy().view(np.uint32)
                assert orc.check_permutation(perm_new), (name, call)
                assert np.array_equal(canonical_ids(chars, offs, perm_new, lcp_new), want), \
                    (name, call)
                assert np.array_equal(lcp_new[1:].astype(np.uint64), rlcp[1:]), (name, call)
                assert np.array_equal(lcp_new[1:], lcp_ref[1:]), (name, call)
                assert np.array_equal(canonical_ids(chars, offs, perm_new, lcp_new),
                                      canonical_ids(chars, offs, perm_ref, lcp_ref)), (name, call)
    finally:
        ctx.close()


def test_noalloc_rejects_more_than_its_maximum(pkg):
    import torch
    lib = pkg._native.gpu()
    chars, offs, nchars = pkg.workloads.random_strings(16, 0, 4, b"ab", 23)
    dc = _dev(torch, chars, np.uint8)
    do = _dev(torch, offs, np.int64)
    out = torch.empty(16, dtype=torch.int32, device="cuda")
    rc = lib.pssgpu_sort_device_noalloc(dc.data_ptr(), nchars, do.data_ptr(), 2049,
                                        out.data_ptr(), None, None)
    assert rc == 1  # PSSGPU_EINVAL, nothing launched
    assert b"max 2048" in lib.pssgpu_last_error()
