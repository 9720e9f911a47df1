"""Full-size checks of the benchmarked sort.

The benchmark's headline sorts 64 Mi strings of the prefix workload: 4096
Zipf-chosen 48-char prefixes plus U[8,24]-char suffixes, 4,362,027,854 chars.
That is the only configuration whose arena exceeds 4 GiB: offsets need 33
bits and a packed string handle 33 + 26 = 59 bits. Here that exact input is
sorted as bench.py times it (pssgpu_sort_device on a resident arena, no LCP),
and through the host entry point with the LCP array. Both outputs are checked
by the oracle's order, permutation and LCP-rescan checks. A permutation in
strcmp order whose LCP array rescans equal is the unique sorted string
sequence, so this is the same bar as a comparison with pS5's output, up to
the order of equal strings.

The file name makes pytest collect it after the other parity tests, so a
failure elsewhere is reported first.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_HEADLINE = 64 * 1024 * 1024
CHARS_HEADLINE = 4_362_027_854


@pytest.fixture(scope="module")
def headline(pkg):
    chars, offs, nchars = pkg.workloads.prefixes(n=N_HEADLINE)
    assert nchars == CHARS_HEADLINE and nchars > 1 << 32
    return chars, offs, nchars


def test_headline_device_sort(pkg, orc, ctx, headline):
    import torch
    chars, offs, nchars = headline
    dc = torch.from_numpy(chars).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    dp = torch.empty(N_HEADLINE, dtype=torch.int32, device="cuda")
    ctx.sort_device(dc, nchars, do, dp, None)
    perm = dp.cpu().numpy().view(np.uint32)
    del dc, do, dp
    torch.cuda.empty_cache()
    assert orc.check_permutation(perm)
    assert orc.check_order(chars, offs, perm) == -1
    # the measurement side's own checks (bench.py's "verified") agree
    assert pkg.workloads.check_permutation(perm)
    assert pkg.workloads.check_sorted(chars, nchars, offs, perm) == -1


def test_headline_host_sort_with_lcp(pkg, orc, ctx, headline):
    chars, offs, nchars = headline
    perm, lcp = ctx.sort_host(chars[:nchars], offs, lcp=True)
    assert orc.check_permutation(perm)
    assert orc.check_order(chars, offs, perm) == -1
    assert orc.check_lcp32(chars, offs, perm, lcp) == -1
    # mean LCP of the workload is about 50 chars (48-char shared prefixes)
    assert 45 < float(lcp[1:].mean()) < 60
