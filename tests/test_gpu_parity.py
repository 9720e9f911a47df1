"""GPU parity tests: the CUDA path, called through the C ABI, against the
golden fixtures from the reference pS5, against the oracle restatement on
seeded inputs, and through size-independent properties (order, permutation,
LCP rescan) at full workload sizes. Integer work: everything is bit-exact."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from golden_util import canonical_ids

pytestmark = pytest.mark.gpu

GOLDEN = sorted((Path(__file__).parent / "golden").glob("*.npz"))


def check_against_oracle(orc, chars, offs, perm, lcp):
    ids, rlcp = orc.sort_ids_lcp(chars, offs)
    assert orc.check_permutation(perm)
    assert np.array_equal(canonical_ids(chars, offs, perm, lcp),
                          canonical_ids(chars, offs, ids, rlcp))
    assert np.array_equal(lcp[1:].astype(np.uint64), rlcp[1:])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_golden(ctx_any, path):
    z = np.load(path)
    chars, offs, gids, glcp = z["chars"], z["offs"], z["ids"], z["lcp"]
    perm, lcp = ctx_any.sort_host(chars, offs, lcp=True)
    assert np.array_equal(canonical_ids(chars, offs, perm, lcp), gids)
    assert np.array_equal(lcp[1:].astype(np.uint64), glcp[1:])


@pytest.mark.parametrize("n,lmin,lmax,alpha,seed", [
    (2, 0, 3, b"ab", 1),
    (31, 0, 5, b"ab", 2),
    (33, 0, 9, b"ab", 3),
    (2048, 0, 12, b"abc", 4),
    (2049, 0, 12, b"abc", 5),
    (5000, 0, 40, b"0123456789", 6),
    (100000, 0, 30, b"ab", 7),
    (300000, 1, 64, bytes(range(32, 127)), 8),
    (1000000, 0, 20, b"ACGT", 9),
])
def test_random_vs_oracle(pkg, orc, ctx_any, n, lmin, lmax, alpha, seed):
    chars, offs, _ = pkg.workloads.random_strings(n, lmin, lmax, alpha, seed)
    perm, lcp = ctx_any.sort_host(chars, offs, lcp=True)
    check_against_oracle(orc, chars, offs, perm, lcp)


@pytest.mark.parametrize("strings", [
    [],
    [b"only"],
    [b"b", b"a"],
    [b""] * 5000,
    [b"same"] * 10000,
    [b"\xff" * 40] * 3000 + [b"\xff" * 39],
    [b"a" * k for k in range(0, 3000, 7)],
    [b"z" * 2000 + bytes([97 + i % 26]) + b"q" * (i % 5) for i in range(5000)],
    [b"w" * 100 + bytes([97 + i % 26, 97 + (i // 26) % 26]) for i in range(3000)],
    [bytes([97 + i % 3]) * (1 + i % 17) for i in range(4000)],
], ids=["empty", "one", "two", "all_empty", "all_equal", "ff_bytes", "prefix_chain",
        "deep_shared_prefix", "split_class_tied", "split_class_runs"])
def test_edge_cases(pkg, orc, ctx_any, strings):
    chars, offs = pkg.pack_strings(strings)
    if len(strings) == 0:
        perm, lcp = ctx_any.sort_host(np.zeros(1, np.uint8), np.zeros(0, np.uint64), lcp=True)
        assert perm.shape == (0,)
        return
    perm, lcp = ctx_any.sort_host(chars, offs, lcp=True)
    check_against_oracle(orc, chars, offs, perm, lcp)


def _rand_tails(n, k, seed):
    rng = np.random.default_rng(seed)
    return [bytes(rng.integers(97, 100, k, dtype=np.uint8)) for _ in range(n)]


@pytest.mark.parametrize("case", ["all_equal_big", "long_prefix_big", "few_differ_early",
                                  "one_differs_first_char", "prefix_outliers",
                                  "outliers_past_one_jump", "many_deep_pairs"])
def test_common_prefix_jump(pkg, orc, ctx_any, case):
    """Big segments whose samples all share a prefix jump over it inside the
    pass: all strings equal, a long shared prefix (several jumps of at most
    256 chars), a few strings leaving the prefix early, one string differing
    at char 0, rare strings below and above the prefix (shorter ones, smaller
    and larger chars: the two prefix buckets, at the segment depth),
    outliers that leave a 600-char prefix beyond the first jump, and many
    pairs of strings sharing 1-3 KB each (several deep groups in one warp
    window jump together)."""
    if case == "all_equal_big":
        strings = [b"q" * 500] * 100000
    elif case == "long_prefix_big":
        strings = [b"p" * 1000 + t for t in _rand_tails(50000, 3, 1)]
    elif case == "few_differ_early":
        strings = [b"r" * 300 + t for t in _rand_tails(30000, 2, 2)]
        strings += [b"r" * 5 + b"a" + t for t in _rand_tails(10, 4, 3)]
    elif case == "prefix_outliers":
        strings = [b"m" * 60 + t for t in _rand_tails(100000, 3, 4)]
        strings += [b"m" * 20, b"m" * 33 + b"a", b"m" * 59 + b"z", b"m" * 45 + b"zz",
                    b"m" * 8 + b"\x01", b"m" * 60, b"m" * 61 + b"\xff"]
    elif case == "outliers_past_one_jump":
        strings = [b"k" * 600 + t for t in _rand_tails(60000, 3, 5)]
        strings += [b"k" * 300 + b"a", b"k" * 270 + b"z", b"k" * 100, b"k" * 700, b"k" * 599]
    elif case == "many_deep_pairs":
        rng = np.random.default_rng(6)
        strings = []
        for _ in range(700):
            x = bytes(rng.choice(np.frombuffer(b"ACGT", np.uint8), int(rng.integers(1000, 3000))))
            strings += [x + b"A", x + b"C" + x[:5]]
        strings += [bytes(rng.choice(np.frombuffer(b"ACGT", np.uint8), 20)) for _ in range(600)]
    else:
        strings = [b"s" * 40] * 20000 + [b"a"]
    chars, offs = pkg.pack_strings(strings)
    perm, lcp = ctx_any.sort_host(chars, offs, lcp=True)
    check_against_oracle(orc, chars, offs, perm, lcp)


def _group_strings(case):
    """Strings in groups that share a long prefix behind their first 8 chars,
    with members that leave the prefix early (shorter, smaller or larger
    chars at every position), shuffled."""
    rng = np.random.default_rng({"groups_outliers": 41, "many_groups": 42, "groups_behind_jump": 43,
                                 "groups_indirect": 44, "groups_offsets_shuffled": 45}[case])
    lower = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz", np.uint8)
    ngroups = 400 if case == "many_groups" else 40
    head = b"commonhead:0123456789" if case == "groups_behind_jump" else b""
    strings = []
    for g in range(ngroups):
        pre = head + bytes(rng.choice(lower, int(rng.integers(20, 120))))
        size = int(rng.integers(50, 300)) if case == "many_groups" else int(rng.integers(300, 4000))
        for _ in range(size):
            strings.append(pre + bytes(rng.choice(lower[:3], int(rng.integers(0, 4)))))
        for pos in range(len(head) + 1, len(pre)):
            if case == "many_groups" and pos % 7:
                continue
            strings.append(pre[:pos])
            strings.append(pre[:pos] + b"\x01" + pre[pos + 1:])
            strings.append(pre[:pos] + b"\xff" + pre[pos + 1:])
            strings.append(pre[:pos] + bytes([pre[pos] - 1]) + b"zz")
            strings.append(pre[:pos] + bytes([pre[pos] + 1]))
    order = rng.permutation(len(strings))
    return [strings[i] for i in order]


@pytest.mark.parametrize("case", ["groups_outliers", "many_groups", "groups_behind_jump",
                                  "groups_indirect", "groups_offsets_shuffled"])
def test_group_jumps(pkg, orc, ctx_any, case):
    """'=' buckets whose samples share more chunks behind the splitter take a
    jump of their own: members that leave the group's chunks below or above
    (at every position, ending early or with other chars) and members that
    match them; more groups than a segment keeps; groups behind a common-prefix
    jump of the whole input; the same with offsets read through the offset
    array; offsets in an order unrelated to the arena (the first pass cannot
    stage a warp's strings)."""
    strings = _group_strings(case)
    chars, offs = pkg.pack_strings(strings)
    if case == "groups_offsets_shuffled":
        offs = offs[np.random.default_rng(46).permutation(len(offs))].copy()
    if case == "groups_indirect":
        c = pkg.Context(0)
        try:
            c.set_option(c.OPT_INDIRECT_HANDLES, 1)
            perm, lcp = c.sort_host(chars, offs, lcp=True)
        finally:
            c.close()
    else:
        perm, lcp = ctx_any.sort_host(chars, offs, lcp=True)
    check_against_oracle(orc, chars, offs, perm, lcp)


def test_deep_repeats_suffixes(pkg, orc, ctx_any):
    # a periodic text: suffix LCPs up to the text length
    text = (b"abcab" * 4000)[:19999] + b"\0"
    chars = np.frombuffer(text, dtype=np.uint8).copy()
    offs = np.arange(len(text), dtype=np.uint64)
    perm, lcp = ctx_any.sort_host(chars, offs, lcp=True)
    check_against_oracle(orc, chars, offs, perm, lcp)


def _suffix_text(case):
    """A NUL-terminated text and its suffix count."""
    if case == "periodic":
        t = (b"abcab" * 8000)[:39999]
    elif case == "dna_copies":
        return None
    elif case == "binary":
        t = bytes(np.random.default_rng(51).integers(97, 99, 60000, dtype=np.uint8))
    elif case == "runs_of_a":
        t = b"a" * 12000 + b"b" + b"a" * 3000
    elif case == "high_bytes":
        # chars 1..255 (round 0's text-char keys compare them unsigned), with
        # repeats of 10 KB and 1 KB so that groups reach the doubling
        r = bytes(np.random.default_rng(54).integers(1, 256, 20000, dtype=np.uint8))
        t = r + r[5000:15000] + r[:1000] * 3 + r
    else:  # an inner NUL: not a suffix set, sorted as strings
        t = bytes(np.random.default_rng(52).integers(97, 100, 30000, dtype=np.uint8))
        t = t[:15000] + b"\0" + t[15001:]
    return np.frombuffer(t + b"\0", dtype=np.uint8).copy()


@pytest.mark.parametrize("case", ["periodic", "dna_copies", "binary", "runs_of_a", "high_bytes",
                                  "inner_nul"])
@pytest.mark.parametrize("with_lcp", [True, False])
def test_suffix_doubling(pkg, orc, case, with_lcp):
    """Suffix sets through the multi-launch path, where groups sharing 8 or
    more chars finish by rank doubling: a periodic text (groups of thousands,
    LCPs up to the text length), a DNA text with copied 1-10 KiB blocks, a
    binary text, long runs of one char, chars 1..255 with repeats, and a text
    with a NUL inside (not a suffix set: the string path). Checked against
    the oracle; the doubling must have run for the suffix sets."""
    if case == "dna_copies":
        chars = pkg.workloads.dna_text(length=1 << 20, seed=53)[: (1 << 20) + 1].copy()
    else:
        chars = _suffix_text(case)
    n = chars.shape[0]
    offs = np.arange(n, dtype=np.uint64)
    c = pkg.Context(0)
    try:
        c.set_option(c.OPT_SINGLE_LAUNCH, 0)
        perm, lcp = c.sort_host(chars, offs, lcp=with_lcp)
        used = {k["name"]: k["launches"] for k in c.kernel_stats()}.get("doubling", 0)
    finally:
        c.close()
    assert (used > 0) == (case != "inner_nul")
    if with_lcp:
        check_against_oracle(orc, chars, offs, perm, lcp)
    else:
        assert orc.check_permutation(perm)
        assert orc.check_order(chars, offs, perm) == -1


@pytest.mark.parametrize("n,alpha,lmax,seed", [(3000, b"ab", 40, 31), (200000, b"abc", 30, 32)])
def test_indirect_handles(pkg, orc, n, alpha, lmax, seed):
    """The path for inputs whose string id and arena offset do not fit one
    64-bit handle (offsets read through the offset array), forced on."""
    c = pkg.Context(0)
    try:
        c.set_option(c.OPT_INDIRECT_HANDLES, 1)
        chars, offs, _ = pkg.workloads.random_strings(n, 0, lmax, alpha, seed)
        perm, lcp = c.sort_host(chars, offs, lcp=True)
        check_against_oracle(orc, chars, offs, perm, lcp)
    finally:
        c.close()


@pytest.mark.parametrize("case", ["tied_long_keys", "half_shared_prefix", "big_equal_bucket"])
def test_single_launch_hands_big_buckets_to_the_passes(pkg, orc, ctx, case):
    """Buckets of the single-launch sort over 2048 strings that are not all
    equal continue in the pass loop (a second pass must run); all-equal ones
    are copied out inside the launch."""
    rng = np.random.default_rng(47)
    lower = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz", np.uint8)
    if case == "tied_long_keys":
        heads = [bytes(rng.choice(lower, 8)) for _ in range(20)]
        strings = [heads[i % 20] + bytes(rng.choice(lower[:4], int(rng.integers(1, 12))))
                   for i in range(100000)]
    elif case == "half_shared_prefix":
        pre = bytes(rng.choice(lower, 100))
        strings = [pre + bytes(rng.choice(lower, int(rng.integers(0, 6)))) for _ in range(150000)]
        strings += [bytes(rng.choice(lower, int(rng.integers(1, 30)))) for _ in range(150000)]
    else:
        strings = [b"x"] * 30000 + [bytes(rng.choice(lower, int(rng.integers(1, 9))))
                                    for _ in range(30000)]
    strings = [strings[i] for i in rng.permutation(len(strings))]
    chars, offs = pkg.pack_strings(strings)
    perm, lcp = ctx.sort_host(chars, offs, lcp=True)
    check_against_oracle(orc, chars, offs, perm, lcp)
    if case != "big_equal_bucket":
        assert ctx.stats()["passes"] >= 2


def test_single_launch_wait_limit(pkg, orc):
    """A grid-barrier wait of the single-launch sort that runs out of polls
    ends the sort with PSSGPU_ETIMEOUT (no hang), and the context sorts
    normally once the limit is raised again."""
    chars, offs, _ = pkg.workloads.random_strings(300000, 0, 20, b"abcd", 48)
    c = pkg.Context(0)
    try:
        c.set_option(c.OPT_WAIT_LIMIT, 1)
        with pytest.raises(pkg.SortError) as e:
            c.sort_host(chars, offs, lcp=False)
        assert e.value.status == 4  # PSSGPU_ETIMEOUT
        c.set_option(c.OPT_WAIT_LIMIT, 1 << 22)
        perm, lcp = c.sort_host(chars, offs, lcp=True)
        check_against_oracle(orc, chars, offs, perm, lcp)
    finally:
        c.close()


def test_unterminated_device_arena(pkg, ctx_any):
    """The device entry checks the arena's last char on the device: an
    arena that does not end with NUL is PSSGPU_EINVAL on both paths."""
    import torch
    chars, offs, nchars = pkg.workloads.random_strings(5000, 1, 9, b"ab", 49)
    chars = chars.copy()
    chars[nchars - 1] = 97
    dc = torch.from_numpy(chars).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    dp = torch.empty(len(offs), dtype=torch.int32, device="cuda")
    with pytest.raises(pkg.SortError) as e:
        ctx_any.sort_device(dc, nchars, do, dp)
    assert e.value.status == 1 and "NUL" in str(e.value)


def test_lcp_optional(pkg, ctx):
    chars, offs, _ = pkg.workloads.random_strings(20000, 0, 10, b"abc", 11)
    p1, _ = ctx.sort_host(chars, offs, lcp=False)
    p2, l2 = ctx.sort_host(chars, offs, lcp=True)
    assert np.array_equal(canonical_ids(chars, offs, p1, l2), canonical_ids(chars, offs, p2, l2))


def test_digits_config_full(pkg, orc, ctx):
    chars, offs, nchars = pkg.workloads.digits(seed=1)
    perm, lcp = ctx.sort_host(chars[:nchars], offs, lcp=True)
    check_against_oracle(orc, chars[:nchars], offs, perm, lcp)


def test_dna_suffix_config_full(pkg, orc, ctx):
    chars, offs, n = pkg.workloads.dna_suffixes()
    perm, lcp = ctx.sort_host(chars[: n], offs, lcp=True)
    assert orc.check_permutation(perm)
    assert orc.check_order(chars, offs, perm) == -1
    assert orc.check_lcp32(chars, offs, perm, lcp) == -1


def test_prefix_config_properties(pkg, orc, ctx):
    # the 64 Mi-string workload at a quarter of its size keeps the test short;
    # bench.py sorts the full size
    chars, offs, nchars = pkg.workloads.prefixes(n=16 * 1024 * 1024)
    perm, lcp = ctx.sort_host(chars[:nchars], offs, lcp=True)
    assert orc.check_permutation(perm)
    assert orc.check_order(chars, offs, perm) == -1
    assert orc.check_lcp32(chars, offs, perm, lcp) == -1


def test_prefix_small_vs_oracle(pkg, orc, ctx):
    chars, offs, nchars = pkg.workloads.prefixes(n=400000, seed=12)
    perm, lcp = ctx.sort_host(chars[:nchars], offs, lcp=True)
    check_against_oracle(orc, chars[:nchars], offs, perm, lcp)


def _arena_from_lengths(lens, alpha, seed):
    rng = np.random.default_rng(seed)
    lens = np.asarray(lens, np.uint64)
    offs = np.zeros(len(lens), np.uint64)
    offs[1:] = np.cumsum(lens[:-1] + 1)
    total = int(offs[-1] + lens[-1]) + 1
    chars = rng.choice(np.frombuffer(alpha, np.uint8), total).astype(np.uint8)
    chars[(offs + lens).astype(np.int64)] = 0
    return chars, offs


@pytest.mark.parametrize("case", ["gaps8", "gaps16", "decreasing", "gap_over_16_bits",
                                  "gap_255", "gap_256", "gap_65535", "threshold"])
def test_host_offsets_as_gaps(pkg, orc, ctx, case):
    # host offset arrays of 1 Mi or more strings that never decrease cross
    # PCIe as 1- or 2-byte gaps and are rebuilt on the device; the others are
    # copied as they are. Every form must sort exactly as the oracle does.
    # A gap is a string's length + 1: 255 is the widest 1-byte gap, 65535 the
    # widest 2-byte one; "threshold" has exactly 2^20 strings.
    n = (1 << 20) if case == "threshold" else 1_100_000
    rng = np.random.default_rng(71)
    lens = rng.integers(0, 12, n)
    if case == "gaps16":
        lens[::997] = rng.integers(300, 700, len(lens[::997]))
    if case == "gap_over_16_bits":
        lens[n // 2] = 70_000
    if case == "gap_255":
        lens[n // 3] = 254
    if case == "gap_256":
        lens[n // 3] = 255
    if case == "gap_65535":
        lens[n - 2] = 65_534
    chars, offs = _arena_from_lengths(lens, b"abcd", 72)
    if case == "decreasing":
        offs = offs[rng.permutation(n)]
    perm, lcp = ctx.sort_host(chars, offs, lcp=True)
    check_against_oracle(orc, chars, offs, perm, lcp)
    # the same strings through the device entry point (offsets copied as they are)
    import torch
    dp = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.sort_device(torch.from_numpy(chars).cuda(), len(chars),
                    torch.from_numpy(offs.view(np.int64)).cuda(), dp)
    assert np.array_equal(canonical_ids(chars, offs, dp.cpu().numpy().view(np.uint32), lcp),
                          canonical_ids(chars, offs, perm, lcp))


def test_device_api(pkg, orc, ctx):
    import torch
    chars, offs, nchars = pkg.workloads.random_strings(50000, 0, 16, b"abcd", 13)
    dc = torch.from_numpy(chars).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    dp = torch.empty(len(offs), dtype=torch.int32, device="cuda")
    dl = torch.zeros(len(offs), dtype=torch.int32, device="cuda")
    ctx.sort_device(dc, nchars, do, dp, dl)
    perm = dp.cpu().numpy().view(np.uint32)
    lcp = dl.cpu().numpy().view(np.uint32)
    check_against_oracle(orc, chars, offs, perm, lcp)


TEXT_GOLDEN = sorted((Path(__file__).parent / "golden" / "text").glob("*.npz"))


@pytest.mark.parametrize("path", TEXT_GOLDEN, ids=[p.stem for p in TEXT_GOLDEN])
def test_text_golden(pkg, orc, ctx, path):
    """A text split into lines (or suffixes) on the device and sorted gives
    the reference psstest's sorted output for the same file, and the LCP
    array of the oracle."""
    z = np.load(path)
    text, suffix = z["text"].tobytes(), bool(z["suffix"])
    perm, lcp = ctx.sort_text_host(text, ctx.TEXT_SUFFIXES if suffix else ctx.TEXT_LINES)
    arena, offs = orc.split_text(text, suffix)
    assert perm.shape[0] == offs.shape[0]
    assert orc.sorted_output(arena, offs, perm) == z["output"].tobytes()
    if perm.shape[0] > 1:
        check_against_oracle(orc, arena, offs, perm, lcp)


def _random_text(size, seed):
    rng = np.random.default_rng(seed)
    t = rng.choice(np.frombuffer(b"ab\n", np.uint8), size, p=[0.45, 0.45, 0.10]).astype(np.uint8)
    t[rng.integers(0, size, max(1, size // 5000))] = 0  # NULs end strings too
    return t


@pytest.mark.parametrize("size,mode", [(3 << 20, 0), ((1 << 16) + 1, 0), ((1 << 16) + 8, 0),
                                       (9, 0), (1, 0), (70001, 1)])
def test_prepare_text_device(pkg, orc, ctx, size, mode):
    """Device-side preparation equals the restated loader byte for byte and
    offset for offset (many chunks, the last byte at a chunk or word
    boundary, a one-byte text, suffixes); an offset array that is too small
    is refused with the text left unchanged."""
    import torch
    t = _random_text(size, size)
    dt = torch.zeros(size + 16, dtype=torch.uint8, device="cuda")
    dt[:size] = torch.from_numpy(t).cuda()
    arena, offs = orc.split_text(t, suffix=mode == 1)
    n = offs.shape[0]
    small = torch.zeros(max(n - 1, 1), dtype=torch.int64, device="cuda")
    if n > 1:
        with pytest.raises(pkg.SortError):
            ctx.prepare_text_device(dt, size, mode, small)
        assert np.array_equal(dt[:size].cpu().numpy(), t)
    do = torch.zeros(n, dtype=torch.int64, device="cuda")
    assert ctx.prepare_text_device(dt, size, mode, do) == n
    assert np.array_equal(dt.cpu().numpy(), arena)
    assert np.array_equal(do.cpu().numpy().view(np.uint64), offs)
    dp = torch.empty(n, dtype=torch.int32, device="cuda")
    dl = torch.zeros(n, dtype=torch.int32, device="cuda")
    ctx.sort_device(dt, size, do, dp, dl)
    if n > 1 and size < (1 << 20):
        check_against_oracle(orc, arena, offs, dp.cpu().numpy().view(np.uint32),
                             dl.cpu().numpy().view(np.uint32))


def test_sort_text_digits_config_full(pkg, orc, ctx):
    """The 10 MiB digits workload as a newline-separated text: split and
    sorted on the device; order, permutation and LCPs checked in full."""
    chars, offs0, nchars = pkg.workloads.digits(seed=1)
    text = chars[:nchars].copy()
    text[text == 0] = 10
    perm, lcp = ctx.sort_text_host(text, ctx.TEXT_LINES)
    arena, offs = orc.split_text(text)
    assert offs.shape[0] == offs0.shape[0] and np.array_equal(offs, offs0)
    assert orc.check_permutation(perm)
    assert orc.check_order(arena, offs, perm) == -1
    assert orc.check_lcp32(arena, offs, perm, lcp) == -1


def _oracle_runs(orc, chars, offs, K, seed, empty_run=False):
    """Strings dealt at random to K runs, each sorted with its LCP array by
    the oracle: (ids, lcp, boundaries)."""
    rng = np.random.default_rng(seed)
    deal = rng.integers(0, K, offs.shape[0])
    if empty_run:
        deal[deal == 1] = 0
    ids, lcps, runs = [], [], [0]
    for k in range(K):
        members = np.flatnonzero(deal == k).astype(np.uint32)
        if members.shape[0]:
            sub, sub_lcp = orc.sort_ids_lcp(chars, offs[members])
            ids.append(members[sub])
            lcps.append(sub_lcp.astype(np.uint32))
        runs.append(runs[-1] + members.shape[0])
    return np.concatenate(ids), np.concatenate(lcps), np.array(runs, np.uint64)


def _merge_strings(case):
    rng = np.random.default_rng(77)
    if case == "deep":
        base = bytes(rng.integers(97, 123, 300, dtype=np.uint8))
        return ([base[: int(rng.integers(250, 301))] + bytes(rng.integers(97, 99, int(rng.integers(0, 5)),
                                                                        dtype=np.uint8))
                 for _ in range(6000)] + [base] * 50 + [b""] * 20)
    return [bytes(rng.integers(97, 100, int(rng.integers(0, 14)), dtype=np.uint8)) for _ in range(30000)]


@pytest.mark.parametrize("K,case", [(1, "rand"), (2, "rand"), (3, "rand"), (8, "rand"), (33, "rand"),
                                    (5, "empty_run"), (4, "deep"), (7, "deep"), (2, "no_lcp"),
                                    (6, "no_lcp_input")])
def test_merge_lcp(pkg, orc, ctx, K, case):
    """Sorted runs with their LCP arrays merge into the sorted sequence and
    LCP array of all strings: pairs, odd run counts, many runs, an empty run,
    runs sharing 250-300 char prefixes with duplicates and empty strings, the
    merge without LCP output, and without the runs' LCP arrays (compares from
    char 0)."""
    import torch
    chars, offs = pkg.pack_strings(_merge_strings("deep" if case == "deep" else "rand"))
    nchars = chars.shape[0]
    ids, lcp, runs = _oracle_runs(orc, chars, offs, K, 90 + K, empty_run=case == "empty_run")
    dc = torch.from_numpy(np.concatenate([chars, np.zeros(16, np.uint8)])).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    di = torch.from_numpy(ids.view(np.int32)).cuda()
    dl = torch.from_numpy(lcp.view(np.int32)).cuda() if case != "no_lcp_input" else None
    dio = torch.empty_like(di)
    dlo = torch.zeros_like(di) if case not in ("no_lcp", "no_lcp_input") else None
    ctx.merge_lcp_device(dc, nchars, do, runs, di, dl, dio, dlo)
    perm = dio.cpu().numpy().view(np.uint32)
    if dlo is None:
        assert orc.check_permutation(perm)
        assert orc.check_order(chars, offs, perm) == -1
    else:
        check_against_oracle(orc, chars, offs, perm, dlo.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("piece", [1, 3, 8, 128])
@pytest.mark.parametrize("indirect", [0, 1])
def test_merge_lcp_char_caches(pkg, orc, piece, indirect):
    """The piece merge orders heads with equal LCPs from the 7 chars each
    carries from that depth, and reads the arena only past them: strings that
    differ inside the cached chars, after them (a 12-char shared stem then
    variants up to 20 chars deeper), end inside them (duplicates, prefixes of
    one another, empty strings), over several rounds and with a piece start
    (heads read from the arena) at every few outputs."""
    import torch
    rng = np.random.default_rng(31 + piece)
    stem = b"abbabaabbaba"
    strs = [bytes(rng.integers(97, 99, int(rng.integers(0, 30)), dtype=np.uint8)) for _ in range(3000)]
    strs += [stem + bytes(rng.integers(97, 99, int(rng.integers(0, 21)), dtype=np.uint8)) for _ in range(3000)]
    strs += [stem] * 40 + [stem[:5]] * 30 + [b""] * 20
    chars, offs = pkg.pack_strings(strs)
    nchars = chars.shape[0]
    ids, lcp, runs = _oracle_runs(orc, chars, offs, 5, 300 + piece)
    dc = torch.from_numpy(np.concatenate([chars, np.zeros(16, np.uint8)])).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    di = torch.from_numpy(ids.view(np.int32)).cuda()
    dl = torch.from_numpy(lcp.view(np.int32)).cuda()
    dio = torch.empty_like(di)
    dlo = torch.zeros_like(di)
    c = pkg.Context(0)
    try:
        c.set_option(c.OPT_MERGE_PIECE, piece)
        c.set_option(c.OPT_INDIRECT_HANDLES, indirect)
        c.merge_lcp_device(dc, nchars, do, runs, di, dl, dio, dlo)
    finally:
        c.close()
    check_against_oracle(orc, chars, offs, dio.cpu().numpy().view(np.uint32), dlo.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("K,case", [(3, "rand"), (4, "deep"), (2, "no_lcp"), (6, "no_lcp_input")])
def test_merge_lcp_ids_path(pkg, orc, K, case):
    """The merge rounds on string ids with offsets gathered at each use (the
    form an arena over 4 GiB takes; PSSGPU_OPT_INDIRECT_HANDLES forces it
    here) give the same results as the handle form."""
    import torch
    chars, offs = pkg.pack_strings(_merge_strings("deep" if case == "deep" else "rand"))
    nchars = chars.shape[0]
    ids, lcp, runs = _oracle_runs(orc, chars, offs, K, 190 + K)
    dc = torch.from_numpy(np.concatenate([chars, np.zeros(16, np.uint8)])).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    di = torch.from_numpy(ids.view(np.int32)).cuda()
    dl = torch.from_numpy(lcp.view(np.int32)).cuda() if case != "no_lcp_input" else None
    dio = torch.empty_like(di)
    dlo = torch.zeros_like(di) if case not in ("no_lcp", "no_lcp_input") else None
    c = pkg.Context(0)
    try:
        c.set_option(c.OPT_INDIRECT_HANDLES, 1)
        c.merge_lcp_device(dc, nchars, do, runs, di, dl, dio, dlo)
    finally:
        c.close()
    perm = dio.cpu().numpy().view(np.uint32)
    if dlo is None:
        assert orc.check_permutation(perm)
        assert orc.check_order(chars, offs, perm) == -1
    else:
        check_against_oracle(orc, chars, offs, perm, dlo.cpu().numpy().view(np.uint32))


def test_merge_rejects_offsets_outside_the_arena(pkg, orc, ctx):
    import torch
    chars, offs = pkg.pack_strings([b"b", b"a", b"c", b"a"])
    nchars = chars.shape[0]
    offs = offs.copy()
    offs[2] = nchars + 5
    dc = torch.from_numpy(np.concatenate([chars, np.zeros(16, np.uint8)])).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    di = torch.tensor([1, 0, 3, 2], dtype=torch.int32, device="cuda")
    dl = torch.zeros(4, dtype=torch.int32, device="cuda")
    with pytest.raises(pkg.SortError) as e:
        ctx.merge_lcp_device(dc, nchars, do, np.array([0, 2, 4], np.uint64), di, dl,
                             torch.empty_like(di), torch.zeros_like(dl))
    assert e.value.status == 1


def test_sharded_sort_then_merge(pkg, orc, ctx):
    """The top-level composition of the reference (per-shard pS5, then the
    LCP merge): four shards of the prefix workload sorted by the GPU sort
    with LCP output, merged on the device, checked against the oracle."""
    import torch
    chars, offs, nchars = pkg.workloads.prefixes(n=200000, seed=13)
    n = offs.shape[0]
    dc = torch.from_numpy(chars).cuda()
    bounds = np.array([0, 37000, 90000, 150001, n], np.uint64)
    ids = torch.empty(n, dtype=torch.int32, device="cuda")
    lcp = torch.zeros(n, dtype=torch.int32, device="cuda")
    for k in range(4):
        b, e = int(bounds[k]), int(bounds[k + 1])
        do = torch.from_numpy(offs[b:e].view(np.int64)).cuda()
        ctx.sort_device(dc, nchars, do, ids[b:e], lcp[b:e])
        ids[b:e] += b  # shard-local ids -> global ids
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    out = torch.empty_like(ids)
    out_lcp = torch.zeros_like(lcp)
    ctx.merge_lcp_device(dc, nchars, do, bounds, ids, lcp, out, out_lcp)
    check_against_oracle(orc, chars[:nchars], offs, out.cpu().numpy().view(np.uint32),
                         out_lcp.cpu().numpy().view(np.uint32))


def test_pointer_array_dropins(pkg, orc):
    """The three psstest contestant signatures on a raw pointer array."""
    lib = pkg._native.gpu()
    chars, offs, nchars = pkg.workloads.random_strings(30000, 0, 12, b"abc", 14)
    buf = (C.c_ubyte * len(chars)).from_buffer_copy(chars.tobytes())
    base = C.addressof(buf)
    n = len(offs)
    ptr_t = C.c_void_p * n
    ids, rlcp = orc.sort_ids_lcp(chars, offs)
    want = orc.sorted_strings(chars, offs, ids)

    def got_sequence(ptrs):
        got_offs = np.array([p - base for p in ptrs], dtype=np.uint64)
        assert len(set(got_offs.tolist())) == n  # a permutation of the pointers
        return orc.sorted_strings(chars, got_offs, np.arange(n))

    ptrs = ptr_t(*[base + int(o) for o in offs])
    lib.pssgpu_sort_strings(ptrs, n)
    assert got_sequence(ptrs) == want

    ptrs = ptr_t(*[base + int(o) for o in offs])
    lcp = (C.c_size_t * n)()
    lcp[0] = 42
    lib.pssgpu_sort_strings_lcp(ptrs, lcp, n)
    assert got_sequence(ptrs) == want
    assert lcp[0] == 42
    assert np.array_equal(np.array(lcp[1:], dtype=np.uint64), rlcp[1:])

    ptrs = ptr_t(*[base + int(o) for o in offs])
    lcp = (C.c_size_t * n)()
    cache = (C.c_ubyte * n)()
    lib.pssgpu_sort_strings_lcp_cache(ptrs, lcp, cache, n)
    raw = chars.tobytes()
    for i in range(1, n, 97):
        assert cache[i] == raw[ptrs[i] - base + lcp[i]]


def test_suffix_pointer_array_dense_span(pkg, orc):
    """Overlapping suffix pointers (psstest --suffix) through the arena entry,
    which copies the text span once, and through the plain entry, which
    gathers every suffix."""
    text = pkg.workloads.dna_text(length=20000, seed=15)
    buf = (C.c_ubyte * len(text)).from_buffer_copy(text.tobytes())
    base = C.addressof(buf)
    n = 20001
    offs = np.arange(n, dtype=np.uint64)
    ptrs = (C.c_void_p * n)(*[base + i for i in range(n)])
    assert pkg.sort_pointer_array_arena(base, 20001, ptrs, n) == 0
    sa = np.array([p - base for p in ptrs], dtype=np.uint64)
    assert orc.check_permutation(sa.astype(np.uint32))
    assert orc.check_order(text, offs, sa.astype(np.uint32)) == -1
    m = 3001  # plain entry: every suffix gathered (quadratic bytes, kept small)
    ptrs = (C.c_void_p * m)(*[base + 17000 + i for i in range(m)])
    assert pkg.sort_pointer_array(ptrs, m) == 0
    got = np.array([p - base - 17000 for p in ptrs], dtype=np.uint32)
    assert np.array_equal(np.sort(got), np.arange(m, dtype=np.uint32))
    assert orc.check_order(text[17000:], np.arange(m, dtype=np.uint64), got) == -1


def test_pointer_array_separate_allocations(pkg, orc):
    """Strings in separate host allocations: the plain entry reads each string
    through its own pointer and nothing between them."""
    strings = [bytes([97 + (i * 7 + j) % 3 for j in range(i % 13)]) for i in range(5000)]
    bufs = [C.create_string_buffer(s) for s in strings]
    n = len(bufs)
    addr = [C.addressof(b) for b in bufs]
    ptrs = (C.c_void_p * n)(*addr)
    assert pkg.sort_pointer_array(ptrs, n) == 0
    index = {a: i for i, a in enumerate(addr)}
    got = [strings[index[p]] for p in ptrs]
    assert sorted(index[p] for p in ptrs) == list(range(n))
    assert got == sorted(strings)


def test_pointer_array_out_and_arena(pkg, orc):
    """The separate-output entry leaves the input unchanged; the arena entry
    sorts in place or into an output array, with LCP and cache, and rejects a
    pointer outside the arena it was given."""
    chars, offs, nchars = pkg.workloads.random_strings(40000, 0, 14, b"abcd", 16)
    buf = (C.c_ubyte * len(chars)).from_buffer_copy(chars.tobytes())
    base = C.addressof(buf)
    n = len(offs)
    ptr_t = C.c_void_p * n
    ids, rlcp = orc.sort_ids_lcp(chars, offs)
    want = orc.sorted_strings(chars, offs, ids)
    raw = chars.tobytes()

    def sequence(ptrs):
        got_offs = np.array([p - base for p in ptrs], dtype=np.uint64)
        assert np.array_equal(np.sort(got_offs), np.sort(offs))
        return orc.sorted_strings(chars, got_offs, np.arange(n))

    src = [base + int(o) for o in offs]
    ptrs, out = ptr_t(*src), ptr_t()
    assert pkg.sort_pointer_array_out(ptrs, out, n) == 0
    assert list(ptrs) == src
    assert sequence(out) == want

    ptrs = ptr_t(*src)
    lib = pkg._native.gpu()
    lib.pssgpu_sort_strings_out(ptrs, out, n)
    assert list(ptrs) == src and sequence(out) == want

    ptrs, out = ptr_t(*src), ptr_t()
    lcp = (C.c_size_t * n)()
    lcp[0] = 42
    cache = (C.c_ubyte * n)()
    assert pkg.sort_pointer_array_arena(base, nchars, ptrs, n, out, lcp, cache) == 0
    assert list(ptrs) == src
    assert sequence(out) == want
    assert lcp[0] == 42
    assert np.array_equal(np.array(lcp[1:], dtype=np.uint64), rlcp[1:])
    for i in range(1, n, 89):
        assert cache[i] == raw[out[i] - base + lcp[i]]

    ptrs = ptr_t(*src)
    assert pkg.sort_pointer_array_arena(base, nchars, ptrs, n) == 0
    assert sequence(ptrs) == want

    # a pointer beyond the declared arena, and a string not terminated inside it
    ptrs = ptr_t(*src)
    assert pkg.sort_pointer_array_arena(base, int(offs[-1]), ptrs, n) == 1
    assert list(ptrs) == src
    last_len = raw.index(b"\0", int(offs[-1])) - int(offs[-1])
    rc = pkg.sort_pointer_array_arena(base, int(offs[-1]) + 1, ptrs, n)
    assert rc == (1 if last_len > 0 else 0)
    assert pkg.sort_pointer_array_out(ptrs, ptrs, n) == 0  # output == input: in place


@pytest.mark.parametrize("n", [1_100_000, 1_300_000])
def test_pointer_array_arena_large(pkg, orc, n):
    """The arena entry above 2^20 strings (offsets cross PCIe as gaps; the
    context's pinned buffers are reused by the second size and grown), in
    place and with LCP output, twice in a row, against the oracle."""
    chars, offs, nchars = pkg.workloads.random_strings(n, 0, 20, b"abc", 31 + n)
    buf = (C.c_ubyte * len(chars)).from_buffer_copy(chars.tobytes())
    base = C.addressof(buf)
    ids, rlcp = orc.sort_ids_lcp(chars, offs)
    want = np.array([int(offs[i]) for i in ids], dtype=np.uint64)
    src = (C.c_void_p * n)(*[base + int(o) for o in offs])
    for _ in range(2):
        ptrs = (C.c_void_p * n)()
        C.memmove(ptrs, src, C.sizeof(src))
        lcp = (C.c_size_t * n)()
        assert pkg.sort_pointer_array_arena(base, nchars, ptrs, n, None, lcp) == 0
        got = np.frombuffer(ptrs, dtype=np.uint64) - np.uint64(base)
        # equal strings may come in any order: order and multiset of offsets
        assert np.array_equal(np.array(lcp[1:], dtype=np.uint64), rlcp[1:])
        assert orc.check_order(chars, got, np.arange(n, dtype=np.uint32)) == -1
        assert np.array_equal(np.sort(got), np.sort(want))


def test_errors_are_status_codes(pkg, ctx):
    chars = np.frombuffer(b"abc", dtype=np.uint8).copy()  # no terminating NUL
    with pytest.raises(pkg.SortError) as e:
        ctx.sort_host(chars, np.zeros(1, np.uint64))
    assert e.value.status == 1
    chars = np.frombuffer(b"ab\0", dtype=np.uint8).copy()
    with pytest.raises(pkg.SortError) as e:
        ctx.sort_host(chars, np.array([0, 7], np.uint64))  # offset outside the arena
    assert e.value.status == 1
    # the context stays usable after an error
    perm, _ = ctx.sort_host(np.frombuffer(b"b\0a\0", np.uint8).copy(), np.array([0, 2], np.uint64))
    assert perm.tolist() == [1, 0]
