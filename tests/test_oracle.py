"""CPU tests: the oracle restatement is pinned against the reference pS5
(golden fixtures generated from it, and the compiled reference itself where
it is present), unit oracles for key extraction and classification, and the
checkers catch planted mistakes."""
from pathlib import Path

import numpy as np
import pytest

from golden_util import canonical_ids

GOLDEN = sorted((Path(__file__).parent / "golden").glob("*.npz"))


def load(path):
    z = np.load(path)
    return z["chars"], z["offs"], z["ids"], z["lcp"]


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_restatement_matches_golden(orc, path):
    chars, offs, gids, glcp = load(path)
    ids, lcp = orc.sort_ids_lcp(chars, offs)
    assert np.array_equal(canonical_ids(chars, offs, ids, lcp), gids)
    assert np.array_equal(lcp[1:], glcp[1:])
    assert glcp[0] == 42  # the reference never writes lcp[0]


def test_golden_set_present():
    names = {p.stem for p in GOLDEN}
    assert {"edge_mixed", "digits_256k", "alpha_ab", "prefix_30k", "dna_suffix_64k",
            "highbyte_long"} <= names


@pytest.mark.parametrize("seed,alpha,lmax", [(1, b"ab", 12), (2, b"0123456789", 40),
                                             (3, bytes(range(1, 256)), 20)])
def test_restatement_matches_reference_run(pkg, orc, seed, alpha, lmax):
    if not orc.ref_available():
        pytest.skip("reference pS5 not built here")
    chars, offs, _ = pkg.workloads.random_strings(40000, 0, lmax, alpha, seed)
    ids, lcp = orc.sort_ids_lcp(chars, offs)
    rids, rlcp = orc.ref_sort(chars, offs, threads=4, lcp=True)
    assert np.array_equal(canonical_ids(chars, offs, ids, lcp),
                          canonical_ids(chars, offs, rids, rlcp))
    assert np.array_equal(lcp[1:], rlcp[1:])
    assert rlcp[0] == 42


def test_key_extraction_matches_reference(pkg, orc):
    if not orc.ref_available():
        pytest.skip("reference pS5 not built here")
    chars, offs, _ = pkg.workloads.random_strings(2000, 0, 30, b"\x01a\xff", seed=4)
    rng = np.random.default_rng(0)
    for i in rng.integers(0, len(offs), 500):
        for depth in (0, 1, 3, 7, 8, 13):
            ln = chars.tobytes().index(b"\0", int(offs[i])) - int(offs[i])
            if depth > ln:
                continue
            assert orc.get_uint64(chars, offs[i], depth) == orc.ref_get_uint64(chars, offs[i], depth)


def test_classification_matches_reference_find_bkt(orc):
    if not orc.ref_available():
        pytest.skip("reference pS5 not built here")
    rng = np.random.default_rng(5)
    spl = np.sort(rng.integers(0, 2**63, 1023, dtype=np.uint64) * np.uint64(2))
    spl[100:110] = spl[100]  # duplicated splitters
    keys = np.concatenate([rng.integers(0, 2**63, 5000, dtype=np.uint64) * np.uint64(2),
                           spl[::7], spl[::11] + np.uint64(1), np.array([0, 2**64 - 1], np.uint64)])
    assert np.array_equal(orc.classify(spl, keys), orc.ref_find_bkt(spl, keys))


def test_checkers_catch_planted_mistakes(pkg, orc):
    chars, offs, _ = pkg.workloads.random_strings(5000, 1, 10, b"abcd", seed=6)
    ids, lcp = orc.sort_ids_lcp(chars, offs)
    assert orc.check_order(chars, offs, ids) == -1
    assert orc.check_permutation(ids)
    assert orc.check_lcp32(chars, offs, ids, lcp.astype(np.uint32)) == -1
    bad = ids.copy()
    bad[[10, 4000]] = bad[[4000, 10]]
    assert orc.check_order(chars, offs, bad) != -1
    dup = ids.copy()
    dup[3] = dup[4]
    assert not orc.check_permutation(dup)
    badl = lcp.astype(np.uint32).copy()
    badl[77] += 1
    assert orc.check_lcp32(chars, offs, ids, badl) == 77


def test_distinguishing_prefix(pkg, orc):
    chars, offs = pkg.pack_strings([b"abc", b"abd", b"b", b"ba"])
    ids = orc.sort_ids(chars, offs)
    d, s = orc.dprefix(chars, offs, ids)
    assert s == 2 + 0 + 1  # lcp(abc,abd)=2, lcp(abd,b)=0, lcp(b,ba)=1
    assert d > 0


TEXT_GOLDEN = sorted((Path(__file__).parent / "golden" / "text").glob("*.npz"))


@pytest.mark.parametrize("path", TEXT_GOLDEN, ids=[p.stem for p in TEXT_GOLDEN])
def test_text_split_matches_psstest(orc, path):
    """The restated text loading (lines / suffixes, newline and NUL
    separators, the forced last NUL) sorted by the oracle reproduces the
    reference psstest's -o output on the same file."""
    z = np.load(path)
    arena, offs = orc.split_text(z["text"].tobytes(), bool(z["suffix"]))
    ids = orc.sort_ids(arena, offs)
    assert orc.sorted_output(arena, offs, ids) == z["output"].tobytes()


def test_text_split_counts(orc):
    # separators at 1, 2, 4, 6, 8 of 13 bytes; the last byte becomes NUL
    arena, offs = orc.split_text(b"b\n\na\nc\0d\nlast")
    assert offs.tolist() == [0, 2, 3, 5, 7, 9]
    assert bytes(arena[:13]) == b"b\0\0a\0c\0d\0las\0"
    arena, offs = orc.split_text(b"x\ny\n", suffix=True)
    assert offs.tolist() == [0, 1, 2, 3] and bytes(arena[:4]) == b"x\ny\0"
    assert orc.split_text(b"")[1].shape == (0,)
    assert orc.split_text(b"\n")[1].tolist() == [0]


def _split_text_loops(text: bytes, suffix: bool):
    """The loader and the pointer-array build as the reference writes them,
    loop for loop (src/tools/input.hpp:275-297, src/psstest.cpp:479-518)."""
    data = bytearray(text) + bytearray(9)
    size = len(text)
    count = 1
    if not suffix:
        for i in range(size):
            if data[i] == 10 or data[i] == 0:
                data[i] = 0
                if i + 1 < size:
                    count += 1
    else:
        count = size
    data[size - 1] = 0
    if not suffix:
        starts = [i for i in range(size) if i == 0 or data[i - 1] == 0]
    else:
        starts = list(range(size))
    assert len(starts) == count
    return bytes(data[:size]), starts


@pytest.mark.parametrize("seed", range(12))
def test_text_split_matches_loop_restatement(orc, seed):
    """The vectorised restatement equals the reference's loops on random
    texts over {a, b, newline, NUL} of 1..300 bytes, in both modes."""
    rng = np.random.default_rng(seed)
    for _ in range(40):
        size = int(rng.integers(1, 301))
        text = bytes(rng.choice(np.frombuffer(b"ab\n\0", np.uint8), size, p=[0.4, 0.4, 0.15, 0.05]))
        for suffix in (False, True):
            arena, offs = orc.split_text(text, suffix)
            data, starts = _split_text_loops(text, suffix)
            assert bytes(arena[:size]) == data and not arena[size:].any()
            assert offs.tolist() == starts


@pytest.mark.parametrize("seed", range(6))
def test_lcp_merge_rule(pkg, orc, seed):
    """The LCP rule of the reference's loser tree, restated for two runs:
    merging two sorted runs with their LCP arrays gives the sorted order and
    LCP array of all strings, and reads only the chars behind the LCPs (far
    fewer than compares from char 0)."""
    rng = np.random.default_rng(seed)
    pre = bytes(rng.integers(97, 123, 30, dtype=np.uint8))
    strings = [pre[: int(rng.integers(0, 31))] + bytes(rng.integers(97, 100, int(rng.integers(0, 5)),
                                                                     dtype=np.uint8))
               for _ in range(600)]
    chars, offs = pkg.pack_strings(strings)
    deal = rng.integers(0, 2, len(strings))
    parts = []
    for k in (0, 1):
        members = np.flatnonzero(deal == k).astype(np.uint32)
        sub, sub_lcp = orc.sort_ids_lcp(chars, offs[members])
        parts += [members[sub], sub_lcp]
    ids, lcp, reads = orc.lcp_merge2(chars, offs, *parts)
    rids, rlcp = orc.sort_ids_lcp(chars, offs)
    assert np.array_equal(canonical_ids(chars, offs, ids, lcp), canonical_ids(chars, offs, rids, rlcp))
    assert np.array_equal(lcp[1:], rlcp[1:])
    full = sum(int(x) + 1 for x in rlcp[1:])  # chars a compare from char 0 reads, at least
    assert reads < full / 4
