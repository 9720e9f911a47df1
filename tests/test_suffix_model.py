"""CPU model of the rank doubling that finishes suffix sets on the device
(csrc/kernels_suffix.cuh), checked against sorting the suffixes outright.

The model follows the kernels' rules step by step: groups of equal 8-char
prefixes are handed over at depth 8; round 0 sorts each group by the 6 text
chars that follow its shared prefix, giving runs of equal chars a subgroup 6
chars deeper; every suffix's rank is then its final position or its group's
start; each later round reads the ranks and group depths of one snapshot,
sorts each group by the rank of its members' suffixes `depth` chars further,
gives singletons their position and runs of equal ranks a subgroup of depth
`depth + depth of the tied group`; positions separated in a round record
that depth, and the LCPs there come from the larger of that depth and the
previous suffix's LCP minus one. Small texts, pure Python: the
method, not the kernels, is under test here (the kernels are checked against
the oracle by the GPU tests).
"""
import numpy as np
import pytest


ROUND0_CHARS = 6  # DBL_ROUND0_CHARS of the kernels


def doubling_model(text: bytes, split_above: int = 0):
    """Suffix array and LCP array of text (which ends with its only NUL) by
    the device method; returns (sa, lcp, rounds). Groups of more than
    split_above members (0: none) are first split by 8 more chars, as the
    string passes do for groups too large to hand over, so the doubling
    starts from groups of different depths."""
    n = len(text)
    body = text[:-1]

    def s(i):
        return body[i:]

    # string-sort stage: by the first 8 chars; equal prefixes of 8 chars
    # (none shorter can tie: suffixes are distinct) form groups at depth 8
    sa = sorted(range(n), key=lambda i: s(i)[:8])
    groups = []
    p = 0
    while p < n:
        e = p + 1
        while e < n and s(sa[e])[:8] == s(sa[p])[:8]:
            e += 1
        if e - p >= 2:
            assert len(s(sa[p])) >= 8
            if split_above and e - p > split_above:
                sub = sorted(sa[p:e], key=lambda i: s(i)[:16])
                sa[p:e] = sub
                q = p
                while q < e:
                    f = q + 1
                    while f < e and s(sa[f])[:16] == s(sa[q])[:16]:
                        f += 1
                    if f - q >= 2:
                        groups.append((q, f - q, 16))
                    q = f
            else:
                groups.append((p, e - p, 8))
        p = e
    isa = [0] * n
    for q, x in enumerate(sa):
        isa[x] = q
    gd = [dict(), dict()]
    for b, m, d in groups:
        for q in range(b, b + m):
            isa[sa[q]] = b
        gd[0][b] = d
    lb = [None] * n
    par, rounds = 0, 0
    while groups:
        round0 = rounds == 0
        rounds += 1
        if round0:  # the text chars behind the shared prefix
            keys = {q: s(sa[q])[d:d + ROUND0_CHARS] for b, m, d in groups for q in range(b, b + m)}
        else:       # ranks of one snapshot
            keys = {q: isa[sa[q] + d] for b, m, d in groups for q in range(b, b + m)}
        nxt = []
        gd[par ^ 1] = {}
        for b, m, d in groups:
            members = sorted(range(b, b + m), key=lambda q: (keys[q], sa[q]))
            order = [(keys[q], sa[q]) for q in members]
            for i, (_, x) in enumerate(order):
                sa[b + i] = x
            i = 0
            while i < m:
                K = order[i][0]
                e = i + 1
                while e < m and order[e][0] == K:
                    e += 1
                if i > 0:
                    lb[b + i] = d
                for q in range(i, e):
                    isa[order[q][1]] = b + i
                if e - i >= 2:
                    nd = d + (ROUND0_CHARS if round0 else gd[par][K])
                    gd[par ^ 1][b + i] = nd
                    nxt.append((b + i, e - i, nd))
                i = e
        groups = nxt
        par ^= 1
    # LCPs at the separated positions, in text order (Phi bound)
    lcp = [None] * n
    prev = None
    for x in range(n):
        q = isa[x]
        if q == 0 or lb[q] is None:
            prev = None
            continue
        y = sa[q - 1]
        h = max(lb[q], prev - 1 if prev else 0)
        a, c = s(x), s(y)
        assert a[:h] == c[:h], "the lower bound overshoots the LCP"
        while h < len(a) and h < len(c) and a[h] == c[h]:
            h += 1
        lcp[q] = h
        prev = h
    return sa, lcp, rounds


def _texts():
    rng = np.random.default_rng(61)
    yield "periodic", (b"abcab" * 400)[:1999]
    yield "binary", bytes(rng.integers(97, 99, 3000, dtype=np.uint8))
    base = bytes(rng.choice(np.frombuffer(b"ACGT", np.uint8), 2500))
    copied = base[:1500] + base[200:700] + base[1500:] + base[100:400]
    yield "copies", copied
    yield "runs", b"a" * 900 + b"b" + b"a" * 300
    yield "tiny", b"ab"


@pytest.mark.parametrize("split_above", [0, 40])
@pytest.mark.parametrize("name,text", list(_texts()), ids=[t[0] for t in _texts()])
def test_rank_doubling_model(name, text, split_above):
    t = text + b"\0"
    sa, lcp, rounds = doubling_model(t, split_above)
    want = sorted(range(len(t)), key=lambda i: t[i:-1])
    assert sa == want
    for q in range(1, len(t)):
        if lcp[q] is None:
            continue
        a, b = t[sa[q - 1]:-1], t[sa[q]:-1]
        k = 0
        while k < min(len(a), len(b)) and a[k] == b[k]:
            k += 1
        assert lcp[q] == k
    if name in ("periodic", "runs"):
        # depth doubling: far fewer rounds than the LCPs / 8
        assert rounds <= 12
