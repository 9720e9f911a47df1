"""Generate the golden fixtures in this directory from the reference pS5.

The reference's own pS5 (parallel_sample_sort_lcp_base with
ClassifyTreeUnrollInterleaveX, compiled from the reference sources into
oracle/_ref/libps5ref.so by oracle/Makefile) sorts each input; the fixture
stores the input arena, the sorted ids in canonical form (ids of equal strings
in increasing order) and the reference's LCP array (lcp[0] = the sentinel 42
the reference tests pre-fill and require unchanged).

Run from the repository root after building: python tests/golden/make_golden.py
The reference tree is only needed here; the fixtures travel without it.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

import __graft_entry__  # noqa: E402
from oracle import oracle as orc  # noqa: E402
from golden_util import canonical_ids  # noqa: E402

pkg = __graft_entry__.load_package()
W = pkg.workloads


def edge_strings():
    rng = np.random.default_rng(11)
    out = [b"", b"", b"a", b"\xff", b"\xff\xff", b"\x01", b"\x7f\x80", b"\xff" * 17]
    for L in (7, 8, 9, 15, 16, 17, 23, 24, 25):
        for c in (b"a", b"b"):
            out.append(c * L)
            out.append(c * (L - 1) + b"b")
    base = bytes(rng.integers(97, 123, 60, dtype=np.uint8))
    for i in range(200):
        tail = bytes(rng.integers(1, 256, int(rng.integers(0, 12)), dtype=np.uint8))
        out.append(base[: 48 + i % 13] + tail)
    out += [b"same string"] * 40
    out += [b"x" * 300 + bytes([65 + i % 3]) for i in range(70)]
    return out


def cases():
    yield "edge_mixed", pkg.pack_strings(edge_strings())
    c, o, _ = W.digits(seed=1, budget=256 * 1024)
    yield "digits_256k", (c, o)
    c, o, _ = W.random_strings(6000, 0, 20, b"ab", seed=5)
    yield "alpha_ab", (c, o)
    c, o, _ = W.prefixes(n=30000, seed=2)
    yield "prefix_30k", (c, o)
    c, o, _ = W.dna_suffixes(length=65536, seed=3)
    yield "dna_suffix_64k", (c, o)
    c, o, _ = W.random_strings(3000, 0, 600, b"\x01\xfe\xff", seed=9)
    yield "highbyte_long", (c, o)


def main():
    for name, (chars, offs) in cases():
        chars = np.ascontiguousarray(chars, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        ids, lcp = orc.ref_sort(chars, offs, threads=4, lcp=True)
        assert orc.check_order(chars, offs, ids) == -1
        cids = canonical_ids(chars, offs, ids, lcp)
        nch = int(offs.max()) + 1 if len(offs) else 1
        end = chars.tobytes().index(b"\0", nch - 1) + 1
        np.savez_compressed(HERE / f"{name}.npz", chars=chars[:end], offs=offs, ids=cids,
                            lcp=lcp.astype(np.uint64))
        print(name, len(offs), "strings,", end, "chars")


if __name__ == "__main__":
    main()
