"""Helpers shared by the fixture generator and the tests (pure numpy)."""
from __future__ import annotations

import numpy as np


def string_lengths(chars: np.ndarray, offs: np.ndarray) -> np.ndarray:
    """strlen of every string of the arena."""
    zeros = np.flatnonzero(np.asarray(chars) == 0).astype(np.uint64)
    pos = np.searchsorted(zeros, np.asarray(offs, dtype=np.uint64))
    return (zeros[pos] - np.asarray(offs, dtype=np.uint64)).astype(np.uint64)


def canonical_ids(chars, offs, ids, lcp) -> np.ndarray:
    """Sorted ids with every run of equal strings put in increasing id order;
    two correct sorts of the same input have the same canonical ids."""
    ids = np.asarray(ids, dtype=np.uint32)
    n = ids.shape[0]
    if n == 0:
        return ids.copy()
    lens = string_lengths(chars, offs)[ids]
    lcp = np.asarray(lcp, dtype=np.uint64)
    eq = np.zeros(n, dtype=bool)
    eq[1:] = (lcp[1:] == lens[1:]) & (lens[1:] == lens[:-1])
    run = np.cumsum(~eq)
    order = np.lexsort((ids, run))
    return ids[order]
