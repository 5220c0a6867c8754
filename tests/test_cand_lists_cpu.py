"""The two-level candidate-list build's exactness argument, restated on the CPU on random leaf boxes.

desert-search_b200/csrc/world.cu (k_cand) keeps, for each cell [A, B] of a 5-axis grid, the leaves whose least
squared distance to the cell is at most the least max-distance of any leaf of the same depth interval.  It
builds the lists of a coarse grid (every second cut of each axis) from all leaves first, then each cell's list
from its coarse cell's list only.  This test checks that both give the same lists, in leaf order.
"""
import itertools

import numpy as np


def spans(lo, hi, A, B):
    """Per leaf: least and greatest squared distance to the box [A, B] (leaf_span)."""
    d0 = np.maximum(np.maximum(lo - B, A - hi), 0)
    da = np.maximum(np.maximum(lo - A, A - hi), 0)
    db = np.maximum(np.maximum(lo - B, B - hi), 0)
    d1 = np.maximum(da, db)
    return (d0 * d0).sum(1), (d1 * d1).sum(1)


def cell_list(lo, hi, cls, A, B, src):
    mn, mx = spans(lo[src], hi[src], A, B)
    best = {c: mx[cls[src] == c].min() for c in set(cls[src])}
    return [int(k) for k, m, c in zip(src, mn, cls[src]) if m <= best[c]]


def cells(cuts):
    for idx in itertools.product(*[range(len(c) - 1) for c in cuts]):
        yield idx, np.array([c[i] for c, i in zip(cuts, idx)]), np.array([c[i + 1] - 1 for c, i in zip(cuts, idx)])


def test_lists_from_coarse_lists_equal_direct_lists():
    rng = np.random.default_rng(13)
    dropped_coarse = dropped_fine = 0
    for _ in range(6):
        n = 60
        lo = rng.integers(-100, 100, (n, 5))
        hi = lo + rng.integers(0, 10, (n, 5))
        cls = rng.integers(0, 3, n)
        cuts = [np.unique(np.concatenate([[-110, 110], rng.integers(-100, 100, 4)])) for _ in range(5)]
        coarse_cuts = [c[[min(2 * j, len(c) - 1) for j in range(len(c) // 2 + 1)]] for c in cuts]   # every second cut
        coarse = {idx: cell_list(lo, hi, cls, A, B, np.arange(n)) for idx, A, B in cells(coarse_cuts)}
        for idx, A, B in cells(cuts):
            direct = cell_list(lo, hi, cls, A, B, np.arange(n))
            src = coarse[tuple(i // 2 for i in idx)]
            via = cell_list(lo, hi, cls, A, B, np.array(src, dtype=np.int64))
            assert via == direct, (idx, via, direct)
            dropped_coarse += n - len(src)
            dropped_fine += len(src) - len(via)
    assert dropped_coarse > 0 and dropped_fine > 0      # both levels drop leaves on these cases
