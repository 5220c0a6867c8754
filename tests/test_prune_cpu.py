"""The candidate-list pruning's exactness argument, restated on the CPU on random leaf boxes.

desert-search_b200/csrc/world.cu (k_cand_prune) drops leaf L from a cell's list when a leaf K of the same depth
interval is nearer than L at every integer point of the cell.  It decides that from per-axis minima of
dist_L^2 - dist_K^2 taken at the range ends and the two boxes' ends (axis_min_diff), tests each L first against
its interval's leaf of least max-distance and then the survivors against one another only.  These tests check,
on random boxes small enough to enumerate every point of the cell:
  * the per-axis candidate points give the exact minimum (dominance by enumeration = dominance by axis minima);
  * survivors-only pruning keeps exactly the leaves that no leaf of the list dominates (all pairs tested).
"""
import itertools

import numpy as np


def d2(lo, hi, v):
    d = np.maximum(np.maximum(lo - v, v - hi), 0)
    return d * d


def axis_min_diff(L, K, a, A, B):
    pts = [p for p in (A, B, L[0][a], L[1][a], K[0][a], K[1][a]) if A <= p <= B]
    return min(int(d2(L[0][a], L[1][a], p)) - int(d2(K[0][a], K[1][a], p)) for p in pts)


def dominated_by(L, K, A, B):
    return sum(axis_min_diff(L, K, a, A[a], B[a]) for a in range(5)) > 0


def max_dist(L, A, B):
    return sum(max(int(d2(L[0][a], L[1][a], A[a])), int(d2(L[0][a], L[1][a], B[a]))) for a in range(5))


def prune_all_pairs(leaves, cls, A, B):
    n = len(leaves)
    return [k for k in range(n)
            if not any(j != k and cls[j] == cls[k] and dominated_by(leaves[k], leaves[j], A, B) for j in range(n))]


def prune_survivors(leaves, cls, A, B, stats=None):
    """The kernel's order: the class's best leaf (least max-distance, then list position), then U among itself.
    stats (a dict) gets the leaves dropped by each of the two tests added to "first" and "second"."""
    n = len(leaves)
    best = {}
    for k in range(n):
        key = (max_dist(leaves[k], A, B), k)
        if cls[k] not in best or key < best[cls[k]]:
            best[cls[k]] = key
    keep = [not (best[cls[k]][1] != k and dominated_by(leaves[k], leaves[best[cls[k]][1]], A, B)) for k in range(n)]
    U = [k for k in range(n) if keep[k]]
    out = list(keep)
    for k in U:
        if any(j != k and cls[j] == cls[k] and dominated_by(leaves[k], leaves[j], A, B) for j in U):
            out[k] = False
    if stats is not None:
        stats["first"] = stats.get("first", 0) + n - len(U)
        stats["second"] = stats.get("second", 0) + len(U) - sum(out)
    return [k for k in range(n) if out[k]]


def random_case(rng, n):
    lo = rng.integers(-12, 12, (n, 5))
    hi = lo + rng.integers(0, 8, (n, 5))
    leaves = [(lo[k], hi[k]) for k in range(n)]
    cls = rng.integers(0, 3, n)
    A = rng.integers(-6, 6, 5)
    B = A + rng.integers(0, 3, 5)
    return leaves, cls, A, B


def test_axis_minima_equal_enumeration():
    rng = np.random.default_rng(3)
    for _ in range(200):
        leaves, cls, A, B = random_case(rng, 8)
        pts = np.array(list(itertools.product(*[range(A[a], B[a] + 1) for a in range(5)])))
        dist = np.stack([sum(d2(L[0][a], L[1][a], pts[:, a]) for a in range(5)) for L in leaves])
        for k, j in itertools.permutations(range(len(leaves)), 2):
            assert dominated_by(leaves[k], leaves[j], A, B) == bool(np.all(dist[j] < dist[k]))


def test_survivors_only_equals_all_pairs():
    rng = np.random.default_rng(5)
    stats = {}
    for _ in range(600):
        leaves, cls, A, B = random_case(rng, int(rng.integers(2, 16)))
        assert prune_survivors(leaves, cls, A, B, stats) == prune_all_pairs(leaves, cls, A, B)
    assert stats["first"] > 0 and stats["second"] > 0      # both tests drop leaves on these cases
