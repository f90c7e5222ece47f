"""Adaptive-tree interaction lists on the CPU: the restatement in
oracle/adaptive.py (brute force over every cell, from the lists'
definitions) covers every (target leaf, source particle) pair exactly once
-- near field, W, and the X and V lists of the leaf and its ancestors -- on
clustered and uniform sets at several leaf sizes; and the coverage check
catches a missing or doubled interaction planted in those lists."""
import numpy as np
import pytest

from laplace_fmm_b200.workloads import clustered2d, gaussian_mix3d, plummer_mix3d, uniform3d
from oracle import adaptive as A

CASES = [("plummer", 4000, 8, 16), ("plummer", 20000, 10, 64), ("gaussian", 6000, 8, 16),
         ("gaussian", 12000, 9, 64), ("uniform", 3000, 5, 16)]


def _set(kind, n, seed):
    if kind == "plummer":
        return plummer_mix3d(n, seed=seed)
    if kind == "gaussian":
        return gaussian_mix3d(n, seed=seed)
    return uniform3d(n, seed=seed)


@pytest.fixture(scope="module")
def built(oracle):
    out = {}
    for i, (kind, n, depth, ml) in enumerate(CASES):
        pos, q = _set(kind, n, 70 + i)
        cells = A.adaptive_from_uniform(oracle.tree(3, pos, q, depth, halved=False), ml)
        out[i] = (cells, A.lists(cells), n)
    return out


@pytest.mark.parametrize("case", range(len(CASES)))
def test_every_pair_covered_once(built, case):
    cells, L, n = built[case]
    assert len(cells["leaves"]) > 1
    A.assert_covered_once(cells, L, n)


def test_lists_are_nonempty_where_the_tree_is_adaptive(built):
    """The clustered sets have leaves on several levels, so W and X are used."""
    cells, L, _ = built[1]
    assert len(np.unique(cells["level"][cells["leaves"]])) >= 3
    assert sum(len(w) for w in L["W"]) > 0 and sum(len(x) for x in L["X"]) > 0
    assert sum(len(w) for w in L["W"]) == sum(len(x) for x in L["X"])   # X is W's transpose


def _planted(L, kind, row, how):
    M = {k: [np.array(v) for v in vs] for k, vs in L.items()}
    r = M[kind][row]
    M[kind][row] = r[1:] if how == "drop" else np.concatenate([r, r[:1]])
    return M


@pytest.mark.parametrize("kind,how", [("V", "drop"), ("V", "double"), ("W", "drop"), ("X", "drop"),
                                      ("U", "drop"), ("U", "double")])
def test_planted_mistake_is_caught(built, kind, how):
    cells, L, n = built[1]
    rows = [i for i, r in enumerate(L[kind]) if len(r)]
    M = _planted(L, kind, rows[len(rows) // 2], how)
    with pytest.raises(AssertionError, match="covered"):
        A.assert_covered_once(cells, M, n)


# quadtrees: the 2D half-uniform / half-clustered mixture (64 Gaussians of
# sigma 0.005 and wider ones) and a uniform set
CASES2 = [("clustered", 6000, 10, 16, 0.005), ("clustered", 12000, 12, 32, 0.005),
          ("clustered", 8000, 9, 16, 0.05), ("uniform", 3000, 6, 16, None)]


def _set2(kind, n, seed, sigma):
    if kind == "clustered":
        return clustered2d(n, seed=seed, clusters=8, sigma=sigma)
    g = np.random.Generator(np.random.PCG64(seed))
    return g.random((n, 2)), g.uniform(-1, 1, n)


@pytest.fixture(scope="module")
def built2(oracle):
    out = {}
    for i, (kind, n, depth, ml, sig) in enumerate(CASES2):
        pos, q = _set2(kind, n, 90 + i, sig)
        cells = A.adaptive_from_uniform(oracle.tree(2, pos, q, depth, halved=False), ml, dim=2)
        out[i] = (cells, A.lists(cells), n)
    return out


@pytest.mark.parametrize("case", range(len(CASES2)))
def test_quadtree_every_pair_covered_once(built2, case):
    cells, L, n = built2[case]
    assert len(cells["leaves"]) > 1
    A.assert_covered_once(cells, L, n)


def test_quadtree_lists_are_adaptive(built2):
    cells, L, _ = built2[1]
    assert len(np.unique(cells["level"][cells["leaves"]])) >= 3
    assert sum(len(w) for w in L["W"]) > 0
    assert sum(len(w) for w in L["W"]) == sum(len(x) for x in L["X"])


@pytest.mark.parametrize("kind,how", [("V", "drop"), ("W", "drop"), ("X", "double"), ("U", "drop")])
def test_quadtree_planted_mistake_is_caught(built2, kind, how):
    cells, L, n = built2[1]
    rows = [i for i, r in enumerate(L[kind]) if len(r)]
    M = _planted(L, kind, rows[len(rows) // 2], how)
    with pytest.raises(AssertionError, match="covered"):
        A.assert_covered_once(cells, M, n)
