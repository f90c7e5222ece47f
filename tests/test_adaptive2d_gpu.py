"""Adaptive quadtree (2D, FP64): the GPU's cells and U / W / X / V lists equal
the CPU restatement (oracle/adaptive.py) and cover every (target leaf,
source) pair exactly once; solves on clustered sets against the FP64 direct
sum at sampled targets, with and without separate targets."""
import numpy as np
import pytest

from helpers import gpu_adaptive_tree
from laplace_fmm_b200 import FastMultipole, InteractionType, compute_exact
from laplace_fmm_b200.workloads import clustered2d, rel_l2, sample_targets
from oracle import adaptive as A

pytestmark = pytest.mark.gpu
LOG_EPS = np.log(1e-4)


def rng(s):
    return np.random.Generator(np.random.PCG64(s))


@pytest.mark.parametrize("n,depth,max_leaf,sigma", [(6000, 10, 16, 0.005), (12000, 12, 32, 0.005),
                                                     (8000, 9, 16, 0.05), (3000, 6, 16, None)])
def test_quadtree_lists_match_the_restatement(ctx, oracle, n, depth, max_leaf, sigma):
    if sigma is None:
        g = rng(n)
        pos, q = g.random((n, 2)), g.uniform(-1, 1, n)
    else:
        pos, q = clustered2d(n, seed=200 + depth, clusters=8, sigma=sigma)
    cells, lists, send, _ = gpu_adaptive_tree(ctx, pos, q, depth, max_leaf, dim=2)
    ref = A.adaptive_from_uniform(oracle.tree(2, pos, q, depth, halved=False), max_leaf, dim=2)
    for key in ("level", "code", "parent", "pbeg", "pend", "is_leaf", "leaves"):
        np.testing.assert_array_equal(cells[key], ref[key], err_msg=key)
    R = A.lists(ref)
    for name in "UWXV":
        assert len(lists[name]) == len(R[name])
        for r, (a, b) in enumerate(zip(lists[name], R[name])):
            np.testing.assert_array_equal(a, b, err_msg=f"{name} row {r}")
    cells["coords"] = ref["coords"]
    A.assert_covered_once(cells, lists, n, send)


def _check_direct(f, src, q, idx, tpos=None, tol_pot=1e-9, tol_fld=1e-8):
    tg = src[idx] if tpos is None else tpos[idx]
    pe = compute_exact(InteractionType.Potential2d, (src, q), tg)
    fe = compute_exact(InteractionType.Force2d, (src, q), tg)
    self_t = q[idx] * LOG_EPS if tpos is None else 0.0
    ep = rel_l2(f.potentials[idx] - self_t, pe - self_t)
    ef = rel_l2(f.forces[idx], fe)
    assert ep < tol_pot and ef < tol_fld, (ep, ef)
    return ep, ef


@pytest.mark.parametrize("n,N,depth,max_leaf", [(300000, 21, 12, 32), (100000, 12, 12, 16), (50000, 30, 10, 64)])
def test_adaptive_vs_direct(ctx, n, N, depth, max_leaf):
    """The configuration's mixture (half uniform, half on 64 Gaussians of
    sigma 0.005) on adaptive quadtrees: rel-L2 of potential (self term
    removed) and field at 4096 sampled targets."""
    src, q = clustered2d(n, seed=n + N)
    f = FastMultipole((src, q), N=N, tree_depth=depth, max_leaf=max_leaf)
    assert f.stats["n_w"] > 0 and f.stats["n_x"] > 0 and f.stats["depth"] > 6
    tol = {21: (1e-9, 1e-8), 12: (1e-6, 1e-5), 30: (1e-11, 1e-10)}[N]
    _check_direct(f, src, q, sample_targets(n), tol_pot=tol[0], tol_fld=tol[1])


def _dense_line(seed):
    """A strip 1e-3 wide holding 40,000 particles beside a sparse background:
    coarse leaves border long runs of fine ones (U lists above 100 entries,
    W lists above 150), and no cell is smaller than the 1e-4 distance clamp
    (a tree with cells below it no longer matches the clamped direct sum)."""
    g = rng(seed)
    bg = g.random((3000, 2))
    ln = np.stack([0.5 + 1e-3 * g.random(40000), g.random(40000)], 1)
    src = np.concatenate([bg, ln])
    return src, g.uniform(-1, 1, len(src))


def test_adaptive_dense_line_lists(ctx, oracle):
    src, q = _dense_line(7)
    cells, lists, send, _ = gpu_adaptive_tree(ctx, src, q, 16, 32, dim=2)
    assert max(len(u) for u in lists["U"]) > 64
    ref = A.adaptive_from_uniform(oracle.tree(2, src, q, 16, halved=False), 32, dim=2)
    R = A.lists(ref)
    for name in "UWXV":
        for r, (a, b) in enumerate(zip(lists[name], R[name])):
            np.testing.assert_array_equal(a, b, err_msg=f"{name} row {r}")
    cells["coords"] = ref["coords"]
    A.assert_covered_once(cells, lists, len(src), send)


def test_adaptive_dense_line(ctx):
    src, q = _dense_line(7)
    f = FastMultipole((src, q), N=21, tree_depth=16, max_leaf=32)
    assert f.stats["depth"] >= 10
    _check_direct(f, src, q, sample_targets(len(src)))


def test_adaptive_source_target(ctx):
    src, q = clustered2d(80000, seed=9)
    tgt = np.concatenate([rng(10).random((3000, 2)), clustered2d(3000, seed=11)[0]])
    f = FastMultipole((src, q), tgt, N=21, tree_depth=12, max_leaf=32)
    _check_direct(f, src, q, np.arange(len(tgt)), tpos=tgt)


def test_adaptive_agrees_with_uniform(ctx):
    """On a uniform set the adaptive quadtree and the reference's uniform
    quadtree give the same answer to the truncation error."""
    g = rng(12)
    src = g.random((60000, 2)); q = g.uniform(-1, 1, 60000)
    fa = FastMultipole((src, q), N=25, tree_depth=8, max_leaf=8)
    fu = FastMultipole((src, q), N=25, tree_depth=7)
    assert rel_l2(fa.potentials, fu.potentials) < 1e-11
    assert rel_l2(fa.forces, fu.forces) < 1e-10
