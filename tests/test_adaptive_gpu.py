"""Adaptive octree solver (max-per-leaf split, U/V/W/X lists; no reference
counterpart) against the FP64 direct sum, and its mixed form against its FP64
form.  A missing or doubled interaction shows up as an error of order 1e-2,
far above these bounds."""
import numpy as np
import pytest

from laplace_fmm_b200 import FastMultipole3d, InteractionType, compute_exact
from laplace_fmm_b200.workloads import gaussian_mix3d, plummer_mix3d, rel_l2, uniform3d

pytestmark = pytest.mark.gpu


def noself(pot, q):
    return pot - q * 1e4


def direct(src, q, idx, targets=None):
    t = src[idx] if targets is None else targets[idx]
    return (compute_exact(InteractionType.Potential3d, (src, q), t),
            compute_exact(InteractionType.Force3d, (src, q), t))


def sample(n, k=2048, seed=777):
    return np.sort(np.random.Generator(np.random.PCG64(seed)).choice(n, min(n, k), replace=False))


@pytest.mark.parametrize("gen,n,max_leaf,depth", [("plummer", 200000, 64, 10), ("plummer", 50000, 16, 12),
                                                  ("gauss", 100000, 32, 10), ("uniform", 100000, 64, 8)])
def test_adaptive_fp64_vs_direct(ctx, gen, n, max_leaf, depth):
    if gen == "plummer":
        src, q = plummer_mix3d(n, seed=11)
    elif gen == "gauss":
        src, q = gaussian_mix3d(n, seed=12)
    else:
        src, q = uniform3d(n, seed=13)
    f = FastMultipole3d((src, q), N=13, tree_depth=depth, max_leaf=max_leaf)
    idx = sample(n)
    pe, fe = direct(src, q, idx)
    ep = rel_l2(noself(f.potentials[idx], q[idx]), noself(pe, q[idx]))
    ef = rel_l2(f.forces[idx], fe)
    print(gen, n, max_leaf, "pot", ep, "field", ef, {k: f.stats[k] for k in ("n_leaves", "n_w", "n_x", "depth")})
    assert ep < 3e-6 and ef < 5e-6


def test_adaptive_has_w_and_x_lists(ctx):
    src, q = plummer_mix3d(200000, seed=11)
    f = FastMultipole3d((src, q), N=9, tree_depth=10, max_leaf=64)
    assert f.stats["n_w"] > 0 and f.stats["n_x"] > 0 and f.stats["depth"] > 6


def test_adaptive_mixed_vs_fp64(ctx):
    src, q = plummer_mix3d(300000, seed=21)
    a = FastMultipole3d((src, q), N=13, tree_depth=10, max_leaf=64)
    b = FastMultipole3d((src, q), N=13, tree_depth=10, max_leaf=64, precision="mixed")
    assert rel_l2(noself(b.potentials, q), noself(a.potentials, q)) < 1e-6
    assert rel_l2(b.forces, a.forces) < 1e-6


def test_adaptive_source_target(ctx):
    src, q = plummer_mix3d(80000, seed=31)
    tgt = np.random.Generator(np.random.PCG64(32)).random((20000, 3))
    f = FastMultipole3d((src, q), tgt, N=13, tree_depth=10, max_leaf=32)
    idx = sample(len(tgt))
    pe, fe = direct(src, q, idx, targets=tgt)
    assert rel_l2(f.potentials[idx], pe) < 3e-6
    assert rel_l2(f.forces[idx], fe) < 5e-6


def test_adaptive_single_leaf_is_direct(ctx):
    """max_leaf above n: the root is the only leaf, the result is the direct sum."""
    src, q = uniform3d(3000, seed=5)
    f = FastMultipole3d((src, q), N=5, tree_depth=6, max_leaf=5000)
    pe, fe = direct(src, q, np.arange(3000))
    assert rel_l2(f.potentials, pe) < 1e-6 and rel_l2(f.forces, fe) < 1e-6


@pytest.mark.parametrize("kind,n,depth,max_leaf", [("plummer", 20000, 10, 64), ("plummer", 4000, 8, 16),
                                                   ("gaussian", 12000, 9, 64), ("uniform", 3000, 5, 16)])
def test_adaptive_lists_match_the_restatement(ctx, oracle, kind, n, depth, max_leaf):
    """The GPU's adaptive cells equal the CPU restatement's (built from the
    oracle's uniform tree): levels, codes, parents, particle ranges, leaf
    flags; its U, W, X lists and the V lists of its M2L slot tables equal the
    restatement's as sets, row by row; and on the GPU's own lists every
    (target leaf, source particle) pair is covered exactly once."""
    from helpers import gpu_adaptive_tree
    from laplace_fmm_b200.workloads import gaussian_mix3d
    from oracle import adaptive as A
    gen = {"plummer": plummer_mix3d, "gaussian": gaussian_mix3d, "uniform": uniform3d}[kind]
    pos, q = gen(n, seed=170 + depth)
    cells, lists, send, _ = gpu_adaptive_tree(ctx, pos, q, depth, max_leaf)
    ref = A.adaptive_from_uniform(oracle.tree(3, pos, q, depth, halved=False), max_leaf)
    for key in ("level", "code", "parent", "pbeg", "pend", "is_leaf", "leaves"):
        np.testing.assert_array_equal(cells[key], ref[key], err_msg=key)
    R = A.lists(ref)
    for name in "UWXV":
        assert len(lists[name]) == len(R[name])
        for r, (a, b) in enumerate(zip(lists[name], R[name])):
            np.testing.assert_array_equal(a, b, err_msg=f"{name} row {r}")
    cells["coords"] = ref["coords"]
    A.assert_covered_once(cells, lists, n, send)


def test_adaptive_lists_with_targets_cover_every_source(ctx):
    """Separate targets (zero charges) share the leaves with sources; the
    lists still account once for every (target leaf, source) pair."""
    from helpers import gpu_adaptive_tree
    from oracle import adaptive as A
    src, q = plummer_mix3d(6000, seed=181)
    tgt = np.random.default_rng(182).random((2000, 3))
    cells, lists, send, _ = gpu_adaptive_tree(ctx, src, q, 9, 32, targets=tgt)
    A.assert_covered_once(cells, lists, 8000, send)
