"""CUDA 2D FMM (FP64) against the oracle, the golden fixtures and the direct
sum; trees bit-exact."""
from pathlib import Path

import numpy as np
import pytest

from helpers import assert_trees_equal, gpu_tree
from laplace_fmm_b200 import FastMultipole, InteractionType, compute_exact
from laplace_fmm_b200.workloads import clustered2d, rel_l2

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
TOL = 1e-12


def rng(s):
    return np.random.Generator(np.random.PCG64(s))


@pytest.mark.parametrize("n,depth", [(20000, 6), (3000, 4), (1, 3)])
def test_tree_bit_exact(ctx, oracle, n, depth):
    g = rng(n)
    pts = g.random((n, 2)); q = g.uniform(-1, 1, n)
    a = gpu_tree(ctx, 2, pts, q, depth)
    b = oracle.tree(2, pts, q, depth, halved=False)
    assert_trees_equal(a, b, n)


@pytest.mark.parametrize("name", ["c2d_src", "c2d_st", "c2d_n30"])
def test_golden(ctx, name):
    g = dict(np.load(GOLD / f"{name}.npz"))
    tgt = g.get("tgt")
    if tgt is None:
        f = FastMultipole((g["src"], g["q"]), N=int(g["N"]), tree_depth=int(g["depth"]))
    else:
        f = FastMultipole((g["src"], g["q"]), tgt, N=int(g["N"]), tree_depth=int(g["depth"]))
    assert rel_l2(f.potentials, g["pot"]) < TOL
    fld = np.stack([f.forces.real, f.forces.imag], axis=1)
    assert rel_l2(fld, g["field"]) < TOL


@pytest.mark.parametrize("n,N,depth", [(100000, 21, 7), (20000, 10, 5), (5000, 30, 4), (3000, 1, 4), (300000, 21, 9)])
def test_parity_with_oracle(ctx, oracle, n, N, depth):
    g = rng(n + N)
    src = g.random((n, 2)); q = g.uniform(-1, 1, n)
    f = FastMultipole((src, q), N=N, tree_depth=depth)
    pot, fld = oracle.fmm2d(src, q, N=N, depth=depth)
    assert rel_l2(f.potentials, pot) < TOL
    assert rel_l2(np.stack([f.forces.real, f.forces.imag], 1), fld) < TOL


def test_clustered_source_target(ctx, oracle):
    src, q = clustered2d(40000, seed=1)
    tgt = rng(2).random((5000, 2))
    f = FastMultipole((src, q), tgt, N=16, tree_depth=6)
    pot, fld = oracle.fmm2d(src, q, targets=tgt, N=16, depth=6)
    assert rel_l2(f.potentials, pot) < TOL
    assert rel_l2(np.stack([f.forces.real, f.forces.imag], 1), fld) < TOL


def test_accuracy_vs_direct(ctx):
    src, q = clustered2d(200000, seed=3)
    f = FastMultipole((src, q), N=21, tree_depth=7)
    idx = np.sort(rng(4).choice(len(src), 4096, replace=False))
    pe = compute_exact(InteractionType.Potential2d, (src, q), src[idx])
    fe = compute_exact(InteractionType.Force2d, (src, q), src[idx])
    assert rel_l2(f.potentials[idx], pe) < 1e-9
    assert rel_l2(f.forces[idx], fe) < 1e-8


@pytest.mark.parametrize("ns,nt", [(4000, 500), (100000, 37), (3, 2000)])
def test_direct_matches_oracle(ctx, oracle, ns, nt):
    """Few targets against many sources take the source-split direct sum."""
    g = rng(ns + nt)
    src = g.random((ns, 2)); q = g.uniform(-1, 1, ns)
    tgt = g.random((nt, 2))
    pe = compute_exact(InteractionType.Potential2d, (src, q), tgt)
    fe = compute_exact(InteractionType.Force2d, (src, q), tgt)
    po, fo = oracle.direct2d(src, q, tgt)
    assert rel_l2(pe, po) < 1e-13
    assert rel_l2(np.stack([fe.real, fe.imag], 1), fo) < 1e-13


def engine_context(name):
    import os
    from laplace_fmm_b200 import Context
    os.environ["LFMM_M2L"] = name
    try:
        return Context(0)
    finally:
        del os.environ["LFMM_M2L"]


@pytest.mark.parametrize("n,N,depth", [(400000, 20, 9), (50000, 30, 6), (20000, 3, 5), (30000, 9, 6),
                                       (30000, 17, 6), (30000, 25, 6), (200000, 21, 11)])
def test_m2l_engines_agree(ctx, n, N, depth):
    """The default 2D M2L (the Hankel factorisation, grouped by quadrant class
    and offset), the dense-operator GEMMs and the per-pair warp kernel: the
    same sums in other orders."""
    pair, dense = engine_context("rotation"), engine_context("simt")
    src, q = clustered2d(n, seed=N)
    a = FastMultipole((src, q), N=N, tree_depth=depth, ctx=ctx)
    b = FastMultipole((src, q), N=N, tree_depth=depth, ctx=pair)
    c = FastMultipole((src, q), N=N, tree_depth=depth, ctx=dense)
    pair.close()
    dense.close()
    for other in (b, c):
        assert rel_l2(a.potentials, other.potentials) < 1e-13
        assert rel_l2(a.forces, other.forces) < 1e-13


@pytest.mark.parametrize("n,depth", [(200000, 10), (200000, 11)])
def test_parity_with_oracle_deep_clustered(ctx, oracle, n, depth):
    """The configuration's clustered mixture on the reference's uniform
    quadtree at the depths its full size uses (10-11 levels)."""
    src, q = clustered2d(n, seed=depth)
    f = FastMultipole((src, q), N=21, tree_depth=depth)
    pot, fld = oracle.fmm2d(src, q, N=21, depth=depth)
    assert rel_l2(f.potentials, pot) < TOL
    assert rel_l2(np.stack([f.forces.real, f.forces.imag], 1), fld) < TOL
