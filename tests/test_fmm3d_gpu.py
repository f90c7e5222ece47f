"""CUDA 3D FMM (plain FP64) against the oracle, the golden fixtures and the
FP64 direct sum.  Parity bar: relative L2 of the difference <= 1e-12 for
potential and field (the reference differs from itself by ~1e-16 between
thread counts), bit-exact trees and lists."""
from pathlib import Path

import numpy as np
import pytest

from helpers import assert_trees_equal, gpu_tree
from laplace_fmm_b200 import FastMultipole3d, InteractionType, compute_exact, particle3d_dtype
from laplace_fmm_b200.workloads import rel_l2

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
TOL = 1e-12


def rng(s):
    return np.random.Generator(np.random.PCG64(s))


@pytest.mark.parametrize("n,depth", [(5000, 4), (30000, 5), (100, 6), (1, 2), (2, 3)])
def test_tree_bit_exact(ctx, oracle, n, depth):
    g = rng(n)
    pts = g.random((n, 3)); q = g.uniform(-1, 1, n)
    a = gpu_tree(ctx, 3, pts, q, depth)
    b = oracle.tree(3, pts, q, depth, halved=False)
    assert_trees_equal(a, b, n)
    for L in range(depth):
        np.testing.assert_array_equal(a["levels"][L]["center"], b["levels"][L]["center"])


def test_tree_with_targets(ctx, oracle):
    g = rng(7)
    src = g.random((3000, 3)); q = g.uniform(-1, 1, 3000)
    tgt = g.random((1000, 3)) * 1.4 - 0.2
    a = gpu_tree(ctx, 3, src, q, 4, targets=tgt)
    allp = np.concatenate([tgt, src]); allq = np.concatenate([np.zeros(1000), q])
    b = oracle.tree(3, allp, allq, 4, halved=False)
    assert_trees_equal(a, b, 4000, exact_positions=False)


@pytest.mark.parametrize("name", ["c3d_src", "c3d_st", "c3d_n18", "c3d_deep"])
def test_golden(ctx, name):
    g = dict(np.load(GOLD / f"{name}.npz"))
    tgt = g.get("tgt")
    args = (g["src"], g["q"]) if tgt is None else None
    f = FastMultipole3d((g["src"], g["q"]), tgt, N=int(g["N"]), tree_depth=int(g["depth"])) if tgt is not None \
        else FastMultipole3d(args, N=int(g["N"]), tree_depth=int(g["depth"]))
    assert rel_l2(f.potentials, g["pot"]) < TOL
    assert rel_l2(f.forces, g["field"]) < TOL


@pytest.mark.parametrize("n,N,depth", [(131072, 9, 5), (20000, 13, 4), (8000, 18, 3), (4000, 1, 3), (4000, 2, 4),
                                       (50000, 5, 6)])
def test_parity_with_oracle(ctx, oracle, n, N, depth):
    g = rng(n + N)
    src = g.random((n, 3)); q = g.uniform(-1, 1, n)
    f = FastMultipole3d((src, q), N=N, tree_depth=depth)
    pot, fld = oracle.fmm3d(src, q, N=N, depth=depth)
    assert rel_l2(f.potentials, pot) < TOL
    assert rel_l2(f.forces, fld) < TOL
    assert f.N == N and f.tree_depth == depth


def test_source_target(ctx, oracle):
    g = rng(3)
    src = g.random((20000, 3)); q = g.uniform(-1, 1, 20000)
    tgt = g.random((7000, 3)) * 1.2 - 0.1
    f = FastMultipole3d((src, q), tgt, N=10, tree_depth=4)
    pot, fld = oracle.fmm3d(src, q, targets=tgt, N=10, depth=4)
    assert f.potentials.shape == (7000,)
    assert rel_l2(f.potentials, pot) < TOL and rel_l2(f.forces, fld) < TOL


def test_zero_charge_switches_to_target_mode(ctx, oracle):
    """The reference evaluates only q == 0 particles once any charge is zero."""
    g = rng(4)
    src = g.random((5000, 3)); q = g.uniform(-1, 1, 5000)
    q[::7] = 0.0
    f = FastMultipole3d((src, q), N=8, tree_depth=4)
    pot, fld = oracle.fmm3d(src, q, N=8, depth=4)
    assert np.all(f.potentials[q != 0] == 0.0)
    assert rel_l2(f.potentials, pot) < TOL and rel_l2(f.forces, fld) < TOL


def test_structured_particles_and_auto(ctx, oracle):
    g = rng(5)
    a = np.zeros(6000, particle3d_dtype)
    a["center"] = g.random((6000, 3)); a["q"] = g.uniform(-1, 1, 6000)
    f = FastMultipole3d(a, 1e-6)
    pot, fld = oracle.fmm3d(a["center"], a["q"], eps=1e-6)
    assert rel_l2(f.potentials, pot) < TOL and rel_l2(f.forces, fld) < TOL


def test_coincident_particles(ctx, oracle):
    """Distances below 1e-4 are clamped; duplicates stay finite."""
    g = rng(6)
    src = g.random((3000, 3)); q = g.uniform(-1, 1, 3000)
    src[1000:1100] = src[0]
    f = FastMultipole3d((src, q), N=9, tree_depth=4)
    pot, fld = oracle.fmm3d(src, q, N=9, depth=4)
    assert np.all(np.isfinite(f.potentials))
    assert rel_l2(f.potentials, pot) < TOL and rel_l2(f.forces, fld) < TOL


def test_accuracy_vs_direct(ctx):
    g = rng(8)
    n = 131072
    src = g.random((n, 3)); q = g.uniform(-1, 1, n)
    f = FastMultipole3d((src, q), N=13, tree_depth=5)
    idx = np.sort(g.choice(n, 4096, replace=False))
    pe = compute_exact(InteractionType.Potential3d, (src, q), src[idx])
    fe = compute_exact(InteractionType.Force3d, (src, q), src[idx])
    self_term = q[idx] * 1e4
    assert rel_l2(f.potentials[idx] - self_term, pe - self_term) < 2e-6
    assert rel_l2(f.forces[idx], fe) < 3e-6


@pytest.mark.parametrize("ns,nt", [(4000, 500), (200000, 33), (5, 3000), (1, 1)])
def test_direct_matches_oracle(ctx, oracle, ns, nt):
    """Few targets against many sources take the source-split direct sum."""
    g = rng(9 + ns)
    src = g.random((ns, 3)); q = g.uniform(-1, 1, ns)
    tgt = g.random((nt, 3))
    pe = compute_exact(InteractionType.Potential3d, (src, q), tgt)
    fe = compute_exact(InteractionType.Force3d, (src, q), tgt)
    po, fo = oracle.direct3d(src, q, tgt)
    assert rel_l2(pe, po) < 1e-13 and rel_l2(fe, fo) < 1e-13


def test_wigner_tables_match_oracle(ctx, oracle):
    import ctypes
    th = ctypes.c_double()
    d = np.zeros(18 * 19 * 71 // 6)
    nslots = ctx.lib.lfmm_wignerd_slot(ctx.handle, 0, ctypes.byref(th), d.ctypes.data_as(ctypes.c_void_p))
    assert nslots == 97
    for s in range(nslots):
        ctx.lib.lfmm_wignerd_slot(ctx.handle, s, ctypes.byref(th), d.ctypes.data_as(ctypes.c_void_p))
        assert np.abs(d - oracle.wignerd(18, th.value)).max() < 1e-11


@pytest.mark.parametrize("N,depth", [(9, 5), (13, 4), (6, 6)])
def test_m2l_engines_agree(ctx, oracle, N, depth):
    """Dense direction-GEMM M2L and per-pair rotations: both at parity."""
    import os
    from laplace_fmm_b200 import Context
    os.environ["LFMM_M2L"] = "rotation"
    try:
        rot = Context(0)
    finally:
        del os.environ["LFMM_M2L"]
    g = rng(N * 100 + depth)
    n = 60000
    src = g.random((n, 3)); q = g.uniform(-1, 1, n)
    a = FastMultipole3d((src, q), N=N, tree_depth=depth)
    b = FastMultipole3d((src, q), N=N, tree_depth=depth, ctx=rot)
    pot, fld = oracle.fmm3d(src, q, N=N, depth=depth)
    assert rel_l2(a.potentials, pot) < TOL and rel_l2(a.forces, fld) < TOL
    assert rel_l2(b.potentials, pot) < TOL and rel_l2(b.forces, fld) < TOL
    rot.close()


def test_bad_arguments(ctx):
    from laplace_fmm_b200 import LfmmError
    with pytest.raises(LfmmError):
        FastMultipole3d((np.zeros((0, 3)), np.zeros(0)), N=5, tree_depth=3)
    with pytest.raises(LfmmError):
        FastMultipole3d((np.random.rand(10, 3), np.ones(10)), N=0, tree_depth=3)
