"""Solve plans (tree + CUDA graph built once, charges changed per execution)
give the result of a full solve on the same tree, for every charge vector."""
import numpy as np
import pytest

from laplace_fmm_b200 import FastMultipole3d, Plan3d
from laplace_fmm_b200.workloads import gaussian_mix3d, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-10), ("fp64", 1e-13)])
def test_plan_matches_full_solves(ctx, precision, tol):
    src, q1 = gaussian_mix3d(120000, seed=61)
    g = np.random.default_rng(62)
    q2 = g.uniform(-1, 1, len(src))
    q2[q2 == 0] = 0.5
    plan = Plan3d(src, q1, N=11, tree_depth=8, max_leaf=64, precision=precision, ctx=ctx)
    for q in (q1, q2, q1):
        pot, fld = plan.execute(q)
        f = FastMultipole3d((src, q), N=11, tree_depth=8, max_leaf=64, precision=precision, ctx=ctx)
        assert rel_l2(pot - q * 1e4, f.potentials - q * 1e4) < tol
        assert rel_l2(fld, f.forces) < tol
    plan.close()


def test_plan_rejects_automatic_order(ctx):
    src, q = gaussian_mix3d(5000, seed=63)
    with pytest.raises(Exception):
        Plan3d(src, q, N=2147483647, ctx=ctx)


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-10), ("fp64", 1e-13)])
def test_batch_plan_matches_batch_solves(ctx, precision, tol):
    """A batch plan (the forest and one graph for all problems) gives the
    batch solve's result for every charge vector, problem by problem."""
    from laplace_fmm_b200 import BatchPlan3d, solve_batch
    from laplace_fmm_b200.workloads import batch3d
    probs = batch3d(24, seed=71, nmin=2048, nmax=40000)
    plan = BatchPlan3d(probs, N=11, tree_depth=8, max_leaf=64, precision=precision, ctx=ctx)
    g = np.random.default_rng(72)
    for rep in range(3):
        charges = [c if rep != 1 else g.uniform(-1, 1, len(c)) for _, c in probs]
        pot, fld = plan.execute(np.concatenate(charges))
        res = solve_batch([(p, c) for (p, _), c in zip(probs, charges)], N=11, tree_depth=8, max_leaf=64,
                          precision=precision, ctx=ctx)
        for k, ((pk, fk), c) in enumerate(zip(res, charges)):
            b, e = int(plan.offsets[k]), int(plan.offsets[k + 1])
            assert rel_l2(pot[b:e] - c * 1e4, pk - c * 1e4) < tol, k
            assert rel_l2(fld[b:e], fk) < tol, k
    plan.close()


def test_batch_plan_rejects_bad_offsets(ctx):
    import ctypes
    from laplace_fmm_b200._lib import LfmmSolveOpts
    L = ctx.lib
    pos = np.zeros((10, 3)); q = np.ones(10)
    offs = np.array([0, 6, 4, 10], dtype=np.uint64)
    opts = LfmmSolveOpts(9, 5, 64, 1, 1e-8)
    h = ctypes.c_void_p()
    vp = ctypes.c_void_p
    assert L.lfmm3d_plan_create_batch(ctx.handle, 3, offs.ctypes.data_as(vp), pos.ctypes.data_as(vp),
                                      q.ctypes.data_as(vp), ctypes.byref(opts), ctypes.byref(h)) != 0
