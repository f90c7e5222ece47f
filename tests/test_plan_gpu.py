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
