"""Per-level M2L orders (lfmm3d_solve_levels): every level at the solve's order
reproduces the plain mixed solve exactly; a lower order on the finest level
changes the result by about that order's truncation error; bad arguments are
rejected."""
import ctypes

import numpy as np
import pytest

from laplace_fmm_b200 import FastMultipole3d, InteractionType, compute_exact
from laplace_fmm_b200._lib import LfmmSolveOpts
from laplace_fmm_b200.workloads import plummer_mix3d, rel_l2, sample_targets

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    return plummer_mix3d(300000, seed=31)


def test_full_orders_equal_the_plain_solve(ctx, case):
    src, q = case
    a = FastMultipole3d((src, q), N=14, tree_depth=10, max_leaf=64, precision="mixed")
    b = FastMultipole3d((src, q), N=14, tree_depth=10, max_leaf=64, precision="mixed", level_orders=[14] * 10)
    c = FastMultipole3d((src, q), N=14, tree_depth=10, max_leaf=64, precision="mixed", level_orders=[0] * 3)
    np.testing.assert_array_equal(a.potentials, b.potentials)
    np.testing.assert_array_equal(a.forces, c.forces)


def test_lower_fine_orders_cost_accuracy_gradually(ctx, case):
    src, q = case
    idx = sample_targets(len(src))
    pe = compute_exact(InteractionType.Potential3d, (src, q), src[idx]) - q[idx] * 1e4
    fe = compute_exact(InteractionType.Force3d, (src, q), src[idx])
    errs = []
    for lo in (16, 15, 13):
        f = FastMultipole3d((src, q), N=16, tree_depth=10, max_leaf=64, precision="mixed",
                            level_orders=[0] * 8 + [lo, lo])
        assert f.stats["depth"] >= 9
        errs.append((rel_l2(f.potentials[idx] - q[idx] * 1e4, pe), rel_l2(f.forces[idx], fe)))
    assert errs[0][1] < errs[2][1]          # the field feels the finest levels' order
    assert all(e[0] < 1e-5 and e[1] < 1e-4 for e in errs)


def test_bad_level_arguments(ctx, case):
    src, q = case
    L = ctx.lib
    opts = LfmmSolveOpts(14, 10, 64, 1, 1e-8)
    pot, fld = np.zeros(len(src)), np.zeros((len(src), 3))
    vp = ctypes.c_void_p
    args = (ctx.handle, len(src), src.ctypes.data_as(vp), q.ctypes.data_as(vp), 0, None, ctypes.byref(opts))
    lv = (ctypes.c_int * 23)(*([14] * 23))
    assert L.lfmm3d_solve_levels(*args, lv, 23, pot.ctypes.data_as(vp), fld.ctypes.data_as(vp), None) != 0
    neg = (ctypes.c_int * 2)(14, -1)
    assert L.lfmm3d_solve_levels(*args, neg, 2, pot.ctypes.data_as(vp), fld.ctypes.data_as(vp), None) != 0
