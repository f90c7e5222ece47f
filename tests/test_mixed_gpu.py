"""Mixed-precision 3D form (FP32 scaled expansions below level 4, FP32 near
field with FP64 tile sums) against the plain FP64 form and the FP64 direct
sum.  Stated tolerance of the mixed form: its difference from the plain FP64
form, relative L2 with the self term removed, <= 1e-6 (MIXED_TOL); its error
against direct summation stays within 1.3x of the plain form's."""
import numpy as np
import pytest

from laplace_fmm_b200 import FastMultipole3d, InteractionType, compute_exact
from laplace_fmm_b200.workloads import plummer_mix3d, rel_l2, uniform3d

pytestmark = pytest.mark.gpu
MIXED_TOL = 1e-6


def noself(pot, q):
    return pot - q * 1e4


@pytest.mark.parametrize("N,depth", [(13, 5), (9, 5), (11, 6), (5, 4), (13, 3)])
def test_mixed_vs_plain_uniform(ctx, N, depth):
    src, q = uniform3d(131072, seed=N + depth)
    a = FastMultipole3d((src, q), N=N, tree_depth=depth)
    b = FastMultipole3d((src, q), N=N, tree_depth=depth, precision="mixed")
    assert rel_l2(noself(b.potentials, q), noself(a.potentials, q)) < MIXED_TOL
    assert rel_l2(b.forces, a.forces) < MIXED_TOL


def test_mixed_clustered_vs_direct(ctx):
    src, q = plummer_mix3d(400000, seed=5)
    a = FastMultipole3d((src, q), N=13, tree_depth=6)
    b = FastMultipole3d((src, q), N=13, tree_depth=6, precision="mixed")
    idx = np.sort(np.random.Generator(np.random.PCG64(777)).choice(len(src), 4096, replace=False))
    pe = compute_exact(InteractionType.Potential3d, (src, q), src[idx])
    fe = compute_exact(InteractionType.Force3d, (src, q), src[idx])
    ea = rel_l2(noself(a.potentials[idx], q[idx]), noself(pe, q[idx]))
    eb = rel_l2(noself(b.potentials[idx], q[idx]), noself(pe, q[idx]))
    fa, fb = rel_l2(a.forces[idx], fe), rel_l2(b.forces[idx], fe)
    assert eb < 1.3 * ea + 2e-7 and fb < 1.3 * fa + 2e-7
    assert rel_l2(noself(b.potentials, q), noself(a.potentials, q)) < MIXED_TOL


def test_mixed_source_target(ctx):
    src, q = uniform3d(60000, seed=9)
    tgt = np.random.Generator(np.random.PCG64(10)).random((20000, 3)) * 1.2 - 0.1
    a = FastMultipole3d((src, q), tgt, N=11, tree_depth=5)
    b = FastMultipole3d((src, q), tgt, N=11, tree_depth=5, precision="mixed")
    assert rel_l2(b.potentials, a.potentials) < MIXED_TOL
    assert rel_l2(b.forces, a.forces) < MIXED_TOL


def test_mixed_clamps_the_order_like_the_reference(ctx):
    """N above 18 runs at 18, as the reference clamps it (common/defs.h:31)."""
    src, q = uniform3d(3000, seed=1)
    a = FastMultipole3d((src, q), N=25, tree_depth=3, precision="mixed")
    b = FastMultipole3d((src, q), N=18, tree_depth=3, precision="mixed")
    assert np.array_equal(a.potentials, b.potentials) and np.array_equal(a.forces, b.forces)
