"""Opt-in tensor-core (tcgen05, TF32 hi/lo split) M2L engine against the
default SIMT FP32 GEMM.  Measured accuracy of the tcgen05 engine: ~1e-5
relative to the FP64 form (its FP32 accumulation inside TMEM keeps fewer bits
than the SIMT GEMM's per-offset FP32 partials carried in FP64, 2e-7); the
bound below is that measured level, not the mixed form's 1e-6."""
import os

import pytest

from laplace_fmm_b200 import Context, FastMultipole3d
from laplace_fmm_b200.workloads import plummer_mix3d, rel_l2, uniform3d

pytestmark = pytest.mark.gpu
TC_TOL = 3e-5


def tc_context():
    os.environ["LFMM_M2L"] = "tc"
    try:
        return Context(0)
    finally:
        del os.environ["LFMM_M2L"]


def noself(p, q):
    return p - q * 1e4


@pytest.mark.parametrize("N", [13, 9, 5])
def test_tc_engine_uniform(ctx, N):
    src, q = uniform3d(262144, seed=40 + N)
    tc = tc_context()
    a = FastMultipole3d((src, q), N=N, tree_depth=6, precision="mixed", ctx=tc)
    b = FastMultipole3d((src, q), N=N, tree_depth=6, precision="mixed")
    c = FastMultipole3d((src, q), N=N, tree_depth=6)
    assert rel_l2(noself(a.potentials, q), noself(b.potentials, q)) < TC_TOL
    assert rel_l2(a.forces, b.forces) < TC_TOL
    assert rel_l2(noself(b.potentials, q), noself(c.potentials, q)) < 1e-6
    tc.close()


def test_tc_engine_adaptive(ctx):
    src, q = plummer_mix3d(400000, seed=41)
    tc = tc_context()
    a = FastMultipole3d((src, q), N=13, tree_depth=10, max_leaf=64, precision="mixed", ctx=tc)
    b = FastMultipole3d((src, q), N=13, tree_depth=10, max_leaf=64, precision="mixed")
    assert rel_l2(noself(a.potentials, q), noself(b.potentials, q)) < TC_TOL
    assert rel_l2(a.forces, b.forces) < TC_TOL
    tc.close()
