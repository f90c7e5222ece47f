"""Tensor-core (tcgen05, TF32 hi/lo split) M2L against the SIMT FP32 GEMM
and the FP64 form.  The two FP32 engines differ only by rounding."""
import os

import numpy as np
import pytest

from laplace_fmm_b200 import Context, FastMultipole3d
from laplace_fmm_b200.workloads import plummer_mix3d, rel_l2, uniform3d

pytestmark = pytest.mark.gpu


def simt_context():
    os.environ["LFMM_M2L"] = "simt"
    try:
        return Context(0)
    finally:
        del os.environ["LFMM_M2L"]


def noself(p, q):
    return p - q * 1e4


@pytest.mark.parametrize("N", [13, 9, 5])
def test_tc_matches_simt_uniform(ctx, N):
    src, q = uniform3d(262144, seed=40 + N)
    simt = simt_context()
    a = FastMultipole3d((src, q), N=N, tree_depth=6, precision="mixed")
    b = FastMultipole3d((src, q), N=N, tree_depth=6, precision="mixed", ctx=simt)
    c = FastMultipole3d((src, q), N=N, tree_depth=6)
    assert rel_l2(noself(a.potentials, q), noself(b.potentials, q)) < 2e-7
    assert rel_l2(a.forces, b.forces) < 2e-7
    assert rel_l2(noself(a.potentials, q), noself(c.potentials, q)) < 1e-6
    assert rel_l2(a.forces, c.forces) < 1e-6
    simt.close()


def test_tc_adaptive(ctx):
    src, q = plummer_mix3d(400000, seed=41)
    simt = simt_context()
    a = FastMultipole3d((src, q), N=13, tree_depth=10, max_leaf=64, precision="mixed")
    b = FastMultipole3d((src, q), N=13, tree_depth=10, max_leaf=64, precision="mixed", ctx=simt)
    assert rel_l2(noself(a.potentials, q), noself(b.potentials, q)) < 2e-7
    assert rel_l2(a.forces, b.forces) < 2e-7
    simt.close()
