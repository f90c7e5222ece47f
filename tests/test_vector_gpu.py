"""Vector charges on the GPU (lfmm3d_solve_vector): the reference's fixtures,
the oracle, source / target mode, the zero-charge rule, the mixed form and
the device-buffer entry point."""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from laplace_fmm_b200 import FastMultipole3d
from laplace_fmm_b200.workloads import plummer_mix3d, rel_l2

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name", ["c3d_vec", "c3d_vec_st", "c3d_vec_zero"])
def test_reference_fixtures(ctx, name):
    g = dict(np.load(GOLD / f"{name}.npz"))
    args = ((g["src"], g["q"]),) if "tgt" not in g else ((g["src"], g["q"]), g["tgt"])
    f = FastMultipole3d(*args, N=int(g["N"]), tree_depth=int(g["depth"]), ctx=ctx)
    assert f.potentials.size == 0
    assert rel_l2(f.forces, g["field"]) < 1e-12


@pytest.mark.parametrize("n,N,depth", [(40000, 12, 5), (5000, 15, 4)])
def test_oracle_parity(ctx, oracle, n, N, depth):
    """The vector form runs on the scaled FP64 engine (dense direction
    operators, not the reference's rotation arithmetic) and takes differences
    of field components: measured 1.3e-12 at N = 12, bar 5e-12."""
    g = np.random.default_rng(n)
    src = g.random((n, 3)); q = g.uniform(-1, 1, (n, 3))
    f = FastMultipole3d((src, q), N=N, tree_depth=depth, ctx=ctx)
    assert rel_l2(f.forces, oracle.fmm3d_vec(src, q, N=N, depth=depth)) < 5e-12


def test_mixed_and_adaptive_against_fp64(ctx):
    src, _ = plummer_mix3d(200000, seed=61)
    q = np.random.default_rng(62).uniform(-1, 1, (len(src), 3))
    a = FastMultipole3d((src, q), N=13, tree_depth=10, max_leaf=64, precision="mixed", ctx=ctx)
    b = FastMultipole3d((src, q), N=13, tree_depth=10, max_leaf=64, precision="fp64", ctx=ctx)
    assert rel_l2(a.forces, b.forces) < 1e-6


def test_device_entry_point_matches_host(ctx):
    import torch
    from laplace_fmm_b200._lib import PRECISION, LfmmSolveOpts
    g = np.random.default_rng(63)
    src = g.random((30000, 3)); q = g.uniform(-1, 1, (30000, 3))
    host = FastMultipole3d((src, q), N=11, tree_depth=10, max_leaf=64, ctx=ctx).forces
    d_src, d_q = torch.from_numpy(src).cuda(), torch.from_numpy(q).cuda()
    d_f = torch.empty((len(src), 3), dtype=torch.float64, device="cuda")
    opts = LfmmSolveOpts(11, 10, 64, PRECISION["fp64"], 1e-8)
    vp = ctypes.c_void_p
    ctx.check(ctx.lib.lfmm3d_solve_vector_device(ctx.handle, len(src), vp(d_src.data_ptr()), vp(d_q.data_ptr()), 0,
                                                 None, ctypes.byref(opts), vp(d_f.data_ptr()), None),
              "lfmm3d_solve_vector_device")
    torch.cuda.ExternalStream(ctx.stream).synchronize()
    assert rel_l2(d_f.cpu().numpy(), host) < 1e-14
