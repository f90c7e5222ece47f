"""Device-side check failures of asynchronous solves (device buffers, no
stats) are latched when the solve ends and reported by lfmm_check; a
synchronising call reports them itself.  The failure is raised on the host's
request (lfmm_debug_raise_flags sets the flag word as a failing check
would), so no kernel is made to fail."""
import ctypes

import numpy as np
import pytest

from laplace_fmm_b200._lib import LfmmSolveOpts, LfmmStats

pytestmark = pytest.mark.gpu
ERR_DEVICE = -4


def _bufs(n, seed=3):
    import torch
    g = np.random.default_rng(seed)
    src = torch.from_numpy(g.random((n, 3))).cuda()
    q = torch.from_numpy(g.uniform(-1, 1, n)).cuda()
    pot = torch.zeros(n, dtype=torch.float64, device="cuda")
    fld = torch.zeros(n, 3, dtype=torch.float64, device="cuda")
    return src, q, pot, fld


def _solve(ctx, b, stats=None):
    src, q, pot, fld = b
    vp = ctypes.c_void_p
    o = LfmmSolveOpts(9, 6, 32, 1, 1e-8)
    return ctx.lib.lfmm3d_solve_ex_device(ctx.handle, len(q), vp(src.data_ptr()), vp(q.data_ptr()), 0, None,
                                          ctypes.byref(o), vp(pot.data_ptr()), vp(fld.data_ptr()),
                                          ctypes.byref(stats) if stats is not None else None)


def test_async_solve_error_reported_by_check(ctx):
    b = _bufs(20000)
    L = ctx.lib
    assert _solve(ctx, b) == 0
    assert L.lfmm_check(ctx.handle) == 0
    ref = b[2].clone(), b[3].clone()
    # a flag raised before an asynchronous solve is latched at its end
    assert L.lfmm_debug_raise_flags(ctx.handle, 8) == 0
    assert _solve(ctx, b) == 0
    assert L.lfmm_check(ctx.handle) == ERR_DEVICE
    assert "flags 8" in L.lfmm_last_error(ctx.handle).decode()
    # reported once, and the device word was cleared: the next solve is clean
    assert L.lfmm_check(ctx.handle) == 0
    assert _solve(ctx, b) == 0
    assert L.lfmm_check(ctx.handle) == 0
    assert bool((b[2] == ref[0]).all()) and bool((b[3] == ref[1]).all())


def test_sync_solve_reports_its_own_error(ctx):
    b = _bufs(20000, seed=4)
    L = ctx.lib
    assert L.lfmm_debug_raise_flags(ctx.handle, 1) == 0
    assert _solve(ctx, b, LfmmStats()) == ERR_DEVICE
    assert L.lfmm_check(ctx.handle) == 0
    assert _solve(ctx, b, LfmmStats()) == 0


def test_plan_execute_latches(ctx):
    b = _bufs(20000, seed=5)
    src, q, pot, fld = b
    L = ctx.lib
    vp = ctypes.c_void_p
    hp = vp()
    o = LfmmSolveOpts(9, 6, 32, 1, 1e-8)
    ctx.check(L.lfmm3d_plan_create(ctx.handle, len(q), vp(src.data_ptr()), vp(q.data_ptr()), ctypes.byref(o),
                                   ctypes.byref(hp)), "plan")
    try:
        assert L.lfmm3d_plan_execute(hp, vp(q.data_ptr()), vp(pot.data_ptr()), vp(fld.data_ptr())) == 0
        assert L.lfmm_check(ctx.handle) == 0
        assert L.lfmm_debug_raise_flags(ctx.handle, 2) == 0
        assert L.lfmm3d_plan_execute(hp, vp(q.data_ptr()), vp(pot.data_ptr()), vp(fld.data_ptr())) == 0
        assert L.lfmm_check(ctx.handle) == ERR_DEVICE
        assert L.lfmm_check(ctx.handle) == 0
    finally:
        L.lfmm3d_plan_destroy(hp)
