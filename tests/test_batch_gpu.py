"""Batched solves: a forest of independent problems (each its own box and
root) solved together must give each problem the result it gets alone on
the same tree, and match the FP64 direct sum."""
import numpy as np
import pytest

from laplace_fmm_b200 import FastMultipole3d, compute_exact, InteractionType, solve_batch
from laplace_fmm_b200.workloads import batch3d, rel_l2

pytestmark = pytest.mark.gpu


def noself(p, q):
    return p - q * 1e4


@pytest.fixture(scope="module")
def problems():
    ps = batch3d(10, seed=77, nmin=1500, nmax=60000)
    g = np.random.default_rng(3)
    # a single particle, an empty problem and a shifted, scaled copy
    ps.insert(3, (g.random((1, 3)), np.array([0.5])))
    ps.insert(5, (np.zeros((0, 3)), np.zeros(0)))
    p, q = ps[0]
    ps.append((p * 37.0 - 5.0, q))
    return ps


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-6), ("fp64", 1e-12)])
def test_batch_matches_single_solves(ctx, problems, precision, tol):
    out = solve_batch(problems, N=11, tree_depth=8, max_leaf=64, precision=precision, ctx=ctx)
    assert len(out) == len(problems)
    for (pos, q), (pot, fld) in zip(problems, out):
        assert len(pot) == len(pos)
        if len(pos) < 2:
            continue
        f = FastMultipole3d((pos, q), N=11, tree_depth=8, max_leaf=64, precision=precision, ctx=ctx)
        assert rel_l2(noself(pot, q), noself(f.potentials, q)) < tol
        assert rel_l2(fld, f.forces) < tol


def test_single_particle_gets_its_self_term(ctx, problems):
    out = solve_batch(problems, N=9, tree_depth=8, max_leaf=64, ctx=ctx)
    pot, fld = out[3]
    assert pot[0] == pytest.approx(0.5 * 1e4) and np.all(fld == 0)


def test_batch_accuracy_vs_direct(ctx, problems):
    out = solve_batch(problems, N=13, tree_depth=8, max_leaf=64, ctx=ctx)
    for k in (0, 2, 4):
        pos, q = problems[k]
        idx = np.arange(0, len(pos), max(1, len(pos) // 500))
        pe = compute_exact(InteractionType.Potential3d, (pos, q), pos[idx], ctx=ctx)
        fe = compute_exact(InteractionType.Force3d, (pos, q), pos[idx], ctx=ctx)
        pot, fld = out[k]
        assert rel_l2(noself(pot[idx], q[idx]), noself(pe, q[idx])) < 3e-6
        assert rel_l2(fld[idx], fe) < 1e-5


def test_learned_batch_within_tolerance(ctx, problems):
    """The batch at the network's order: every problem within the tolerance
    on its own samples, and the same result as the fixed-order batch at that
    order."""
    from laplace_fmm_b200.order import WEIGHTS, LearnedSolver
    if not WEIGHTS.exists():
        pytest.skip("trained network not present")
    solver = LearnedSolver(ctx=ctx)
    out, info = solver.solve_batch(problems, tol=1e-6, tree_depth=8, check_targets=64)
    assert 5 <= info["order_N"] <= 18
    assert info["checked_error"] <= 1e-6 and info["checked_error_field"] <= 1e-6
    # every output of a problem of up to 8192 particles, else 64 (more where the judge extended them)
    assert info["checked_targets"] >= sum(len(p) if len(p) <= 8192 else 64 for p, _ in problems)
    if info["order_groups"] != 1:
        pytest.skip("the problems ran at several orders (the per-order groups are tested below)")
    ref = solve_batch(problems, N=info["order_N"], tree_depth=8, max_leaf=64, ctx=ctx)
    for k, ((pos, q), (pot, fld), (rp, rf)) in enumerate(zip(problems, out, ref)):
        if len(pos) < 2 or info["fp64_resolved"]:
            continue
        assert rel_l2(noself(pot, q), noself(rp, q)) < 1e-12
        assert rel_l2(fld, rf) < 1e-12


def test_learned_batch_orders_per_problem(ctx):
    """Problems that need different orders (uniform sets and tight clusters):
    each runs at its own order, the problems of each order solved together;
    every problem within the tolerance at its samples against the FP64 direct
    sum, and the threshold network picks the batch's leaf size."""
    from laplace_fmm_b200.order import WEIGHTS, LEAF_CANDIDATES, LearnedSolver
    from laplace_fmm_b200.workloads import gaussian_mix3d, uniform3d
    if not WEIGHTS.exists():
        pytest.skip("trained network not present")
    probs = [uniform3d(20000, seed=s) for s in range(3)]
    probs += [gaussian_mix3d(40000, seed=300 + s, kmin=1, kmax=1, smin=0.005, smax=0.006) for s in range(3)]
    probs += [gaussian_mix3d(30000, seed=310 + s) for s in range(4)]
    solver = LearnedSolver(ctx=ctx, leaf=True)
    out, info = solver.solve_batch(probs, tol=1e-6, tree_depth=10, max_leaf="auto", check_targets=64)
    assert info["max_leaf"] in LEAF_CANDIDATES
    assert info["order_groups"] >= 1
    for (pos, q), (pot, fld) in zip(probs, out):
        n = len(pos)
        idx = np.arange(64) * (n // 64)
        pe = compute_exact(InteractionType.Potential3d, (pos, q), pos[idx], ctx=ctx) - q[idx] * 1e4
        fe = compute_exact(InteractionType.Force3d, (pos, q), pos[idx], ctx=ctx)
        assert rel_l2(noself(pot[idx], q[idx]), pe) <= 1e-6
        assert rel_l2(fld[idx], fe) <= 1e-6
