"""Order-selection MLP: the CUDA forward / backward / Adam kernels against the
FP64 numpy restatement in oracle/mlp.py (which is itself checked against
finite differences on the CPU)."""
import numpy as np
import pytest

from oracle import mlp as om


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, om.F)).astype(np.float32)
    T = rng.normal(size=(n, om.O)).astype(np.float32)
    M = (rng.random((n, om.O)) < 0.7).astype(np.float32)
    return X, T, M


def test_oracle_gradient_matches_finite_differences():
    X, T, M = _batch(37, 1)
    p = om.init(3).astype(np.float64)
    p[om.NPARAM - om.O:] = 0.1
    _, g = om.loss_and_grad(p, X, T, M)
    rng = np.random.default_rng(2)
    for i in rng.choice(om.NPARAM, 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (om.loss_and_grad(pp, X, T, M)[0] - om.loss_and_grad(pm, X, T, M)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i])


def test_parameter_count_matches_header():
    from laplace_fmm_b200.order import N_PARAMS
    import re
    from pathlib import Path
    text = (Path(__file__).resolve().parent.parent / "include" / "lfmm.h").read_text()
    expr = re.search(r"#define LFMM_MLP_PARAMS \((.*)\)", text).group(1)
    assert eval(expr) == N_PARAMS == om.NPARAM


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 31, 33, 1000])
def test_forward_matches_oracle(ctx, n):
    from laplace_fmm_b200.order import OrderMLP
    X, _, _ = _batch(n, n)
    p = om.init(n)
    p[-om.O:] = 0.3
    net = OrderMLP(p, ctx=ctx)
    Y = net.forward(X, normalised=True)
    ref = om.forward(p, X)
    assert np.abs(Y - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("n", [5, 64, 4096])
def test_gradient_matches_oracle(ctx, n):
    from laplace_fmm_b200.order import OrderMLP
    X, T, M = _batch(n, 10 + n)
    p = om.init(n + 1)
    net = OrderMLP(p, ctx=ctx)
    loss = net.loss_grad(X, T, M)
    rl, rg = om.loss_and_grad(p, X, T, M)
    g = net.grad.cpu().numpy()
    assert abs(loss - rl) <= 1e-5 * abs(rl)
    assert np.linalg.norm(g - rg) <= 1e-4 * np.linalg.norm(rg)


@pytest.mark.gpu
def test_adam_matches_oracle(ctx):
    from laplace_fmm_b200.order import OrderMLP
    X, T, M = _batch(300, 7)
    p = om.init(5)
    net = OrderMLP(p, ctx=ctx)
    rp, rm, rv = p.astype(np.float64), np.zeros(om.NPARAM), np.zeros(om.NPARAM)
    for step in range(1, 4):
        net.train_step(X, T, M, lr=1e-2)
        _, g = om.loss_and_grad(rp, X, T, M)
        rp, rm, rv = om.adam(rp, g, rm, rv, step, lr=1e-2)
    assert np.abs(net.params_host() - rp).max() <= 2e-5


@pytest.mark.gpu
def test_training_reduces_loss(ctx):
    """A learnable map (a fixed random MLP's outputs) is fitted by the kernels."""
    from laplace_fmm_b200.order import OrderMLP
    rng = np.random.default_rng(0)
    X = rng.normal(size=(4096, om.F)).astype(np.float32)
    T = om.forward(om.init(99), X).astype(np.float32)
    M = np.ones_like(T)
    net = OrderMLP(seed=1, ctx=ctx)
    first = net.loss_grad(X, T, M)
    for _ in range(200):
        last = net.train_step(X, T, M, lr=3e-3)
    assert last < 0.1 * first
