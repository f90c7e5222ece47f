"""Learned order selection: host side of the MLP kernels in ``csrc/mlp.cu``.

The network maps 16 features of a leaf box to log10 of that box's RMS
absolute potential error (outputs 0-6) and field error (outputs 7-13) at the
orders p = 4, 6, 8, 10, 12, 14, 16 (``ORDERS``).  Training, inference and
the optimiser all run in the library's CUDA kernels (``lfmm_mlp_forward``,
``lfmm_mlp_grad``, ``lfmm_mlp_adam``); torch only holds the device buffers.
The reference has no counterpart: it derives one order from eps by a fixed
formula (cpu/multipole3d.cpp:1328-1331), which stays the fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from ._lib import PRECISION, Context, LfmmError, LfmmLearnedInfo, LfmmSolveOpts, LfmmStats, default_context

N_IN, N_HIDDEN, N_OUT = 16, 64, 14
N_PARAMS = N_HIDDEN * N_IN + N_HIDDEN + N_HIDDEN * N_HIDDEN + N_HIDDEN + N_OUT * N_HIDDEN + N_OUT
ORDERS = (4, 6, 8, 10, 12, 14, 16)       # expansion order p of each output pair (N = p + 1 degrees)
N_ORD = len(ORDERS)
WEIGHTS = Path(__file__).resolve().parent / "order_mlp.npz"


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise LfmmError("the order MLP runs on the GPU; no CUDA device is visible")
    return torch


def he_init(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases, packed in the kernels' layout."""
    rng = np.random.default_rng(seed)
    parts = []
    for rows, cols in ((N_HIDDEN, N_IN), (N_HIDDEN, N_HIDDEN), (N_OUT, N_HIDDEN)):
        bound = np.sqrt(6.0 / cols)
        parts += [rng.uniform(-bound, bound, size=rows * cols), np.zeros(rows)]
    return np.concatenate(parts).astype(np.float32)


class OrderMLP:
    """Parameters on the device plus the Adam state; every op is a CUDA kernel."""

    def __init__(self, params: np.ndarray | None = None, ctx: Context | None = None, seed: int = 0,
                 x_mean: np.ndarray | None = None, x_std: np.ndarray | None = None):
        torch = _torch()
        self.ctx = ctx or default_context(0)
        dev = torch.device("cuda", self.ctx.device)
        p = he_init(seed) if params is None else np.ascontiguousarray(params, dtype=np.float32)
        if p.shape != (N_PARAMS,):
            raise ValueError(f"expected {N_PARAMS} parameters, got {p.shape}")
        self.params = torch.from_numpy(p.copy()).to(dev)
        self.grad = torch.zeros(N_PARAMS, dtype=torch.float32, device=dev)
        self.m = torch.zeros_like(self.grad)
        self.v = torch.zeros_like(self.grad)
        self.step_count = 0
        self.x_mean = np.zeros(N_IN, np.float32) if x_mean is None else np.asarray(x_mean, np.float32)
        self.x_std = np.ones(N_IN, np.float32) if x_std is None else np.asarray(x_std, np.float32)
        self._dev = dev

    # -- device helpers ----------------------------------------------------
    def _to_dev(self, a: np.ndarray):
        torch = _torch()
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(self._dev)

    def _sync_lib(self):
        """Wait for the library's stream (torch work is ordered before each
        call by a device synchronise)."""
        torch = _torch()
        s = torch.cuda.ExternalStream(self.ctx.stream, device=self._dev)
        s.synchronize()

    def normalise(self, X: np.ndarray) -> np.ndarray:
        return ((np.asarray(X, np.float32) - self.x_mean) / self.x_std).astype(np.float32)

    # -- network ops -------------------------------------------------------
    def forward(self, X: np.ndarray, normalised: bool = False) -> np.ndarray:
        """log10 error predictions [n][14] for feature rows X [n][16]."""
        torch = _torch()
        Xn = np.asarray(X, np.float32) if normalised else self.normalise(X)
        n = len(Xn)
        if n == 0:
            return np.zeros((0, N_OUT), np.float32)
        dX = self._to_dev(Xn)
        dY = torch.empty((n, N_OUT), dtype=torch.float32, device=self._dev)
        torch.cuda.synchronize(self._dev)
        self.ctx.check(self.ctx.lib.lfmm_mlp_forward(self.ctx.handle, self.params.data_ptr(), n, dX.data_ptr(),
                                                     dY.data_ptr()), "lfmm_mlp_forward")
        self._sync_lib()
        return dY.cpu().numpy()

    def loss_grad(self, X, T, M, normalised: bool = True):
        """Masked MSE loss and its gradient (left in ``self.grad``)."""
        torch = _torch()
        Xn = np.asarray(X, np.float32) if normalised else self.normalise(X)
        n = len(Xn)
        dX, dT, dM = self._to_dev(Xn), self._to_dev(T), self._to_dev(M)
        work = torch.empty(n * (N_OUT + 2 * N_HIDDEN) + 2, dtype=torch.float32, device=self._dev)
        loss = ctypes.c_float()
        torch.cuda.synchronize(self._dev)
        self.ctx.check(self.ctx.lib.lfmm_mlp_grad(self.ctx.handle, self.params.data_ptr(), n, dX.data_ptr(),
                                                  dT.data_ptr(), dM.data_ptr(), self.grad.data_ptr(),
                                                  work.data_ptr(), ctypes.byref(loss)), "lfmm_mlp_grad")
        self._sync_lib()
        return float(loss.value)

    def adam_step(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        self.step_count += 1
        torch = _torch()
        torch.cuda.synchronize(self._dev)
        self.ctx.check(self.ctx.lib.lfmm_mlp_adam(self.ctx.handle, self.params.data_ptr(), self.grad.data_ptr(),
                                                  self.m.data_ptr(), self.v.data_ptr(), self.step_count, lr, beta1,
                                                  beta2, eps), "lfmm_mlp_adam")
        self._sync_lib()

    def train_step(self, X, T, M, lr: float = 1e-3) -> float:
        loss = self.loss_grad(X, T, M)
        self.adam_step(lr)
        return loss

    def params_host(self) -> np.ndarray:
        return self.params.cpu().numpy()

    def shift_outputs(self, delta: float, delta_field: float | None = None):
        """Add the calibration offsets to the outputs (log10 errors): delta to
        the potential's, delta_field (default: delta) to the field's."""
        b = N_PARAMS - N_OUT
        self.params[b:b + N_ORD] += float(delta)
        self.params[b + N_ORD:] += float(delta if delta_field is None else delta_field)

    def predicted_log10(self, feats: np.ndarray) -> np.ndarray:
        """log10 of the problem-level RMS absolute error at each output (the
        potential's at the seven orders, then the field's), from its leaves'
        features (leaves weighted by their particles), as the solver aggregates
        them; minus log10 of the RMS potential / field it is the rel-L2."""
        Y = self.forward(feats).astype(np.float64)
        w = 10.0 ** feats[:, 0].astype(np.float64) - 1.0
        return 0.5 * np.log10((w[:, None] * 10.0 ** (2.0 * Y)).sum(0) / max(w.sum(), 1.0))

    def folded_params(self) -> np.ndarray:
        """Parameters with the input normalisation folded into the first layer
        (W1' = W1 / std, b1' = b1 - W1' mean): the network on raw features, as
        the solver runs it."""
        p = self.params_host().astype(np.float64)
        nw1 = N_HIDDEN * N_IN
        W1 = p[:nw1].reshape(N_HIDDEN, N_IN)
        b1 = p[nw1:nw1 + N_HIDDEN]
        W1f = W1 / self.x_std.astype(np.float64)
        b1f = b1 - W1f @ self.x_mean.astype(np.float64)
        out = p.copy()
        out[:nw1] = W1f.ravel()
        out[nw1:nw1 + N_HIDDEN] = b1f
        return out.astype(np.float32)

    def device_params(self, folded: bool = True):
        """A device tensor holding the parameters the solver takes."""
        torch = _torch()
        if not folded:
            return self.params
        return torch.from_numpy(self.folded_params()).to(self._dev)

    # -- persistence ---------------------------------------------------------
    def save(self, path: Path | str = WEIGHTS, **meta):
        np.savez(path, params=self.params_host(), folded=self.folded_params(), x_mean=self.x_mean,
                 x_std=self.x_std, **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path: Path | str = WEIGHTS, ctx: Context | None = None) -> "OrderMLP":
        z = np.load(path)
        return cls(z["params"], ctx=ctx, x_mean=z["x_mean"], x_std=z["x_std"])


def _f64(a, cols):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, cols)) if cols else \
        np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def features(src, q, targets=None, tree_depth: int = 10, max_leaf: int = 64, ctx: Context | None = None):
    """Per-leaf features [n_leaves][16] of the adaptive tree and the leaf of
    every input particle (targets first, then sources)."""
    ctx = ctx or default_context(0)
    src, q = _f64(src, 3), _f64(q, 0)
    tgt = None if targets is None else _f64(targets, 3)
    nt = 0 if tgt is None else len(tgt)
    opts = LfmmSolveOpts(0, tree_depth, max_leaf, 1, 1e-8)
    cap = (len(src) + nt) + 1
    feats = np.zeros((cap, N_IN), np.float32)
    leaf_of = np.zeros(len(src) + nt, np.int32)
    nl = ctypes.c_size_t()
    ctx.check(ctx.lib.lfmm3d_features(ctx.handle, len(src), _p(src), _p(q), nt, _p(tgt), ctypes.byref(opts),
                                      _p(feats), cap, _p(leaf_of), ctypes.byref(nl)), "lfmm3d_features")
    return feats[:nl.value].copy(), leaf_of


def load_params(path: Path | str = WEIGHTS, leaf: bool = False) -> np.ndarray:
    """The trained order network (input normalisation folded in) shipped with
    the package; leaf=True appends the leaf-size threshold network, the
    buffer the solver takes when the threshold is learned too (max_leaf
    LFMM_AUTO)."""
    z = np.load(path)
    p = z["folded"].astype(np.float32)
    if leaf:
        if "leaf_folded" not in z:
            raise LfmmError(f"{path} holds no threshold network (train it: python -m laplace_fmm_b200.train_order --leaf)")
        p = np.concatenate([p, z["leaf_folded"].astype(np.float32)])
    return p


# the leaf-size thresholds the threshold network chooses among (the solver's list)
LEAF_CANDIDATES = (16, 24, 32, 48, 64, 96, 128, 192)


def leaf_features(src, q, N: int, tree_depth: int = 10, candidates=LEAF_CANDIDATES, ctx: Context | None = None):
    """The threshold network's inputs [K][16]: per candidate threshold, the
    counts of the adaptive tree it would give, at order N."""
    ctx = ctx or default_context(0)
    src, q = _f64(src, 3), _f64(q, 0)
    cand = (ctypes.c_int * len(candidates))(*candidates)
    feats = np.zeros((len(candidates), N_IN), np.float32)
    ctx.check(ctx.lib.lfmm3d_leaf_features(ctx.handle, len(src), _p(src), _p(q), 0, None, int(tree_depth), int(N),
                                           cand, len(candidates), _p(feats)), "lfmm3d_leaf_features")
    return feats


class LearnedSolver:
    """3D solve at the order the network picks for a tolerance, with the
    fixed-order fallback judged by a sampled FP64 direct-sum check."""

    def __init__(self, params: np.ndarray | None = None, ctx: Context | None = None, leaf: bool = False):
        """leaf=True: the threshold network too (solve with max_leaf="auto")."""
        torch = _torch()
        self.ctx = ctx or default_context(0)
        p = load_params(leaf=leaf) if params is None else np.ascontiguousarray(params, dtype=np.float32)
        self.leaf = len(p) == 2 * N_PARAMS
        self.d_params = torch.from_numpy(p).to(torch.device("cuda", self.ctx.device))

    def _leaf(self, max_leaf):
        if max_leaf == "auto":
            if not self.leaf:
                raise LfmmError("max_leaf='auto' needs the threshold network (LearnedSolver(leaf=True))")
            return 2147483647
        return int(max_leaf)

    def solve(self, src, q, targets=None, tol: float = 1e-6, tree_depth: int = 10, max_leaf: int = 64,
              precision: str = "mixed", check_targets: int = 256, stats: bool = False):
        src, q = _f64(src, 3), _f64(q, 0)
        tgt = None if targets is None else _f64(targets, 3)
        nt = 0 if tgt is None else len(tgt)
        nout = nt if nt else len(src)
        pot = np.zeros(nout)
        fld = np.zeros((nout, 3))
        opts = LfmmSolveOpts(0, tree_depth, self._leaf(max_leaf), PRECISION[precision], tol)
        info = LfmmLearnedInfo()
        st = LfmmStats()
        _torch().cuda.synchronize(self.d_params.device)
        self.ctx.check(self.ctx.lib.lfmm3d_solve_learned(
            self.ctx.handle, len(src), _p(src), _p(q), nt, _p(tgt), ctypes.byref(opts),
            ctypes.c_void_p(self.d_params.data_ptr()), tol, check_targets, _p(pot), _p(fld), ctypes.byref(info),
            ctypes.byref(st) if stats else None), "lfmm3d_solve_learned")
        out = {"potentials": pot, "forces": fld, "info": info.as_dict()}
        if stats:
            out["stats"] = st.as_dict()
        return out

    def solve_batch(self, problems, tol: float = 1e-6, tree_depth: int = 10, max_leaf: int = 64,
                    precision: str = "mixed", check_targets: int = 64):
        """Independent problems [(positions, charges), ...] as one batch at the
        order the network picks (the highest any problem needs), each problem
        judged on its own samples.  Returns ([(pot, forces), ...], info)."""
        torch = _torch()
        dev = self.d_params.device
        parts = [(_f64(p, 3), _f64(c, 0)) for p, c in problems]
        offs = np.zeros(len(parts) + 1, dtype=np.uint64)
        offs[1:] = np.cumsum([len(p) for p, _ in parts])
        d_pos = torch.from_numpy(np.concatenate([p for p, _ in parts])).to(dev)
        d_q = torch.from_numpy(np.concatenate([c for _, c in parts])).to(dev)
        n = int(offs[-1])
        d_pot = torch.empty(n, dtype=torch.float64, device=dev)
        d_fld = torch.empty(n, 3, dtype=torch.float64, device=dev)
        opts = LfmmSolveOpts(0, tree_depth, self._leaf(max_leaf), PRECISION[precision], tol)
        info = LfmmLearnedInfo()
        vp = ctypes.c_void_p
        torch.cuda.synchronize(dev)
        self.ctx.check(self.ctx.lib.lfmm3d_solve_batch_learned_device(
            self.ctx.handle, len(parts), offs.ctypes.data_as(vp), vp(d_pos.data_ptr()), vp(d_q.data_ptr()),
            ctypes.byref(opts), vp(self.d_params.data_ptr()), tol, check_targets, vp(d_pot.data_ptr()),
            vp(d_fld.data_ptr()), ctypes.byref(info), None), "lfmm3d_solve_batch_learned_device")
        torch.cuda.ExternalStream(self.ctx.stream, device=dev).synchronize()
        pot, fld = d_pot.cpu().numpy(), d_fld.cpu().numpy()
        return [(pot[offs[k]:offs[k + 1]], fld[offs[k]:offs[k + 1]]) for k in range(len(parts))], info.as_dict()
