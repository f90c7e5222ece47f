"""Train the order-selection network on (feature, measured error) pairs that
the FMM generates itself, on the GPU.

    python -m laplace_fmm_b200.train_order [--train 512] [--heldout 64]

Problems: 1-8 isotropic Gaussian clusters (sigma log-uniform in [0.005, 0.2],
centres uniform in the unit cube), N log-uniform in [1e4, 1e6], charges
uniform in [-1, 1]; plus larger ones (1e6-8e6 particles, Gaussian clusters or
a Plummer sphere in a uniform background) so that the network covers
millions of particles; adaptive octree (<= 10 levels, <= 64 per leaf).  Each
problem is labelled by solving it (mixed form) at p = 4, 6, ..., 14, 16 and
comparing with the FP64 direct sum at 1024 sampled targets: the labels of a
leaf at order p are log10 of the RMS absolute potential error and of the RMS
field error magnitude of its sampled targets, so that the leaves' labels,
weighted by their particle counts and divided by the RMS potential (self
term removed) or the RMS field, give the problem's rel-L2 of each output.
The solver gets those RMS values from the same sampled direct sum that
judges its result.  Leaves without a sampled target are masked out.

Threshold network (``--leaf``): the same architecture, output 0 = log10 of
the solve's device time; rows = (problem, order N in {12, 16}, leaf-size
threshold in {16, ..., 192}), inputs = the counts of the adaptive tree that
threshold gives (``lfmm3d_leaf_features``), labels = the timed mixed solve
(least of three after a warm-up); the solver builds the threshold of least
predicted time.

Training: Adam (lr 1e-3), batches of 4096 leaves, masked mean-squared error,
all in the library's CUDA kernels.  The held-out problems measure what the
network gains over the fixed order: the order it picks for tolerance 1e-6
(on both outputs), the error reached there, and the fastest fixed order
that meets the tolerance on every training problem.  Writes ``order_mlp.npz`` beside this
file (parameters with the input normalisation folded in, plus the
normalisation, the loss curve and the held-out summary).
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from ._lib import LfmmSolveOpts, default_context
from .order import (LEAF_CANDIDATES, N_ORD, N_OUT, N_PARAMS, ORDERS, WEIGHTS, LearnedSolver, OrderMLP, features,
                    leaf_features)
from .workloads import gaussian_mix3d, plummer_mix3d

DEPTH, MAX_LEAF, SAMPLES = 10, 64, 1024


def problem(i: int, kind: str):
    """Seeded problem i of a set: 'train' / 'heldout' (1-8 Gaussian clusters,
    N log-uniform in [1e4, 1e6]) or 'large' (N log-uniform in [1e6, 8e6]:
    Gaussian clusters, or a Plummer sphere of scale radius log-uniform in
    [0.02, 0.1] mixed 50/50 with a uniform background)."""
    base = {"train": 10_000, "heldout": 90_000, "large": 50_000, "xl": 70_000}[kind]
    g = np.random.default_rng(base + i)
    if kind == "xl":
        # 8e6-16.8e6 particles: a Plummer sphere in a uniform background
        n = int(round(10 ** g.uniform(np.log10(8e6), np.log10(16.8e6))))
        a = float(10 ** g.uniform(np.log10(0.03), np.log10(0.08)))
        return plummer_mix3d(n, seed=base + i, a=a)
    if kind != "large":
        n = int(round(10 ** g.uniform(4.0, 6.0)))
        return gaussian_mix3d(n, seed=base + i)
    n = int(round(10 ** g.uniform(6.0, np.log10(8e6))))
    if i % 2 == 0:
        return gaussian_mix3d(n, seed=base + i)
    a = float(10 ** g.uniform(np.log10(0.02), -1.0))
    return plummer_mix3d(n, seed=base + i, a=a)


def solve(ctx, pos, q, N):
    import ctypes
    pot = np.zeros(len(pos))
    fld = np.zeros((len(pos), 3))
    opts = LfmmSolveOpts(N, DEPTH, MAX_LEAF, 1, 1e-8)
    vp = ctypes.c_void_p
    ctx.check(ctx.lib.lfmm3d_solve_ex(ctx.handle, len(pos), pos.ctypes.data_as(vp), q.ctypes.data_as(vp), 0, None,
                                      ctypes.byref(opts), pot.ctypes.data_as(vp), fld.ctypes.data_as(vp), None),
              "solve")
    return pot, fld


def direct(ctx, pos, q, idx):
    import ctypes
    tgt = np.ascontiguousarray(pos[idx])
    pot = np.zeros(len(idx))
    fld = np.zeros((len(idx), 3))
    vp = ctypes.c_void_p
    ctx.check(ctx.lib.lfmm3d_direct(ctx.handle, len(pos), pos.ctypes.data_as(vp), q.ctypes.data_as(vp), len(idx),
                                    tgt.ctypes.data_as(vp), pot.ctypes.data_as(vp), fld.ctypes.data_as(vp)),
              "direct")
    return pot, fld


def label(ctx, pos, q, seed):
    """Features, per-leaf labels [leaves][14] (potential, then field), mask,
    and the sampled rel-L2 of the whole problem at each order: err[7] of the
    potential, errf[7] of the field; the RMS potential and RMS field."""
    feats, leaf_of = features(pos, q, tree_depth=DEPTH, max_leaf=MAX_LEAF, ctx=ctx)
    g = np.random.default_rng(seed)
    idx = np.sort(g.choice(len(pos), min(SAMPLES, len(pos)), replace=False))
    self_term = q[idx] * 1e4
    exact, exact_f = direct(ctx, pos, q, idx)
    exact = exact - self_term
    scale = np.sqrt(np.mean(exact ** 2))           # RMS potential: rel-L2 = RMS error / scale
    fscale = np.sqrt(np.mean(np.sum(exact_f ** 2, 1)))
    nl = len(feats)
    T = np.zeros((nl, N_OUT), np.float32)
    M = np.zeros((nl, N_OUT), np.float32)
    leaves = leaf_of[idx]
    counts = np.bincount(leaves, minlength=nl)
    has = counts > 0
    err, errf = np.zeros(N_ORD), np.zeros(N_ORD)
    for k, p in enumerate(ORDERS):
        pot, fld = solve(ctx, pos, q, p + 1)
        e = pot[idx] - self_term - exact                             # absolute errors
        ef2 = np.sum((fld[idx] - exact_f) ** 2, 1)
        err[k] = np.sqrt(np.mean(e ** 2)) / scale
        errf[k] = np.sqrt(np.mean(ef2)) / fscale
        ms = np.bincount(leaves, weights=e ** 2, minlength=nl)
        mf = np.bincount(leaves, weights=ef2, minlength=nl)
        T[has, k] = 0.5 * np.log10(ms[has] / counts[has] + 1e-30)
        T[has, N_ORD + k] = 0.5 * np.log10(mf[has] / counts[has] + 1e-30)
        M[has, k] = M[has, N_ORD + k] = 1.0
    return feats, T, M, err, errf, scale, fscale


LEAF_ORDERS = (12, 16)       # orders (degrees) the threshold labels are timed at


def time_solves(ctx, pos, q, N, thresholds, reps=3):
    """Device time (ms, CUDA events on the solver's stream, the least of reps
    after one warm-up) of the mixed solve at order N for each leaf-size
    threshold."""
    import ctypes
    import torch
    vp = ctypes.c_void_p
    n = len(pos)
    ds, dq = torch.from_numpy(pos).cuda(), torch.from_numpy(q).cuda()
    pot = torch.empty(n, dtype=torch.float64, device="cuda")
    fld = torch.empty(n, 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = []
    for m in thresholds:
        opts = LfmmSolveOpts(N, DEPTH, int(m), 1, 1e-8)
        best = 1e30
        for r in range(reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.check(ctx.lib.lfmm3d_solve_ex_device(ctx.handle, n, vp(ds.data_ptr()), vp(dq.data_ptr()), 0, None,
                                                     ctypes.byref(opts), vp(pot.data_ptr()), vp(fld.data_ptr()),
                                                     None), "solve")
            e1.record(stream)
            e1.synchronize()
            if r:
                best = min(best, e0.elapsed_time(e1))
        out.append(best)
    return np.array(out)


def label_leaf(ctx, pos, q):
    """Threshold-network rows of one problem: features [len(LEAF_ORDERS) * K][16]
    and the log10 solve time of each (order, threshold)."""
    X, T = [], []
    for N in LEAF_ORDERS:
        X.append(leaf_features(pos, q, N, tree_depth=DEPTH, ctx=ctx))
        T.append(np.log10(time_solves(ctx, pos, q, N, LEAF_CANDIDATES)))
    return np.concatenate(X), np.concatenate(T)


def train_leaf(a, ctx):
    """Label, train and evaluate the threshold network; stores it beside the
    order network in the weights file.  Returns the summary."""
    t0 = time.time()
    rows = {"train": [], "heldout": []}
    sets = (("train", a.leaf_train), ("large", a.large), ("xl", a.xl), ("heldout", a.leaf_heldout))
    for kind, count in sets:
        for i in range(count):
            pos, q = problem(i, kind)
            X, T = label_leaf(ctx, pos, q)
            rows["heldout" if kind == "heldout" else "train"].append((kind, i, len(pos), X, T))
    t_label = time.time() - t0
    X = np.concatenate([r[3] for r in rows["train"]])
    Tl = np.concatenate([r[4] for r in rows["train"]])
    T = np.zeros((len(X), N_OUT), np.float32)
    M = np.zeros((len(X), N_OUT), np.float32)
    T[:, 0] = Tl
    M[:, 0] = 1.0
    net = OrderMLP(seed=5, ctx=ctx, x_mean=X.mean(0), x_std=X.std(0) + 1e-6)
    Xn = net.normalise(X)
    g = np.random.default_rng(4)
    losses = []
    for ep in range(a.leaf_epochs):
        perm = g.permutation(len(Xn))
        tot = 0.0
        for b in range(0, len(perm), a.leaf_batch):
            j = perm[b:b + a.leaf_batch]
            tot += net.train_step(Xn[j], T[j], M[j], lr=a.lr) * len(j)
        losses.append(tot / len(perm))
    K = len(LEAF_CANDIDATES)

    def evaluate(rs):
        picked_ratio, at64_ratio, hits = [], [], 0
        for kind, i, n, Xr, Tr in rs:
            for j in range(len(LEAF_ORDERS)):
                y = net.forward(Xr[j * K:(j + 1) * K])[:, 0]
                t = 10.0 ** Tr[j * K:(j + 1) * K]
                k = int(np.argmin(y))
                picked_ratio.append(t[k] / t.min())
                at64_ratio.append(t[LEAF_CANDIDATES.index(64)] / t[k])
                hits += int(k == int(np.argmin(t)))
        return {"mean_time_over_best": float(np.mean(picked_ratio)),
                "worst_time_over_best": float(np.max(picked_ratio)),
                "mean_speedup_over_64": float(np.mean(at64_ratio)),
                "best_picked": hits, "cases": len(picked_ratio)}

    summary = {"leaf_train_problems": len(rows["train"]), "leaf_heldout_problems": len(rows["heldout"]),
               "rows": int(len(X)), "candidates": list(LEAF_CANDIDATES), "orders": list(LEAF_ORDERS),
               "loss_first": losses[0], "loss_last": losses[-1], "label_s": t_label,
               "train": evaluate(rows["train"]), "heldout": evaluate(rows["heldout"])}
    z = dict(np.load(a.out))
    z.update(leaf_params=net.params_host(), leaf_folded=net.folded_params(), leaf_x_mean=net.x_mean,
             leaf_x_std=net.x_std, leaf_losses=np.array(losses), leaf_summary=np.asarray(json.dumps(summary)))
    np.savez(a.out, **z)
    return summary


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=512)
    ap.add_argument("--heldout", type=int, default=64)
    ap.add_argument("--large", type=int, default=32, help="extra training problems of 1e6-8e6 particles")
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--quantile", type=float, default=0.7,
                    help="calibration: the quantile of the training problems' shortfall added to the outputs")
    ap.add_argument("--data", default=None, help="save the labelled problems here (npz)")
    ap.add_argument("--out", default=str(WEIGHTS))
    ap.add_argument("--leaf", action="store_true",
                    help="train only the leaf-size threshold network (the order network in --out is kept)")
    ap.add_argument("--leaf-train", type=int, default=256, help="training problems timed for the threshold labels")
    ap.add_argument("--leaf-heldout", type=int, default=32)
    ap.add_argument("--xl", type=int, default=4, help="problems of 8e6-16.8e6 particles in the threshold labels")
    ap.add_argument("--leaf-epochs", type=int, default=400)
    ap.add_argument("--leaf-batch", type=int, default=256)
    a = ap.parse_args(argv)
    ctx = default_context(0)
    if a.leaf:
        summary = train_leaf(a, ctx)
        print(json.dumps(summary))
        return 0
    t0 = time.time()
    data = {"train": [], "heldout": []}
    for kind, count in (("train", a.train), ("large", a.large), ("heldout", a.heldout)):
        for i in range(count):
            pos, q = problem(i, kind)
            data["heldout" if kind == "heldout" else "train"].append((len(pos),) + label(ctx, pos, q, seed=7 + i))
    t_label = time.time() - t0
    if a.data:
        blob = {}
        for kind in ("train", "heldout"):
            for i, (n, feats, T_, M_, err, errf, scale, fscale) in enumerate(data[kind]):
                blob.update({f"{kind}{i}_feats": feats, f"{kind}{i}_T": T_, f"{kind}{i}_M": M_,
                             f"{kind}{i}_err": err, f"{kind}{i}_errf": errf, f"{kind}{i}_scale": np.float64(scale),
                             f"{kind}{i}_fscale": np.float64(fscale), f"{kind}{i}_n": np.int64(n)})
        np.savez_compressed(a.data, **blob)
    X = np.concatenate([d[1] for d in data["train"]])
    T = np.concatenate([d[2] for d in data["train"]])
    M = np.concatenate([d[3] for d in data["train"]])
    keep = M.sum(1) > 0
    X, T, M = X[keep], T[keep], M[keep]
    mean, std = X.mean(0), X.std(0) + 1e-6
    net = OrderMLP(seed=1, ctx=ctx, x_mean=mean, x_std=std)
    Xn = net.normalise(X)
    g = np.random.default_rng(3)
    losses = []
    for ep in range(a.epochs):
        perm = g.permutation(len(Xn))
        tot = 0.0
        for b in range(0, len(perm), a.batch):
            j = perm[b:b + a.batch]
            tot += net.train_step(Xn[j], T[j], M[j], lr=a.lr) * len(j)
        losses.append(tot / len(perm))
    t_train = time.time() - t0 - t_label
    # calibration: the network's problem-level prediction against the measured
    # rel-L2 of every training problem near the tolerance, for the potential
    # and the field apart; a quantile of each output's shortfall is added to
    # its outputs (folded into their biases)
    res, resf = [], []
    for n, feats, T_t, M_t, err, errf, scale, fscale in data["train"]:
        pred = net.predicted_log10(feats)
        for k in range(N_ORD):
            if 1e-3 * a.tol <= err[k] <= 1e3 * a.tol:
                res.append(np.log10(err[k]) - (pred[k] - np.log10(scale)))
            if 1e-3 * a.tol <= errf[k] <= 1e3 * a.tol:
                resf.append(np.log10(errf[k]) - (pred[N_ORD + k] - np.log10(fscale)))
    delta = float(np.quantile(res, a.quantile)) if res else 0.0
    delta_f = float(np.quantile(resf, a.quantile)) if resf else 0.0
    net.shift_outputs(delta, delta_f)
    # held-out: the learned solve (with its sampled check and fallback) against
    # the fixed order that meets the tolerance (both outputs) on every training problem
    ok = lambda d, k: d[4][k] <= a.tol and d[5][k] <= a.tol
    fixed = next((p for k, p in enumerate(ORDERS) if all(ok(d, k) for d in data["train"])), ORDERS[-1])
    solver = LearnedSolver(net.folded_params(), ctx=ctx)
    picked, first_ok, final_ok, best, t_learned, t_fixed = [], 0, 0, [], 0.0, 0.0
    for i, (n, feats, T_h, M_h, err, errf, scale, fscale) in enumerate(data["heldout"]):
        pos, q = problem(i, "heldout")
        solve(ctx, pos, q, fixed + 1)                        # warm the operator caches
        s0 = time.perf_counter()
        r = solver.solve(pos, q, tol=a.tol, tree_depth=DEPTH, max_leaf=MAX_LEAF, check_targets=256)
        s1 = time.perf_counter()
        solve(ctx, pos, q, fixed + 1)
        s2 = time.perf_counter()
        t_learned += s1 - s0
        t_fixed += s2 - s1
        info = r["info"]
        picked.append(info["predicted_N"] - 1)
        first_ok += int(not info["fallback"])
        final_ok += int(max(info["checked_error"], info["checked_error_field"]) <= a.tol)
        best.append(next((pp for k, pp in enumerate(ORDERS) if err[k] <= a.tol and errf[k] <= a.tol), ORDERS[-1]))
    summary = {"train_problems": a.train, "large_problems": a.large, "heldout_problems": a.heldout,
               "leaves": int(len(X)),
               "loss_first": losses[0], "loss_last": losses[-1], "label_s": t_label, "train_s": t_train,
               "calibration_log10": delta, "calibration_log10_field": delta_f,
               "calibration_residuals": len(res) + len(resf),
               "fixed_p_all_train": fixed, "heldout_mean_p_picked": float(np.mean(picked)),
               "heldout_mean_p_best_even": float(np.mean(best)), "heldout_no_fallback": first_ok,
               "heldout_within_tol": final_ok, "heldout_s_learned": t_learned, "heldout_s_fixed": t_fixed}
    net.save(a.out, losses=np.array(losses), summary=json.dumps(summary))
    print(json.dumps(summary))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
