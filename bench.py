"""Benchmark: Mparticles/s of one FMM solve on one B200, with its accuracy.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c1|c2|c3|c5|c6]
                    [--impl ours|reference|reference-gpu]

A step is one full solve (tree build through outputs in input order) of the
configuration's seeded synthetic particle set.  ``value`` times solves on
device-resident inputs (CUDA events on the solver's stream, K solves after W
warm-up solves, barrier + synchronise around the timed region, max over
ranks); ``e2e`` times the same solve through the public host-buffer entry
point (pinned host inputs copied in and results copied out every step).
Every solve rebuilds the tree and re-reads every particle; the working set
exceeds L2 (126 MB) for the 16M-particle configuration, and for the smaller
ones an L2 flush (a 256 MB write) runs between timed steps.

Multi-GPU: the solver does not shard one problem (no collective); with
``--gpus N`` every rank solves its own independent copy of the
configuration (weak scaling, replicas), rank 0 prints the line.

``--impl reference`` times the reference's own CPU FMM (compiled from its
sources into oracle/_ref) on the host cores, on a bounded sample of the same
configuration; only rank 0 runs it.  ``--impl reference-gpu`` times the
reference's own CUDA FMM (its unmodified sources built for sm_100a into
oracle/_ref/libfmmref_gpu.so) on the same particles, with its uniform tree
(the configuration's depth; ``--depth`` for the adaptive configurations), and
states its accuracy against the FP64 direct sum.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    # 3D uniform, 131,072 particles, FP64, p = 8 (N = 9), uniform depth 5 (max 64 per leaf)
    "c1": dict(dim=3, n=131072, gen="uniform3d", seed=12345, N=9, depth=5, precision="fp64",
               metric="3D FMM Mparticles/s, plain FP64 form at p=8",
               workload="3D uniform 131,072 particles, FP64, p=8 (N=9), uniform octree depth 5"),
    # 2D clustered, 4,194,304 particles, p = 20 (N = 21), FP64, adaptive
    # quadtree (<= 12 levels, <= 32 per leaf); the reference's uniform
    # quadtree (depth 11) timed beside it
    "c2": dict(dim=2, n=4194304, gen="clustered2d", seed=4242, N=21, depth=12, max_leaf=32, uniform_depth=11,
               precision="fp64", metric="2D FMM Mparticles/s, FP64 at p=20",
               workload="2D half uniform / half 64 Gaussian clusters (sigma 0.005) 4,194,304 particles, FP64, "
                        "p=20 (N=21), adaptive quadtree (<=12 levels, <=32 per leaf)"),
    # 3D clustered, 16,777,216 particles (Plummer a = 0.05 + uniform), adaptive octree
    # mixed form at the order the network picks for rel-L2 <= 1e-6 on potential
    # and field (sampled check of 256 outputs judged on its upper confidence
    # bound, fixed-order fallback); the plain FP64 form beside it at p = 15
    # (N = 16), the lowest fixed order at which both outputs reach 1e-6 here
    # (N = 15: field 1.007e-6)
    "c3": dict(dim=3, n=16777216, gen="plummer_mix3d", seed=2024, N=16, depth=10, max_leaf=64, precision="mixed",
               learned=True, learned_leaf=True, tol=1e-6, check_targets=256,
               workload="3D Plummer (a=0.05) + uniform 16,777,216 particles, adaptive octree (<=10 levels), mixed "
                        "precision at the learned order and learned leaf size for rel-L2 <= 1e-6 on potential and "
                        "field; beside it the plain FP64 form and the mixed form at p=15 (N=16), <=64 per leaf"),
    # 1024 independent problems, N log-uniform in [2048, 262144] (about 60M particles),
    # each uniform in its own unit cube or one Gaussian cluster (sigma 0.05), solved
    # as one batch (mixed, N = 14); the plain FP64 form (p = 10, N = 11) one problem
    # at a time beside it
    "c5": dict(dim=3, batch=True, count=1024, seed=5150, N=14, plain_N=11, depth=10, max_leaf=64,
               precision="mixed", n=0, learned=True, learned_leaf=True, tol=1e-6, check_targets=128,
               workload="batched 3D: 1024 problems, N log-uniform in [2048, 262144], uniform or one Gaussian "
                        "cluster (sigma 0.05) each, mixed precision at the learned order and leaf size for rel-L2 "
                        "<= 1e-6 (128 checked outputs per problem), adaptive octrees (<=10 levels); "
                        "plain FP64 p=10 one problem at a time beside it"),
    # learned order on the 64 held-out problems of the order network (1-8
    # Gaussian clusters, N log-uniform in [1e4, 1e6]) at tol 1e-6 on potential
    # and field, against the lowest single fixed order that meets tol on all 64
    "c4": dict(dim=3, heldout=True, count=64, n=0, N=17, depth=10, max_leaf=64, precision="mixed", learned=True,
               learned_leaf=True, tol=1e-6, check_targets=1024,
               metric="3D FMM Mparticles/s at rel-L2<=1e-6 vs FP64 direct: learned order vs best fixed order",
               workload="learned order, 3D: the 64 held-out problems (1-8 Gaussian clusters, sigma log-uniform in "
                        "[0.005, 0.2], N log-uniform in [1e4, 1e6]), mixed precision, adaptive octrees (<=10 levels), "
                        "learned order and leaf size, tol 1e-6 on potential and field (1024 checked outputs); the "
                        "lowest fixed order meeting tol on all 64 at <=64 per leaf beside it"),
    # vector charges (the reference's FastMultipole3d<Vector3d>): 4,194,304 particles of the
    # clustered mixture, charges U(-1, 1)^3, mixed precision, N = 12, adaptive octree;
    # the FP64 form beside it
    "c6": dict(dim=3, vector=True, n=4194304, gen="plummer_mix3d", seed=606, N=12, depth=10, max_leaf=64,
               precision="mixed", metric="3D vector-charge FMM Mparticles/s (field q x r / r^3)",
               workload="3D vector charges: Plummer (a=0.05) + uniform 4,194,304 particles, charges U(-1,1)^3, "
                        "adaptive octree (<=10 levels, <=64 per leaf), mixed precision, p=11 (N=12)"),
}
DEFAULT_CONFIG = "c3"
METRIC = "3D FMM Mparticles/s at rel-L2<=1e-6 vs FP64 direct: mixed+learned-p vs plain"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default=DEFAULT_CONFIG, choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-series", action="store_true",
                    help="with --impl reference: the reference CPU FMM on 1/64, 1/16 and 1/4 of the set (one solve "
                         "each, uniform depth three levels below its own automatic depth)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP64 form beside the mixed one")
    ap.add_argument("--no-learned", action="store_true", help="mixed form at the fixed order N instead of the learned one")
    ap.add_argument("--no-plan", action="store_true", help="skip timing repeated solves through a solve plan")
    ap.add_argument("--max-leaf", type=int, default=None, help="override the adaptive split threshold (0: uniform)")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default=None, help="override the configuration's")
    ap.add_argument("--order", type=int, default=None, help="override N (degrees)")
    ap.add_argument("--depth", type=int, default=None, help="override the tree depth")
    ap.add_argument("--particles", type=int, default=None,
                    help="override the particle count (small cases for profiling; not a bench line)")
    a = ap.parse_args()
    cfg = dict(CONFIGS[a.config])
    if a.precision:
        cfg["precision"] = a.precision
    overridden = []
    if a.precision:
        overridden.append(f"precision {a.precision}")
    if a.order:
        cfg["N"] = a.order
        overridden.append(f"N {a.order}")
    if a.depth:
        cfg["depth"] = a.depth
        overridden.append(f"tree depth {a.depth}")
    if a.max_leaf is not None:
        overridden.append(f"max leaf {a.max_leaf}")
    if overridden:
        cfg["workload"] += " [overridden: " + ", ".join(overridden) + "]"
    if a.particles:
        cfg["n"] = a.particles
        cfg["workload"] += f" [particle count overridden: {a.particles:,}]"
    if a.max_leaf is not None:
        cfg["max_leaf"] = a.max_leaf
    a.cfg = cfg
    return a


def max_over_ranks(value: float, dist, device="cuda") -> float:
    """The largest value over the ranks (device time of the slowest rank);
    the value itself on one process."""
    if not dist:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: int, world: int, ms: float) -> float:
    """Whole-job throughput in millions of units per second: every rank
    processes its own copy of the workload (replicas, weak scaling)."""
    return world * units_per_rank / (ms * 1e-3) / 1e6


def make_particles(cfg):
    from laplace_fmm_b200 import workloads as W
    return getattr(W, cfg["gen"])(cfg["n"], seed=cfg["seed"])


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0])); mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- peaks
def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "bf16_tflops": d.get("bf16_tflops", 1590.0),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def fp64_peak_tflops(torch):
    """Dense FP64 throughput measured here (cuBLAS DGEMM 8192^3, best of 5):
    the denominator for the FP64 kernels, which MEASURED_PEAKS.json lacks."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    torch.matmul(a, b); torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(); torch.matmul(a, b); e.record(); e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def fp32_peak_tflops(torch):
    """Dense FP32 (SIMT, TF32 off) throughput measured here: cuBLAS SGEMM 8192^3."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(8192, 8192, dtype=torch.float32, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float32, device="cuda")
    torch.matmul(a, b); torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(); torch.matmul(a, b); e.record(); e.synchronize()
        best = min(best, s.elapsed_time(e))
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def tf32_peak_tflops(torch):
    """Dense TF32 tensor-core throughput measured here: cuBLAS FP32 GEMM 8192^3
    with TF32 allowed (the denominator for the tcgen05 M2L kernel)."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(8192, 8192, dtype=torch.float32, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float32, device="cuda")
    torch.matmul(a, b); torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(); torch.matmul(a, b); e.record(); e.synchronize()
        best = min(best, s.elapsed_time(e))
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def launches_per_solve(depth, dim, radix_passes, adaptive, precision, learned=False, parts=False):
    """Kernels the library enqueues for one solve (tree + FMM passes), counted
    from the launch sites; the learned solve adds its features (far strength
    per level, accumulation per level, leaf features), the network, the
    prediction sums, the sampled direct sum (split kernel and reduction) and
    the RMS and error sums.  An ncu launch list of the 16.8M-particle learned
    solve shows 277 launches per solve: these 276 and the statistics pass of
    a timing context."""
    extra = (1 + (depth - 2) + (depth - 1) + 1 + 1 + 1 + 2 + 1 + 1) if learned else 0
    scan = 3
    tree = 2 + 1 + radix_passes * (1 + scan + 1) + 1 + 1 + scan + 1 + 1
    tree += (depth - 1) * (1 + scan + 1 + 1) + depth + 1
    lists = depth - 1
    if adaptive or precision != "fp64":
        tree += depth + depth * (1 + scan) + depth + 1 + scan + 1 + 1 + lists + 2 + 2 + 3 * scan
        # plan (class count, scatter, slot table) + GEMM per level; split
        # reductions and FP64 converts on the coarse levels 2-3
        m2l = max(0, depth - 2) * (3 + 1) + 2 + 2 * 2
        m2m = (depth - 1) * (2 if precision == "mixed" else 1)  # mixed: plan + tensor-core GEMM per level
        leaves = 2 if precision == "mixed" else 1               # FP32: near field, then the expansions
        fmm = 1 + 1 + m2m + m2l + 1 + max(0, depth - 3) + leaves
        return (tree, fmm) if parts else tree + fmm + extra
    if adaptive and dim == 2:
        tree += depth + depth * (1 + scan) + depth + 1 + scan + 1 + 1 + lists + 2 + 2 + 3 * scan
        # P2M, M2M per level, per M2L level: class count, scatter, slot table,
        # Hankel M2L (+ a split reduction on the small levels); P2L, L2L adds,
        # leaf work units (count + scan) and the leaves
        levels = max(0, depth - 2)
        split = sum(1 for L in range(2, depth) if 4 ** L < 37000)
        fmm = 1 + (depth - 1) + 4 * levels + split + 1 + max(0, depth - 3) + 1 + scan + 1
        return (tree, fmm) if parts else tree + fmm
    tree += lists
    if dim == 3:
        fmm = 1 + (depth - 1) + max(0, depth - 2) * 5 + max(0, depth - 3) + 1
    else:
        # per level 2..depth-1: class count, scatter, slot table, Hankel M2L,
        # and a split reduction on the levels too small to fill the GPU
        # (fewer than ~37k cells: levels up to 7); L2L adds; leaf work units
        # (count + scan) and the leaves
        levels = max(0, depth - 2)
        split = sum(1 for L in range(2, depth) if 4 ** L < 37000)
        fmm = 1 + (depth - 1) + 4 * levels + split + max(0, depth - 3) + 1 + scan + 1
    return tree + fmm


# ---------------------------------------------------------------- ours
def run_ours(args, cfg, rank, world, local_rank):
    import torch
    from laplace_fmm_b200 import Context
    from laplace_fmm_b200._lib import PRECISION, LfmmLearnedInfo, LfmmSolveOpts, LfmmStats
    from laplace_fmm_b200.workloads import rel_l2, sample_targets
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local_rank),
                                timeout=__import__("datetime").timedelta(seconds=300))
    dim, n, N, depth = cfg["dim"], cfg["n"], cfg["N"], cfg["depth"]
    max_leaf = cfg.get("max_leaf", 0)
    prec = PRECISION[cfg["precision"]]
    pos, q = make_particles(cfg)
    ctx = Context(local_rank)
    L = ctx.lib
    d_src = torch.from_numpy(pos).cuda()
    d_q = torch.from_numpy(q).cuda()
    d_pot = torch.empty(n, dtype=torch.float64, device="cuda")
    d_fld = torch.empty(n, dim, dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    vp = ctypes.c_void_p
    learned = bool(cfg.get("learned")) and not args.no_learned
    d_params = None
    info_box = {}
    learned_leaf = learned and bool(cfg.get("learned_leaf")) and args.max_leaf is None
    if learned:
        from laplace_fmm_b200.order import load_params
        d_params = torch.from_numpy(load_params(leaf=learned_leaf)).cuda()

    def call(c, device, precision, stats=None, host=None, tree=None):
        """One solve through the C ABI (device buffers, or pinned host buffers);
        the configuration's precision runs the learned solve when it has one.
        tree = (depth, max_leaf) overrides the configuration's tree."""
        depth_, max_leaf_ = tree if tree else (depth, max_leaf)
        src, qq, pot, fld = host if host else (d_src, d_q, d_pot, d_fld)
        sp = ctypes.byref(stats) if stats is not None else None
        if dim == 3 and learned and precision == prec and tree is None:
            opts = LfmmSolveOpts(N, depth, 2147483647 if learned_leaf else max_leaf, precision, cfg["tol"])
            info = LfmmLearnedInfo()
            fn = L.lfmm3d_solve_learned_device if device else L.lfmm3d_solve_learned
            st = fn(c.handle, n, vp(src.data_ptr()), vp(qq.data_ptr()), 0, None, ctypes.byref(opts),
                    vp(d_params.data_ptr()), cfg["tol"], cfg["check_targets"], vp(pot.data_ptr()),
                    vp(fld.data_ptr()), ctypes.byref(info), sp)
            info_box.update(info.as_dict())
        elif dim == 3 or max_leaf_ > 0:
            opts = LfmmSolveOpts(N, depth_, max_leaf_, precision, 1e-8)
            if dim == 3:
                fn = L.lfmm3d_solve_ex_device if device else L.lfmm3d_solve_ex
            else:
                fn = L.lfmm2d_solve_ex_device if device else L.lfmm2d_solve_ex
            st = fn(c.handle, n, vp(src.data_ptr()), vp(qq.data_ptr()), 0, None, ctypes.byref(opts),
                    vp(pot.data_ptr()), vp(fld.data_ptr()), sp)
        else:
            fn = L.lfmm2d_solve_device if device else L.lfmm2d_solve
            st = fn(c.handle, n, vp(src.data_ptr()), vp(qq.data_ptr()), 0, None, N, depth_, 1e-8, precision,
                    vp(pot.data_ptr()), vp(fld.data_ptr()), sp)
        c.check(st, "solve")

    def step_dev():
        call(ctx, True, prec)

    torch.cuda.synchronize()
    for _ in range(args.warmup):
        step_dev()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                starts[k].record(stream)
            step_dev()
            ends[k].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / args.steps, dist)
    # per-phase split (separate timed solve with phase events)
    ctx_t = Context(local_rank, timing=True)
    st = LfmmStats()
    call(ctx_t, True, prec)                       # warm the operator cache of this context
    call(ctx_t, True, prec, stats=st)
    torch.cuda.synchronize()
    stats = st.as_dict()
    # the plain FP64 form of the same configuration (the comparison the metric names)
    plain = None
    if dim == 3 and prec != 0 and not args.no_plain:
        for _ in range(2):
            call(ctx_t, True, 0)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(1, min(args.steps, 3))
        with torch.cuda.stream(torch.cuda.ExternalStream(ctx_t.stream)):
            t0.record()
        for _ in range(reps):
            call(ctx_t, True, 0)
        with torch.cuda.stream(torch.cuda.ExternalStream(ctx_t.stream)):
            t1.record()
        t1.synchronize()
        pms = t0.elapsed_time(t1) / reps
        plain = {"value": n / (pms * 1e-3) / 1e6, "unit": "Mparticles/s", "ms_per_step": pms, "precision": "fp64"}
    # the mixed form at the configuration's fixed order and leaf size (what the
    # learned order and leaf size are measured against)
    mixed_fixed = None
    if dim == 3 and learned and not args.no_plain:
        ft = (depth, max_leaf)
        for _ in range(2):
            call(ctx_t, True, prec, tree=ft)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(1, min(args.steps, 3))
        with torch.cuda.stream(torch.cuda.ExternalStream(ctx_t.stream)):
            t0.record()
        for _ in range(reps):
            call(ctx_t, True, prec, tree=ft)
        with torch.cuda.stream(torch.cuda.ExternalStream(ctx_t.stream)):
            t1.record()
        t1.synchronize()
        fms = t0.elapsed_time(t1) / reps
        # its phases (one more solve with the phase events): the tree phase here is
        # the tree build alone, without the learned solve's prediction and check
        stf = LfmmStats()
        call(ctx_t, True, prec, stats=stf, tree=ft)
        torch.cuda.synchronize()
        mixed_fixed = {"value": n / (fms * 1e-3) / 1e6, "unit": "Mparticles/s", "ms_per_step": fms,
                       "precision": cfg["precision"], "N_degrees": N, "max_leaf": max_leaf,
                       "phases_ms": {k: v for k, v in stf.as_dict().items() if k.startswith("ms_")},
                       "what": "the mixed form at the fixed order and leaf size, no prediction or check"}
    # 2D: the reference's uniform quadtree on the same particles beside the adaptive one
    if dim == 2 and max_leaf > 0 and cfg.get("uniform_depth") and not args.no_plain:
        ut = (cfg["uniform_depth"], 0)
        for _ in range(2):
            call(ctx_t, True, prec, tree=ut)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(1, min(args.steps, 3))
        with torch.cuda.stream(torch.cuda.ExternalStream(ctx_t.stream)):
            t0.record()
        for _ in range(reps):
            call(ctx_t, True, prec, tree=ut)
        with torch.cuda.stream(torch.cuda.ExternalStream(ctx_t.stream)):
            t1.record()
        t1.synchronize()
        pms = t0.elapsed_time(t1) / reps
        plain = {"value": n / (pms * 1e-3) / 1e6, "unit": "Mparticles/s", "ms_per_step": pms, "precision": "fp64",
                 "tree": f"uniform quadtree depth {cfg['uniform_depth']} (the reference's tree)"}
    ctx_t.close()
    # a solve plan at the same order: the tree and a CUDA graph built once,
    # charges changed per execution (device buffers)
    plan_line = None
    if dim == 3 and max_leaf > 0 and not args.no_plan:
        Nplan = stats.get("order_N") or N
        hp = ctypes.c_void_p()
        ml_plan = info_box.get("max_leaf") or max_leaf if learned_leaf else max_leaf
        popts = LfmmSolveOpts(Nplan, depth, ml_plan, prec, 1e-8)
        ctx.check(L.lfmm3d_plan_create(ctx.handle, n, vp(d_src.data_ptr()), vp(d_q.data_ptr()), ctypes.byref(popts),
                                       ctypes.byref(hp)), "plan")
        for _ in range(max(1, args.warmup)):
            ctx.check(L.lfmm3d_plan_execute(hp, vp(d_q.data_ptr()), vp(d_pot.data_ptr()), vp(d_fld.data_ptr())), "plan")
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(args.steps):
            ctx.check(L.lfmm3d_plan_execute(hp, vp(d_q.data_ptr()), vp(d_pot.data_ptr()), vp(d_fld.data_ptr())), "plan")
        p1.record(stream)
        p1.synchronize()
        pl_ms = p0.elapsed_time(p1) / args.steps
        L.lfmm3d_plan_destroy(hp)
        plan_line = {"value": world * n / (pl_ms * 1e-3) / 1e6, "unit": "Mparticles/s", "ms_per_step": pl_ms,
                     "N_degrees": Nplan, "max_leaf": ml_plan,
                     "what": "repeated solves on one geometry: tree and CUDA graph built once"}
    # accuracy on 4096 seeded targets against the FP64 direct sum (on the GPU)
    idx = sample_targets(n)
    tgt = torch.from_numpy(np.ascontiguousarray(pos[idx])).cuda()
    e_pot = torch.empty(len(idx), dtype=torch.float64, device="cuda")
    e_fld = torch.empty(len(idx), dim, dtype=torch.float64, device="cuda")
    direct = L.lfmm3d_direct_device if dim == 3 else L.lfmm2d_direct_device
    step_dev()
    ctx.check(direct(ctx.handle, n, vp(d_src.data_ptr()), vp(d_q.data_ptr()), len(idx), vp(tgt.data_ptr()),
                     vp(e_pot.data_ptr()), vp(e_fld.data_ptr())), "direct")
    torch.cuda.synchronize()
    fp, ff = d_pot.cpu().numpy()[idx], d_fld.cpu().numpy()[idx]
    ep, ef = e_pot.cpu().numpy(), e_fld.cpu().numpy()
    self_term = q[idx] * (1e4 if dim == 3 else np.log(1e-4))
    acc = {"rel_l2_pot_noself": rel_l2(fp - self_term, ep - self_term), "rel_l2_pot": rel_l2(fp, ep),
           "rel_l2_field": rel_l2(ff, ef), "targets": int(len(idx))}
    # end to end through the host API with pinned buffers
    e2e = None
    if not args.no_e2e:
        h_src = torch.from_numpy(pos).pin_memory(); h_q = torch.from_numpy(q).pin_memory()
        h_pot = torch.empty(n, dtype=torch.float64).pin_memory()
        h_fld = torch.empty(n, dim, dtype=torch.float64).pin_memory()

        def step_host():
            call(ctx, False, prec, host=(h_src, h_q, h_pot, h_fld))

        for _ in range(max(1, args.warmup)):
            step_host()
        tot = 0.0
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            step_host()
            e.record(stream)
            e.synchronize()
            tot += s.elapsed_time(e)
        e2e_ms = max_over_ranks(tot / args.steps, dist)
        e2e = {"value": aggregate_rate(n, world, e2e_ms), "unit": "Mparticles/s", "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": int(h_src.numel() * 8 + h_q.numel() * 8),
               "d2h_bytes_per_step": int(h_pot.numel() * 8 + h_fld.numel() * 8)}
    return dict(ms=ms, stats=stats, acc=acc, e2e=e2e, clocks=clk.summary(), torch=torch, dist=dist, ctx=ctx,
                plain=plain, learned=dict(info_box) if learned else None, plan=plan_line, mixed_fixed=mixed_fixed)


def m2l_flops(N):
    """Algorithmic flops of one rotation-based M2L: two y-rotations, the
    z-translation and two z-rotations (the reference's operator count)."""
    nx2 = N * (N + 1) // 2
    return 2 * sum((n + 1) * (4 * n + 2) for n in range(N)) + 4 * sum(m * m for m in range(1, N + 1)) + 12 * nx2


# DRAM bytes per millisecond of m2l_tc_kernel time (M2L mode, FP16 operands
# gathered by TMA), from an ncu capture of a 2,097,152-particle case of the
# default workload at N = 17 (176.6 MB read + 73.4 MB written in one 1.061 ms
# launch); the kernel's traffic grows with its work, so a full launch's
# traffic is this rate times its duration.
M2L_TC_DRAM_BYTES_PER_MS = (176.6e6 + 73.4e6) / 1.061


# DRAM bytes per particle of p2p_f32_kernel (mixed 3D form), from an ncu
# capture of a 2,097,152-particle case of the default workload (146.5 MB read
# + 83.0 MB written in one launch): the kernel reads the particle arrays
# (repeated source reads hit L2) and writes the outputs, so its traffic grows
# with the particles.
P2P_DRAM_BYTES_PER_PARTICLE = (146.5e6 + 83.0e6) / 2097152


def padded(N):
    return (N * (N + 1) + 15) // 16 * 16


def tc_executed_per_pair(N, epb=64):
    """Tensor flops the tcgen05 M2L executes per V pair, averaged over the 189
    far offsets of an octant class: B_hi T_hi over the slot's K blocks (epb
    inputs each: 64 for FP16 operands, 32 for TF32; a partial last block runs
    only its K steps below the padded row count) and output columns, plus the
    two hi/lo corrections over the drained columns (degrees < 12) and their K
    blocks; a slot of |d|^2 >= 8 is truncated by 3, 4, 5, 6 degrees for |d|^2
    in [8, 9], [10, 13], [14, 19], [20, 27], never below the drained columns
    (csrc/m2l_tc.cu, tc_trunc)."""
    nc = padded(N)
    na = nc if nc <= 160 else 160
    kb_all, kbc = (nc + epb - 1) // epb, (na + epb - 1) // epb
    step = epb // 4

    def k_in(b):
        left = nc - b * epb
        return epb if left >= epb else (left + step - 1) // step * step

    tot = 0.0
    offs = [(x, y, z) for x in range(-2, 4) for y in range(-2, 4) for z in range(-2, 4)
            if max(abs(x), abs(y), abs(z)) > 1]
    for x, y, z in offs:
        d2 = x * x + y * y + z * z
        r = 0 if d2 < 8 else 3 if d2 < 10 else 4 if d2 < 14 else 5 if d2 < 20 else 6
        nd = max(1, N - r)
        kb = max(kbc, min(kb_all, (nd * (nd + 1) + epb - 1) // epb))
        cols = min(nc, epb * kb)
        tot += sum(2.0 * cols * k_in(b) for b in range(kb)) + sum(2 * 2.0 * na * k_in(b) for b in range(kbc))
    return tot / len(offs)


def roofline(cfg, stats, peaks, fp64_tflops, fp32_tflops, tf32_tflops, phase=None):
    """Roofline of the dominant phase (device time from the phase events; for
    the tensor-core M2L, the summed CUDA-event time of its kernel launches).
    P2P: 20 flops per particle pair; M2L: the rotation method's algorithmic
    flops per V pair (executed dense-GEMM / tensor flops reported beside it)."""
    phases = {"leaves": stats["ms_leaves"], "m2l": stats["ms_m2l"], "tree": stats["ms_tree"],
              "upward": stats["ms_upward"], "l2l": stats["ms_l2l"]}
    dom = phase or max(phases, key=phases.get)
    ms = phases[dom]
    fp64 = cfg["precision"] == "fp64"
    if dom == "m2l" and cfg["dim"] == 2:
        # 2D: one complex N x N operator per far pair, 8 N^2 real flops; the
        # GEMMs run it as a real MT x MT block (MT = 2N rounded up to 16)
        ms_k = stats.get("ms_m2l_kernel") or ms
        N = cfg["N"]
        mt = (2 * N + 15) // 16 * 16
        flops = 8.0 * N * N * stats["n_far_pairs"]
        executed = 2.0 * mt * mt * stats["n_far_pairs"]
        achieved = flops / (ms_k * 1e-3) / 1e12
        return {"kernel": "m2l_gemm_kernel<double, *, 4, 2> (2D FP64 GEMMs by quadrant class and offset)",
                "bound": "fp64", "achieved": achieved, "peak": fp64_tflops, "unit": "TFLOP/s",
                "frac": achieved / fp64_tflops, "peak_source": "measured cuBLAS DGEMM", "algorithmic_flops": flops,
                "executed_dense_flops": executed, "executed_tflops": executed / (ms_k * 1e-3) / 1e12,
                "kernel_ms": ms_k, "kernel_launches": stats.get("n_m2l_kernel", 0), "phase_ms": phases["m2l"],
                "traffic": None}
    if dom == "m2l" and stats.get("n_m2l_kernel", 0) > 0 and stats["ms_m2l_kernel"] > 0:
        ms = stats["ms_m2l_kernel"]
        N = stats.get("order_N") or cfg["N"]
        flops = float(m2l_flops(N)) * stats["n_far_pairs"]
        # per V pair: B_hi T_hi over the slot's columns and K blocks, and the
        # two corrections over the drained columns and their source degrees;
        # the farther offsets run truncated (the kernel's rule), averaged here
        # over the 189 far offsets of an octant class
        tensor = tc_executed_per_pair(N) * stats["n_far_pairs"]
        achieved = flops / (ms * 1e-3) / 1e12
        bf16 = peaks["bf16_tflops"]
        return {"kernel": "m2l_tc_kernel (tcgen05 FP16 hi/lo, direction-grouped)", "bound": "tensor",
                "achieved": achieved, "peak": bf16, "unit": "TFLOP/s", "frac": achieved / bf16,
                "peak_source": f"MEASURED_PEAKS.json bf16_tflops ({peaks['source']}); the kernel runs FP16 MMAs, "
                               "whose dense rate is bf16's",
                "algorithmic_flops": flops,
                "executed_tensor_flops": tensor, "executed_tensor_tflops": tensor / (ms * 1e-3) / 1e12,
                "executed_frac": tensor / (ms * 1e-3) / 1e12 / bf16,
                "kernel_ms": ms, "kernel_launches": stats["n_m2l_kernel"], "phase_ms": phases["m2l"],
                "traffic": M2L_TC_DRAM_BYTES_PER_MS * ms / stats["n_m2l_kernel"],
                "traffic_unit": "bytes per launch (ncu capture of a 2M-particle case, scaled by kernel time)"}
    peak = fp64_tflops if fp64 else fp32_tflops
    src = "measured cuBLAS DGEMM" if fp64 else "measured cuBLAS SGEMM (TF32 off)"
    if dom == "leaves":
        flops = 20.0 * stats["n_p2p_pairs"]     # 2D: 20 flops and one FP64 log per pair
        achieved = flops / (ms * 1e-3) / 1e12
        line = {"kernel": "leaves kernel (P2P + M2P + L2P)", "bound": "fp64" if fp64 else "fp32",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": src, "algorithmic_flops": flops, "phase_ms": ms, "traffic": None,
                "flop_model": "20 flops per near-field (target, source) pair; the phase time also holds "
                              "the expansions' evaluation at the targets (M2P over W, L2P)"}
        if cfg["dim"] == 3 and not fp64 and stats.get("n_particles"):
            # the near-field kernel's DRAM bytes: P2P_DRAM_BYTES_PER_PARTICLE x particles
            line["kernel"] = "p2p_f32_kernel (near field) + eval_scaled_kernel (M2P, L2P)"
            line["traffic"] = P2P_DRAM_BYTES_PER_PARTICLE * stats["n_particles"]
            line["traffic_unit"] = ("bytes of the near-field launch (ncu capture of a 2M-particle case, "
                                    "scaled by particles)")
        return line
    if dom == "m2l":
        Nd = stats.get("order_N") or cfg["N"]
        flops = float(m2l_flops(Nd)) * stats["n_far_pairs"]
        R = Nd * (Nd + 1)
        executed = 2.0 * R * R * stats["n_far_pairs"]
        achieved = flops / (ms * 1e-3) / 1e12
        return {"kernel": "m2l_gemm_kernel (direction-grouped GEMM)", "bound": "fp64" if fp64 else "fp32",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": src, "algorithmic_flops": flops, "executed_dense_flops": executed,
                "executed_tflops": executed / (ms * 1e-3) / 1e12, "phase_ms": ms, "traffic": None}
    # tree / upward: HBM-bound passes over the particles
    nbytes = stats["n_particles"] * (2 * 32 + 2 * 8 + 4)
    achieved = nbytes / (ms * 1e-3) / 1e9
    return {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "algorithmic_bytes": nbytes, "phase_ms": ms, "traffic": None}


# ---------------------------------------------------------------- CPU legs
def cpu_sample(cfg):
    """Bounded sample of the configuration for the host-core baselines (a few
    seconds per solve): the full problem for the small configurations; for
    the large ones every 64th particle of the seeded set (the same mixture)
    on a uniform tree three levels shallower (the reference has no adaptive
    tree).  Returns (stride, depth, description)."""
    if cfg["n"] <= 200000:
        return 1, cfg["depth"], "full problem"
    d = max(3, cfg.get("uniform_depth", cfg["depth"]) - 3)
    return 64, d, f"every 64th particle of the seeded set ({cfg['n'] // 64}), uniform depth {d}"


def cpu_solver():
    from oracle.oracle import ORACLE_SO, REF_SO, Oracle, Reference, build
    if REF_SO.exists():
        return Reference(), "reference"
    if not ORACLE_SO.exists():
        build(("oracle",))
    return Oracle(), "port"


def run_cpu(cfg, pos, q, steps):
    solver, kind = cpu_solver()
    cores = os.cpu_count() or 1
    solver.set_threads(cores)
    stride, depth, sample = cpu_sample(cfg)
    p, qq = np.ascontiguousarray(pos[::stride]), np.ascontiguousarray(q[::stride])
    n = len(p)
    fn = solver.fmm3d if cfg["dim"] == 3 else solver.fmm2d
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        fn(p, qq, N=cfg["N"], depth=depth)
        times.append(time.perf_counter() - t0)
    s = float(np.median(times))
    return {"value": n / s / 1e6, "unit": "Mparticles/s", "cores": cores, "kind": kind, "sample": sample,
            "seconds_per_solve": s}


def base_config(cfg, world):
    return {"workload": cfg["workload"], "particles": cfg["n"], "order_p": cfg["N"] - 1, "N_degrees": cfg["N"],
            "tree_depth": cfg["depth"], "precision": cfg["precision"],
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "inputs > L2" if cfg["n"] * 32 > 126e6 else "L2 flushed (256 MB write) between steps"}


def run_batch(args, cfg):
    """Batched solves: one forest solve of all problems (device buffers), the
    plain FP64 form one problem at a time, per-problem accuracy."""
    import torch
    from laplace_fmm_b200 import Context
    from laplace_fmm_b200._lib import PRECISION, LfmmLearnedInfo, LfmmSolveOpts, LfmmStats
    from laplace_fmm_b200.workloads import batch3d, rel_l2
    probs = batch3d(cfg["count"], seed=cfg["seed"])
    sizes = np.array([len(p) for p, _ in probs], dtype=np.uint64)
    offs = np.zeros(len(probs) + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(sizes)
    pos = np.ascontiguousarray(np.concatenate([p for p, _ in probs]))
    q = np.ascontiguousarray(np.concatenate([c for _, c in probs]))
    n = len(pos)
    ctx = Context(0)
    L = ctx.lib
    vp = ctypes.c_void_p
    d_src, d_q = torch.from_numpy(pos).cuda(), torch.from_numpy(q).cuda()
    d_pot = torch.empty(n, dtype=torch.float64, device="cuda")
    d_fld = torch.empty(n, 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream)
    learned = bool(cfg.get("learned")) and not args.no_learned
    learned_leaf = learned and bool(cfg.get("learned_leaf"))
    opts = LfmmSolveOpts(cfg["N"], cfg["depth"], 2147483647 if learned_leaf else cfg["max_leaf"],
                         PRECISION[cfg["precision"]], 1e-8)
    info = LfmmLearnedInfo()
    if learned:
        from laplace_fmm_b200.order import load_params
        d_params = torch.from_numpy(load_params(leaf=learned_leaf)).cuda()

    def step():
        if learned:
            ctx.check(L.lfmm3d_solve_batch_learned_device(
                ctx.handle, len(probs), offs.ctypes.data_as(vp), vp(d_src.data_ptr()), vp(d_q.data_ptr()),
                ctypes.byref(opts), vp(d_params.data_ptr()), cfg["tol"], cfg["check_targets"], vp(d_pot.data_ptr()),
                vp(d_fld.data_ptr()), ctypes.byref(info), None), "learned batch")
        else:
            ctx.check(L.lfmm3d_solve_batch_device(ctx.handle, len(probs), offs.ctypes.data_as(vp),
                                                  vp(d_src.data_ptr()), vp(d_q.data_ptr()), ctypes.byref(opts),
                                                  vp(d_pot.data_ptr()), vp(d_fld.data_ptr()), None), "batch")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(0) as clk:
        for k in range(args.steps):
            starts[k].record(stream)
            step()
            ends[k].record(stream)
        torch.cuda.synchronize()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / args.steps
    # per-problem accuracy against its own FP64 direct sum: every output of a problem of up to 65536
    # particles, 8192 evenly spread outputs of a larger one (a sample of a few dozen outputs can miss the
    # high-field targets that dominate the norm and overstate a problem's rel-L2 several times)
    pot, fld = d_pot.cpu().numpy(), d_fld.cpu().numpy()
    errs_p, errs_f = [], []
    for k, (p, c) in enumerate(probs):
        b = int(offs[k])
        idx = np.arange(len(p)) if len(p) <= 65536 else np.arange(0, len(p), len(p) // 8192)
        tgt = torch.from_numpy(np.ascontiguousarray(p[idx])).cuda()
        ep = torch.empty(len(idx), dtype=torch.float64, device="cuda")
        ef = torch.empty(len(idx), 3, dtype=torch.float64, device="cuda")
        ctx.check(L.lfmm3d_direct_device(ctx.handle, len(p), vp(d_src.data_ptr() + 24 * b),
                                         vp(d_q.data_ptr() + 8 * b), len(idx), vp(tgt.data_ptr()),
                                         vp(ep.data_ptr()), vp(ef.data_ptr())), "direct")
        stream.synchronize()
        self_t = c[idx] * 1e4
        errs_p.append(rel_l2(pot[b + idx] - self_t, ep.cpu().numpy() - self_t))
        errs_f.append(rel_l2(fld[b + idx], ef.cpu().numpy()))
    # the plain FP64 form, one problem at a time (uniform octree, automatic
    # depth); warmed on the first problems, timed once over all of them
    def plain_all(count=None):
        for k, (p, c) in enumerate(probs[:count]):
            b = int(offs[k])
            ctx.check(L.lfmm3d_solve_device(ctx.handle, len(p), vp(d_src.data_ptr() + 24 * b),
                                            vp(d_q.data_ptr() + 8 * b), 0, None, cfg["plain_N"], 2147483647, 1e-8,
                                            0, vp(d_pot.data_ptr() + 8 * b), vp(d_fld.data_ptr() + 24 * b), None),
                      "plain")

    plain_all(8)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    plain_all()
    t1.record(stream)
    t1.synchronize()
    pms = t0.elapsed_time(t1)
    ep_ = np.array(errs_p); ef_ = np.array(errs_f)
    worst = [{"problem": int(k), "particles": int(len(probs[k][0])), "rel_l2_pot_noself": float(ep_[k]),
              "rel_l2_field": float(ef_[k])} for k in np.argsort(-np.maximum(ep_, ef_))[:5]]
    line = {"metric": "batched 3D FMM aggregate Mparticles/s", "value": n / (ms * 1e-3) / 1e6,
            "unit": "Mparticles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/tf32",
            "data": "synthetic (seeded PCG64)",
            "config": {"workload": cfg["workload"], "problems": len(probs), "particles": int(n),
                       "N_degrees": cfg["N"], "tree_depth": cfg["depth"], "precision": cfg["precision"],
                       "parallelism": "single GPU", "l2": "inputs > L2"},
            "accuracy": {"rel_l2_pot_noself_median": float(np.median(ep_)), "rel_l2_pot_noself_p95":
                         float(np.quantile(ep_, 0.95)), "rel_l2_pot_noself_max": float(ep_.max()),
                         "rel_l2_field_median": float(np.median(ef_)), "rel_l2_field_max": float(ef_.max()),
                         "targets_per_problem": "every output up to 65536 particles, else 8192 evenly spread", "within_tol": int(np.sum(np.maximum(ep_, ef_) <= cfg["tol"])),
                         "worst_problems": worst},
            "plain_fp64_one_at_a_time": {"value": n / (pms * 1e-3) / 1e6, "unit": "Mparticles/s",
                                         "ms": pms, "N_degrees": cfg["plain_N"]},
            "speedup_vs_plain_fp64": pms / ms, "clocks": clk.summary()}
    if learned:
        line["learned_order"] = dict(info.as_dict(), tol=cfg["tol"], check_targets_per_problem=cfg["check_targets"])
        line["config"]["N_degrees"] = info.order_N
    # the same batch as a batch plan (forest and one CUDA graph built once, new
    # charges per execution) at the order and leaf size the learned solve used
    if not args.no_plan:
        Np = info.order_N if learned else cfg["N"]
        mlp = (info.max_leaf or cfg["max_leaf"]) if learned else cfg["max_leaf"]
        popts = LfmmSolveOpts(Np, cfg["depth"], mlp, PRECISION[cfg["precision"]], 1e-8)
        hp = ctypes.c_void_p()
        ctx.check(L.lfmm3d_plan_create_batch(ctx.handle, len(probs), offs.ctypes.data_as(vp), vp(d_src.data_ptr()),
                                             vp(d_q.data_ptr()), ctypes.byref(popts), ctypes.byref(hp)), "batch plan")
        for _ in range(max(1, args.warmup)):
            ctx.check(L.lfmm3d_plan_execute(hp, vp(d_q.data_ptr()), vp(d_pot.data_ptr()), vp(d_fld.data_ptr())), "plan")
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(args.steps):
            ctx.check(L.lfmm3d_plan_execute(hp, vp(d_q.data_ptr()), vp(d_pot.data_ptr()), vp(d_fld.data_ptr())), "plan")
        p1.record(stream)
        p1.synchronize()
        pl_ms = p0.elapsed_time(p1) / args.steps
        L.lfmm3d_plan_destroy(hp)
        line["batch_plan_execute"] = {"value": n / (pl_ms * 1e-3) / 1e6, "unit": "Mparticles/s", "ms_per_step": pl_ms,
                                      "N_degrees": Np, "max_leaf": mlp,
                                      "what": "repeated batch solves: forest and one CUDA graph built once"}
    ctx.close()
    print(json.dumps(line))
    return 0


def vector_launches(depth, precision):
    """One tree, three scalar passes, the nonzero-charge, three component and
    one cross-product kernels."""
    tree, fmm = launches_per_solve(depth, 3, (3 * (depth - 1) + 7) // 8, True, precision, parts=True)
    return tree + 3 * fmm + 1 + 3 + 1


def run_vector(args, cfg):
    """Vector charges: the solve on device buffers, end to end through the
    host entry point, accuracy at 4096 targets against the FP64 direct sum
    (three scalar direct sums combined by the cross product), the FP64 form
    beside it and the reference's own vector FMM on the host cores."""
    import torch
    from laplace_fmm_b200 import Context
    from laplace_fmm_b200._lib import PRECISION, LfmmSolveOpts, LfmmStats
    from laplace_fmm_b200.workloads import rel_l2, sample_targets
    n, N, depth, ml = cfg["n"], cfg["N"], cfg["depth"], cfg["max_leaf"]
    pos, _ = make_particles(cfg)
    q3 = np.random.Generator(np.random.PCG64(cfg["seed"] + 1)).uniform(-1, 1, (n, 3))
    ctx = Context(0)
    L = ctx.lib
    vp = ctypes.c_void_p
    stream = torch.cuda.ExternalStream(ctx.stream)
    d_src, d_q = torch.from_numpy(pos).cuda(), torch.from_numpy(q3).cuda()
    d_fld = torch.empty((n, 3), dtype=torch.float64, device="cuda")

    def solve(precision, stats=None, host=None, c=None):
        c = c or ctx
        opts = LfmmSolveOpts(N, depth, ml, PRECISION[precision], 1e-8)
        sp = ctypes.byref(stats) if stats is not None else None
        if host:
            hs, hq, hf = host
            c.check(L.lfmm3d_solve_vector(c.handle, n, vp(hs.data_ptr()), vp(hq.data_ptr()), 0, None,
                                          ctypes.byref(opts), vp(hf.data_ptr()), sp), "vector solve")
        else:
            c.check(L.lfmm3d_solve_vector_device(c.handle, n, vp(d_src.data_ptr()), vp(d_q.data_ptr()), 0, None,
                                                 ctypes.byref(opts), vp(d_fld.data_ptr()), sp), "vector solve")

    def timed(fn, steps):
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for k in range(steps):
            starts[k].record(stream)
            fn()
            ends[k].record(stream)
        torch.cuda.synchronize()
        return sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / steps

    for _ in range(args.warmup):
        solve(cfg["precision"])
    with ClockSampler(0) as clk:
        ms = timed(lambda: solve(cfg["precision"]), args.steps)
    st = LfmmStats()
    ctx_t = Context(0, timing=True)
    solve(cfg["precision"], c=ctx_t)                  # warms this context's caches
    solve(cfg["precision"], stats=st, c=ctx_t)
    torch.cuda.synchronize()
    ctx_t.close()
    field = d_fld.cpu().numpy()
    # accuracy: B = sum_c e_c x E^(c) from three FP64 direct sums at the sampled targets
    idx = sample_targets(n)
    tgt = torch.from_numpy(np.ascontiguousarray(pos[idx])).cuda()
    E = []
    for c in range(3):
        qc = torch.from_numpy(np.ascontiguousarray(q3[:, c])).cuda()
        ep = torch.empty(len(idx), dtype=torch.float64, device="cuda")
        ef = torch.empty((len(idx), 3), dtype=torch.float64, device="cuda")
        ctx.check(L.lfmm3d_direct_device(ctx.handle, n, vp(d_src.data_ptr()), vp(qc.data_ptr()), len(idx),
                                         vp(tgt.data_ptr()), vp(ep.data_ptr()), vp(ef.data_ptr())), "direct")
        stream.synchronize()
        E.append(ef.cpu().numpy())
    Bd = np.stack([E[1][:, 2] - E[2][:, 1], E[2][:, 0] - E[0][:, 2], E[0][:, 1] - E[1][:, 0]], axis=1)
    acc = {"rel_l2_field": rel_l2(field[idx], Bd), "targets": len(idx)}
    # the FP64 form
    solve("fp64")
    pms = timed(lambda: solve("fp64"), max(1, min(args.steps, 3)))
    # end to end through the host entry point (pinned buffers)
    hs, hq = torch.from_numpy(pos).pin_memory(), torch.from_numpy(q3).pin_memory()
    hf = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    solve(cfg["precision"], host=(hs, hq, hf))
    e2e_ms = timed(lambda: solve(cfg["precision"], host=(hs, hq, hf)), max(1, min(args.steps, 3)))
    # the reference's own vector FMM (host cores) on every 64th particle, uniform depth 7
    cpu = None
    if not args.no_cpu_baseline:
        solver, kind = cpu_solver()
        if kind == "reference":
            cores = os.cpu_count() or 1
            solver.set_threads(cores)
            p, qq = np.ascontiguousarray(pos[::64]), np.ascontiguousarray(q3[::64])
            t0 = time.perf_counter()
            solver.fmm3d_vec(p, qq, N=N, depth=7)
            s = time.perf_counter() - t0
            cpu = {"value": len(p) / s / 1e6, "unit": "Mparticles/s", "cores": cores, "kind": kind,
                   "sample": f"every 64th particle of the seeded set ({len(p)}), uniform depth 7"}
    peaks = measured_peaks()
    stats = st.as_dict()
    tf32 = tf32_peak_tflops(torch)
    line = {"metric": cfg["metric"], "value": n / (ms * 1e-3) / 1e6, "unit": "Mparticles/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/tf32", "data": "synthetic (seeded PCG64)",
            "config": base_config(cfg, 1), "accuracy": acc,
            "phases_ms_last_pass": {k: stats[k] for k in ("ms_tree", "ms_upward", "ms_m2l", "ms_l2l", "ms_leaves",
                                                          "ms_total", "ms_m2l_kernel")},
            "roofline_last_pass": roofline(cfg, stats, peaks, fp64_peak_tflops(torch), fp32_peak_tflops(torch), tf32),
            "e2e": {"value": n / (e2e_ms * 1e-3) / 1e6, "unit": "Mparticles/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(hs.numel() * 8 + hq.numel() * 8), "d2h_bytes_per_step": int(hf.numel() * 8)},
            "plain_fp64": {"value": n / (pms * 1e-3) / 1e6, "unit": "Mparticles/s", "ms_per_step": pms},
            "speedup_vs_plain_fp64": pms / ms, "cpu_baseline": cpu, "clocks": clk.summary(),
            "gpu_launches": args.steps * vector_launches(depth, cfg["precision"])}
    ctx.close()
    print(json.dumps(line))
    return 0


def run_heldout(args, cfg):
    """The learned order on the network's held-out problems: per problem the
    learned solve (features, network, order, solve, sampled check and
    fallback) and the solve at the lowest single fixed order that meets tol
    on every one of them, both on device buffers and timed with CUDA events
    on the solver's stream (the learned solve's host synchronisations count);
    accuracy of both at up to 4096 sampled targets against the FP64 direct
    sum.  value = all particles / the summed learned solve time."""
    import torch
    from laplace_fmm_b200 import Context
    from laplace_fmm_b200._lib import PRECISION, LfmmLearnedInfo, LfmmSolveOpts
    from laplace_fmm_b200.order import load_params
    from laplace_fmm_b200.train_order import problem
    from laplace_fmm_b200.workloads import rel_l2, sample_targets
    probs = [problem(i, "heldout") for i in range(cfg["count"])]
    ctx = Context(0)
    L = ctx.lib
    vp = ctypes.c_void_p
    stream = torch.cuda.ExternalStream(ctx.stream)
    learned_leaf = bool(cfg.get("learned_leaf"))
    d_params = torch.from_numpy(load_params(leaf=learned_leaf)).cuda()
    prec, tol, depth, ml = PRECISION[cfg["precision"]], cfg["tol"], cfg["depth"], cfg["max_leaf"]
    dev = []
    for pos, q in probs:
        n = len(pos)
        idx = sample_targets(n)
        ds, dq = torch.from_numpy(pos).cuda(), torch.from_numpy(q).cuda()
        tgt = torch.from_numpy(np.ascontiguousarray(pos[idx])).cuda()
        ep = torch.empty(len(idx), dtype=torch.float64, device="cuda")
        ef = torch.empty(len(idx), 3, dtype=torch.float64, device="cuda")
        ctx.check(L.lfmm3d_direct_device(ctx.handle, n, vp(ds.data_ptr()), vp(dq.data_ptr()), len(idx),
                                         vp(tgt.data_ptr()), vp(ep.data_ptr()), vp(ef.data_ptr())), "direct")
        stream.synchronize()
        self_t = q[idx] * 1e4
        dev.append(dict(n=n, ds=ds, dq=dq, idx=idx, ep=ep.cpu().numpy() - self_t, ef=ef.cpu().numpy(), self_t=self_t,
                        pot=torch.empty(n, dtype=torch.float64, device="cuda"),
                        fld=torch.empty(n, 3, dtype=torch.float64, device="cuda")))
    info = LfmmLearnedInfo()

    def learned(d):
        opts = LfmmSolveOpts(cfg["N"], depth, 2147483647 if learned_leaf else ml, prec, tol)
        ctx.check(L.lfmm3d_solve_learned_device(ctx.handle, d["n"], vp(d["ds"].data_ptr()), vp(d["dq"].data_ptr()),
                                                0, None, ctypes.byref(opts), vp(d_params.data_ptr()), tol,
                                                cfg["check_targets"], vp(d["pot"].data_ptr()),
                                                vp(d["fld"].data_ptr()), ctypes.byref(info), None), "learned")

    def fixed(d, N):
        opts = LfmmSolveOpts(N, depth, ml, prec, 1e-8)
        ctx.check(L.lfmm3d_solve_ex_device(ctx.handle, d["n"], vp(d["ds"].data_ptr()), vp(d["dq"].data_ptr()), 0,
                                           None, ctypes.byref(opts), vp(d["pot"].data_ptr()), vp(d["fld"].data_ptr()),
                                           None), "fixed")

    def errors(d):
        stream.synchronize()
        pot, fld = d["pot"].cpu().numpy()[d["idx"]], d["fld"].cpu().numpy()[d["idx"]]
        return rel_l2(pot - d["self_t"], d["ep"]), rel_l2(fld, d["ef"])

    # the lowest fixed order meeting tol (both outputs) on every problem
    fixed_N = 18
    for Nf in range(10, 19):
        ok = True
        for d in dev:
            fixed(d, Nf)
            ep_, ef_ = errors(d)
            if max(ep_, ef_) > tol:
                ok = False
                break
        if ok:
            fixed_N = Nf
            break

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            t0.record()
        for _ in range(args.steps):
            fn()
        with torch.cuda.stream(stream):
            t1.record()
        t1.synchronize()
        return t0.elapsed_time(t1) / args.steps

    rows = []
    with ClockSampler(0) as clk:
        for d in dev:
            tf = timed(lambda: fixed(d, fixed_N))
            ef_fixed = errors(d)
            tl = timed(lambda: learned(d))
            el = errors(d)
            rows.append(dict(n=d["n"], N=info.order_N, predicted_N=info.predicted_N, max_leaf=info.max_leaf,
                             fallback=info.fallback,
                             fp64=info.fp64_resolved, ms_learned=tl, ms_fixed=tf, err_pot=el[0], err_field=el[1],
                             err_pot_fixed=ef_fixed[0], err_field_fixed=ef_fixed[1]))
    ctx.close()
    ntot = sum(r["n"] for r in rows)
    tl, tf = sum(r["ms_learned"] for r in rows), sum(r["ms_fixed"] for r in rows)
    big = [r for r in rows if r["n"] >= 100000]
    line = {"metric": cfg["metric"], "value": ntot / (tl * 1e-3) / 1e6, "unit": "Mparticles/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tl, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/tf32", "data": "synthetic (seeded PCG64)",
            "config": {"workload": cfg["workload"], "problems": len(rows), "particles": ntot,
                       "tree_depth": depth, "max_leaf": ml, "precision": cfg["precision"], "tol": tol,
                       "parallelism": "single GPU", "l2": "each problem's working set is below L2; no flush"},
            "fixed_order": {"N_degrees": fixed_N, "value": ntot / (tf * 1e-3) / 1e6, "unit": "Mparticles/s",
                            "ms_total": tf, "what": "lowest single fixed order meeting tol on all problems"},
            "gain_vs_fixed": tf / tl,
            "gain_vs_fixed_problems_over_1e5": (sum(r["ms_fixed"] for r in big) / sum(r["ms_learned"] for r in big)
                                                if big else None),
            "within_tol": sum(1 for r in rows if max(r["err_pot"], r["err_field"]) <= tol),
            "max_err_pot": max(r["err_pot"] for r in rows), "max_err_field": max(r["err_field"] for r in rows),
            "mean_N_learned": float(np.mean([r["N"] for r in rows])),
            "fallbacks": sum(1 for r in rows if r["fallback"]), "fp64_reruns": sum(r["fp64"] for r in rows),
            "per_problem": rows, "clocks": clk.summary(),
            "e2e": None, "gpu_launches": None}
    print(json.dumps(line))
    return 0


def run_cpu_series(args, cfg, pos, q):
    """The reference's CPU FMM on growing strided samples of the configuration
    (1/64, 1/16, 1/4), one solve each: how its throughput falls with the
    sample's size on a uniform tree (its automatic depth plus 3, the depth
    the default sample uses)."""
    import math
    solver, kind = cpu_solver()
    cores = os.cpu_count() or 1
    solver.set_threads(cores)
    series = []
    for stride in (64, 16, 4):
        p, qq = np.ascontiguousarray(pos[::stride]), np.ascontiguousarray(q[::stride])
        auto = int(max(2.0, 1 + math.log(len(p) / 100.0) / math.log(8.0)))
        depth = auto + 3
        t0 = time.perf_counter()
        solver.fmm3d(p, qq, N=cfg["N"], depth=depth)
        sec = time.perf_counter() - t0
        series.append({"stride": stride, "particles": len(p), "tree_depth": depth, "seconds": sec,
                       "Mparticles_per_s": len(p) / sec / 1e6})
        print(json.dumps(series[-1]), file=sys.stderr, flush=True)
    print(json.dumps({"impl": "reference", "metric": cfg.get("metric", METRIC), "cpu_series": series,
                      "cores": cores, "kind": kind, "N_degrees": cfg["N"], "workload": cfg["workload"]}))
    return 0


def run_heldout_reference(args, cfg):
    """The reference's CPU FMM on the first held-out problems (a bounded
    sample) at the fixed order N = 17 and its own automatic depth."""
    from laplace_fmm_b200.train_order import problem
    solver, kind = cpu_solver()
    cores = os.cpu_count() or 1
    solver.set_threads(cores)
    probs = [problem(i, "heldout") for i in range(4)]
    ntot, secs = 0, 0.0
    for k in range(args.warmup + args.steps):
        for pos, q in probs:
            t0 = time.perf_counter()
            solver.fmm3d(pos, q, N=cfg["N"])
            if k >= args.warmup:
                secs += time.perf_counter() - t0
                ntot += len(pos)
    v = ntot / secs / 1e6
    sample = f"held-out problems 0-3 ({sum(len(p) for p, _ in probs)} particles), N = {cfg['N']}, the reference's depth"
    print(json.dumps({"impl": "reference", "metric": cfg["metric"], "value": v, "unit": "Mparticles/s",
                      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": secs * 1e3 / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64)",
                      "config": {"workload": cfg["workload"]},
                      "cpu_baseline": {"value": v, "unit": "Mparticles/s", "cores": cores, "kind": kind, "sample": sample},
                      "e2e": {"value": v, "unit": "Mparticles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def run_reference_gpu(args, cfg):
    """The reference's CUDA FMM, timed per constructor call (its whole solve:
    particles copied in, a device synchronisation after every kernel, results
    copied out, so the wall time is its end-to-end time), and its accuracy at
    the 4096 sampled targets against our GPU FP64 direct sum.  The reference
    has only the uniform tree: the configuration's depth, or ``--depth`` for the
    adaptive configurations (default 8)."""
    from oracle.oracle import REF_GPU_SO, ReferenceGPU
    from laplace_fmm_b200 import Context
    from laplace_fmm_b200.workloads import rel_l2, sample_targets
    if not REF_GPU_SO.exists():
        print(json.dumps({"impl": "reference-gpu", "unavailable": "the reference CUDA build (oracle/_ref/libfmmref_gpu.so) "
                                                                  "is absent: make -C oracle ref-gpu"}))
        return 0
    if cfg.get("batch") or cfg.get("vector"):
        print(json.dumps({"impl": "reference-gpu", "unavailable": "the reference GPU path solves one scalar-charge "
                                                                  "problem per call (fmm::gpu::FastMultipole3d<double>)"}))
        return 0
    dim = cfg["dim"]
    adaptive = cfg.get("max_leaf", 0) > 0
    depth = args.depth or (8 if adaptive else cfg["depth"])
    pos, q = make_particles(cfg)
    n = len(pos)
    ref = ReferenceGPU()
    fn = ref.fmm3d if dim == 3 else ref.fmm2d
    secs = []
    for k in range(args.warmup + args.steps):
        pot, fld, sec = fn(pos, q, N=cfg["N"], depth=depth)
        if k >= args.warmup:
            secs.append(sec)
    s = float(np.median(secs))
    ctx = Context(0)
    idx = sample_targets(n)
    tgt = np.ascontiguousarray(pos[idx])
    ep = np.zeros(len(idx)); ef = np.zeros((len(idx), dim))
    direct = ctx.lib.lfmm3d_direct if dim == 3 else ctx.lib.lfmm2d_direct
    vp = ctypes.c_void_p
    ctx.check(direct(ctx.handle, n, pos.ctypes.data_as(vp), q.ctypes.data_as(vp), len(idx), tgt.ctypes.data_as(vp),
                     ep.ctypes.data_as(vp), ef.ctypes.data_as(vp)), "direct")
    ctx.close()
    self_term = q[idx] * (1e4 if dim == 3 else np.log(1e-4))
    acc = {"rel_l2_pot_noself": rel_l2(pot[idx] - self_term, ep - self_term), "rel_l2_pot": rel_l2(pot[idx], ep),
           "rel_l2_field": rel_l2(fld[idx], ef), "targets": int(len(idx)),
           "finite": bool(np.isfinite(pot).all() and np.isfinite(fld).all())}
    v = n / s / 1e6
    conf = base_config(cfg, 1)
    conf.update(tree_depth=depth, tree="uniform", precision="fp64")
    if adaptive:
        conf["workload"] += f" [reference GPU: uniform octree depth {depth}, FP64, N = {cfg['N']}]"
    print(json.dumps({"impl": "reference-gpu", "metric": cfg.get("metric", METRIC), "value": v,
                      "unit": "Mparticles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": s * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                      "dtype": "f64", "data": "synthetic (seeded PCG64)", "config": conf, "accuracy": acc,
                      "seconds_per_solve": secs,
                      "what": "fmm::gpu::FastMultipole3d<double> / fmm::gpu::FastMultipole (unmodified reference "
                              "CUDA sources, sm_100a, allocations zero-filled); wall time of the constructor",
                      "e2e": {"value": v, "unit": "Mparticles/s", "h2d_bytes_per_step": int(n * (dim + 2) * 8),
                              "d2h_bytes_per_step": int(n * (dim + 1) * 8)}}))
    return 0


def main():
    args = parse()
    cfg = args.cfg
    if args.impl == "reference-gpu":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        return run_reference_gpu(args, cfg)
    if cfg.get("batch"):
        return run_batch(args, cfg)
    if cfg.get("heldout") and args.impl == "ours":
        return run_heldout(args, cfg)
    if cfg.get("vector") and args.impl == "ours":
        return run_vector(args, cfg)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if "RANK" not in os.environ:
        world = 1
    if args.impl == "reference":
        if rank != 0:
            return 0
        if cfg.get("heldout"):
            return run_heldout_reference(args, cfg)
        pos, q = make_particles(cfg)
        if args.cpu_series:
            return run_cpu_series(args, cfg, pos, q)
        if cfg.get("vector"):
            # the reference's vector FMM on the same particles and charges (sample as run_vector's)
            q = np.random.Generator(np.random.PCG64(cfg["seed"] + 1)).uniform(-1, 1, (cfg["n"], 3))
            solver, kind = cpu_solver()
            if kind != "reference":
                print(json.dumps({"impl": "reference", "unavailable": "the reference build (oracle/_ref) is absent"}))
                return 0
            cores = os.cpu_count() or 1
            solver.set_threads(cores)
            p, qq = np.ascontiguousarray(pos[::64]), np.ascontiguousarray(q[::64])
            times = []
            for k in range(args.warmup + args.steps):
                t0 = time.perf_counter()
                solver.fmm3d_vec(p, qq, N=cfg["N"], depth=7)
                if k >= args.warmup:
                    times.append(time.perf_counter() - t0)
            s = float(np.median(times))
            v = len(p) / s / 1e6
            sample = f"every 64th particle of the seeded set ({len(p)}), uniform depth 7"
            print(json.dumps({"impl": "reference", "metric": cfg["metric"], "value": v, "unit": "Mparticles/s",
                              "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": s * 1e3, "higher_is_better": True, "scaling": "weak",
                              "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64)",
                              "config": base_config(cfg, 1),
                              "cpu_baseline": {"value": v, "unit": "Mparticles/s", "cores": cores, "kind": kind,
                                               "sample": sample},
                              "e2e": {"value": v, "unit": "Mparticles/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
            return 0
        for _ in range(max(0, min(args.warmup, 1))):
            run_cpu(cfg, pos, q, 1)
        cb = run_cpu(cfg, pos, q, args.steps)
        line = {"impl": "reference", "metric": cfg.get("metric", METRIC), "value": cb["value"], "unit": "Mparticles/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": cb["seconds_per_solve"] * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64)",
                "config": base_config(cfg, 1),
                "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": cb["value"], "unit": "Mparticles/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    r = run_ours(args, cfg, rank, world, local_rank)
    torch, dist = r["torch"], r["dist"]
    line = None
    if rank == 0:
        peaks = measured_peaks()
        fp64 = fp64_peak_tflops(torch)
        fp32 = fp32_peak_tflops(torch)
        tf32 = tf32_peak_tflops(torch)
        stats = r["stats"]
        radix_passes = (cfg["dim"] * (cfg["depth"] - 1) + 7) // 8
        line = {
            "metric": cfg.get("metric", METRIC), "value": aggregate_rate(cfg["n"], world, r["ms"]), "unit": "Mparticles/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if cfg["precision"] == "fp64" else "f32/tf32", "data": "synthetic (seeded PCG64)",
            "config": base_config(cfg, world), "accuracy": r["acc"], "phases_ms": {
                k: stats[k] for k in ("ms_tree", "ms_upward", "ms_m2l", "ms_l2l", "ms_leaves", "ms_total",
                                      "ms_m2l_kernel")},
            "tree": {k: stats[k] for k in ("n_cells", "n_leaves", "n_far_pairs", "n_close_pairs", "n_p2p_pairs",
                                           "n_m2p", "n_w", "n_x")},
            "roofline": roofline(cfg, stats, peaks, fp64, fp32, tf32),
            "roofline_leaves": roofline(cfg, stats, peaks, fp64, fp32, tf32, phase="leaves"),
            "fp64_peak_tflops_measured": fp64, "fp32_peak_tflops_measured": fp32, "tf32_peak_tflops_measured": tf32,
            "peaks_source": peaks["source"], "e2e": r["e2e"], "clocks": r["clocks"],
            "gpu_launches": args.steps * launches_per_solve(stats["depth"], cfg["dim"], radix_passes,
                                                            cfg.get("max_leaf", 0) > 0, cfg["precision"],
                                                            learned=bool(r["learned"])),
        }
        if r["learned"]:
            line["learned_order"] = dict(r["learned"], tol=cfg["tol"], check_targets=cfg["check_targets"])
            line["config"]["N_degrees"] = r["learned"]["order_N"]
            line["config"]["order_p"] = r["learned"]["order_N"] - 1
            line["config"]["plain_fp64_N_degrees"] = cfg["N"]
        if r["plan"]:
            line["plan_execute"] = r["plan"]
        if r.get("mixed_fixed"):
            line["mixed_fixed"] = r["mixed_fixed"]
            line["speedup_vs_mixed_fixed"] = r["mixed_fixed"]["ms_per_step"] / r["ms"]
        if r["plain"]:
            if cfg["dim"] == 2:
                line["uniform_tree"] = r["plain"]
                line["speedup_vs_uniform_tree"] = r["plain"]["ms_per_step"] / r["ms"]
            else:
                line["plain_fp64"] = r["plain"]
                line["speedup_vs_plain_fp64"] = r["plain"]["ms_per_step"] / r["ms"]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if not args.no_cpu_baseline:
            pos, q = make_particles(cfg)
            cb = run_cpu(cfg, pos, q, 2)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
