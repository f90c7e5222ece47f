"""Host-side mirror of the reference's solver interface, over the C ABI.

Names, argument meaning and results follow the reference's classes:

* ``FastMultipole3d(particles, eps=1e-8, N=FMM_AUTO, tree_depth=FMM_AUTO)`` and
  ``FastMultipole3d(sources, targets, ...)`` -- reference
  ``fmm::gpu::FastMultipole3d<double>`` (cuda/multipole3d.h:16-17) and its CPU
  twin (cpu/multipole3d.h:19-21).  Results in ``.potentials`` (n,) and
  ``.forces`` (n, 3), input order; targets must carry q = 0.
* ``FastMultipole(...)`` -- reference ``fmm::gpu::FastMultipole``
  (cuda/multipole.h:11-12): 2D, ``.forces`` complex (n,).
* ``compute_exact(kind, sources, targets=None)`` -- reference
  ``fmm::gpu::ComputeExact<kind>`` (common/simple_math.h:283-313) without the
  text file: returns the direct-sum values.
* ``init_math_constants`` / ``cuda_copy_math_constants`` /
  ``cuda_clear_math_constants`` -- the reference's process-global table set-up
  (common/special_functions.h:154-156); here the tables live in each context,
  so these are no-ops kept for call compatibility.

Particles are accepted as ``(positions, charges)`` pairs or as numpy
structured arrays with the reference's particle layout (``particle3d_dtype``:
centre xyz, q, morton_code = 40 bytes; ``particle2d_dtype``: 32 bytes).
"""
from __future__ import annotations

import ctypes
from enum import Enum

import numpy as np

from ._lib import AUTO, PRECISION, Context, LfmmSolveOpts, LfmmStats, default_context

FMM_AUTO = AUTO
FORCE_EPS = 1.0e-4

particle3d_dtype = np.dtype([("center", "<f8", (3,)), ("q", "<f8"), ("morton_code", "<u8")])
particle2d_dtype = np.dtype([("center", "<c16"), ("q", "<f8"), ("morton_code", "<u8")])


class InteractionType(Enum):
    """Reference common/utils.h:17-23."""
    Potential2d = 0
    Force2d = 1
    Potential3d = 2
    Force3d = 3


def _split(particles, dim):
    """(positions (n, dim) float64 C-contiguous, charges (n,) float64; vector
    charges of a 3D solve stay (n, 3))."""
    if isinstance(particles, np.ndarray) and particles.dtype.names:
        c = particles["center"]
        if dim == 2 and np.iscomplexobj(c):
            pos = np.stack([c.real, c.imag], axis=1)
        else:
            pos = np.asarray(c, dtype=np.float64).reshape(-1, dim)
        q = np.asarray(particles["q"], dtype=np.float64)
        if not (dim == 3 and q.ndim == 2 and q.shape[1] == 3):
            q = q.reshape(-1)
    else:
        pos, q = particles
        pos = np.asarray(pos)
        if dim == 2 and np.iscomplexobj(pos):
            pos = np.stack([pos.real, pos.imag], axis=1)
        pos = pos.reshape(-1, dim)
        q = np.asarray(q, dtype=np.float64)
        if not (dim == 3 and q.ndim == 2 and q.shape[1] == 3):
            q = q.reshape(-1)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    if len(pos) != len(q):
        raise ValueError("positions and charges differ in length")
    return pos, q


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None and a.size else None


class _Solver:
    dim = 3

    def __init__(self, *args, eps: float = 1.0e-8, N: int = FMM_AUTO, tree_depth: int = FMM_AUTO,
                 precision: str = "fp64", max_leaf: int = 0, level_orders=None, ctx: Context | None = None):
        # reference overloads: (particles, eps, N, depth) and (sources, targets, eps, N, depth)
        args = list(args)
        if not args:
            raise TypeError("particles required")
        sources = args.pop(0)
        targets = None
        if args and not isinstance(args[0], (int, float)):
            targets = args.pop(0)
        if args:
            eps = args.pop(0)
        if args:
            N = args.pop(0)
        if args:
            tree_depth = args.pop(0)
        ctx = ctx or default_context()
        dim = self.dim
        spos, sq = _split(sources, dim)
        tpos = None
        if targets is not None:
            tpos, tq = _split(targets, dim) if not isinstance(targets, np.ndarray) or targets.dtype.names \
                else (np.ascontiguousarray(np.asarray(targets, dtype=np.float64).reshape(-1, dim)), None)
        nt = 0 if tpos is None else len(tpos)
        nout = nt if nt else len(spos)
        pot = np.zeros(nout)
        fld = np.zeros((nout, dim))
        stats = LfmmStats()
        if sq.ndim == 2:
            # vector charges (reference FastMultipole3d<Vector3d>): field only
            opts = LfmmSolveOpts(int(N), int(tree_depth), int(max_leaf), PRECISION[precision], float(eps))
            ctx.check(ctx.lib.lfmm3d_solve_vector(ctx.handle, len(spos), _ptr(spos), _ptr(sq), nt, _ptr(tpos),
                                                  ctypes.byref(opts), _ptr(fld), ctypes.byref(stats)),
                      "lfmm3d_solve_vector")
            self.potentials = np.zeros(0)
            self.forces = fld
            self.stats = stats.as_dict()
            self.N = stats.order_N
            self.tree_depth = stats.depth
            return
        if level_orders is not None and dim == 3:
            # per-level M2L orders (degrees of the sources each level's M2L uses)
            opts = LfmmSolveOpts(int(N), int(tree_depth), int(max_leaf), PRECISION[precision], float(eps))
            lv = (ctypes.c_int * max(1, len(level_orders)))(*[int(v) for v in level_orders])
            st = ctx.lib.lfmm3d_solve_levels(ctx.handle, len(spos), _ptr(spos), _ptr(sq), nt, _ptr(tpos),
                                             ctypes.byref(opts), lv, len(level_orders), _ptr(pot), _ptr(fld),
                                             ctypes.byref(stats))
        elif max_leaf:
            opts = LfmmSolveOpts(int(N), int(tree_depth), int(max_leaf), PRECISION[precision], float(eps))
            fn = ctx.lib.lfmm3d_solve_ex if dim == 3 else ctx.lib.lfmm2d_solve_ex
            st = fn(ctx.handle, len(spos), _ptr(spos), _ptr(sq), nt, _ptr(tpos), ctypes.byref(opts), _ptr(pot),
                    _ptr(fld), ctypes.byref(stats))
        else:
            fn = ctx.lib.lfmm3d_solve if dim == 3 else ctx.lib.lfmm2d_solve
            st = fn(ctx.handle, len(spos), _ptr(spos), _ptr(sq), nt, _ptr(tpos), int(N), int(tree_depth),
                    float(eps), PRECISION[precision], _ptr(pot), _ptr(fld), ctypes.byref(stats))
        ctx.check(st, f"lfmm{dim}d_solve")
        self.potentials = pot
        self.forces = fld if dim == 3 else fld[:, 0] + 1j * fld[:, 1]
        self.stats = stats.as_dict()
        self.N = stats.order_N
        self.tree_depth = stats.depth


class FastMultipole3d(_Solver):
    """3D rotation-based Laplace FMM (reference fmm::gpu::FastMultipole3d<double>;
    with charges of shape (n, 3), fmm::FastMultipole3d<Vector3d>: forces =
    sum q x d / r^3, no potentials)."""
    dim = 3


class FastMultipole(_Solver):
    """2D complex Laplace FMM (reference fmm::gpu::FastMultipole)."""
    dim = 2


def compute_exact(kind: InteractionType, sources, targets=None, ctx: Context | None = None):
    """FP64 direct sum on the GPU; returns potentials (n,) or fields."""
    ctx = ctx or default_context()
    dim = 3 if kind in (InteractionType.Potential3d, InteractionType.Force3d) else 2
    spos, sq = _split(sources, dim)
    if targets is None:
        tpos = spos
    elif isinstance(targets, np.ndarray) and targets.dtype.names:
        tpos = _split(targets, dim)[0]
    else:
        tpos = np.ascontiguousarray(np.asarray(targets, dtype=np.float64).reshape(-1, dim))
    pot = np.zeros(len(tpos))
    fld = np.zeros((len(tpos), dim))
    fn = ctx.lib.lfmm3d_direct if dim == 3 else ctx.lib.lfmm2d_direct
    ctx.check(fn(ctx.handle, len(spos), _ptr(spos), _ptr(sq), len(tpos), _ptr(tpos), _ptr(pot), _ptr(fld)),
              "direct")
    if kind in (InteractionType.Potential2d, InteractionType.Potential3d):
        return pot
    return fld if dim == 3 else fld[:, 0] + 1j * fld[:, 1]


def init_math_constants(N: int = 18):
    """Reference fmm::detail::InitMathConstants: tables are per context here."""
    return None


def cuda_copy_math_constants():
    return None


def cuda_clear_math_constants():
    return None


def solve_batch(problems, N: int = FMM_AUTO, tree_depth: int = FMM_AUTO, max_leaf: int = 64,
                precision: str = "mixed", eps: float = 1.0e-8, ctx: Context | None = None):
    """Independent 3D problems [(positions, charges), ...] solved together
    (one forest of octrees, one launch per FMM pass); returns
    [(potentials, forces), ...] in the same order."""
    ctx = ctx or default_context()
    parts = [_split(p, 3) for p in problems]
    offs = np.zeros(len(parts) + 1, dtype=np.uint64)
    offs[1:] = np.cumsum([len(p[0]) for p in parts])
    pos = np.ascontiguousarray(np.concatenate([p[0] for p in parts]))
    q = np.ascontiguousarray(np.concatenate([p[1] for p in parts]))
    n = len(pos)
    pot = np.zeros(n)
    fld = np.zeros((n, 3))
    opts = LfmmSolveOpts(int(N), int(tree_depth), int(max_leaf), PRECISION[precision], float(eps))
    stats = LfmmStats()
    ctx.check(ctx.lib.lfmm3d_solve_batch(ctx.handle, len(parts), offs.ctypes.data_as(ctypes.c_void_p), _ptr(pos),
                                         _ptr(q), ctypes.byref(opts), _ptr(pot), _ptr(fld), ctypes.byref(stats)),
              "lfmm3d_solve_batch")
    return [(pot[offs[k]:offs[k + 1]], fld[offs[k]:offs[k + 1]]) for k in range(len(parts))]


class Plan3d:
    """One geometry, many charge vectors: the adaptive tree of the positions
    and a CUDA graph of the FMM passes are built once; ``execute(charges)``
    replays the graph (lfmm3d_plan_create / lfmm3d_plan_execute).  The
    charges given at creation fix the tree's split into sources and zero-charge
    targets; later charges only change values."""

    def __init__(self, positions, charges, N: int, tree_depth: int = FMM_AUTO, max_leaf: int = 64,
                 precision: str = "mixed", ctx: Context | None = None):
        import torch
        self.ctx = ctx or default_context()
        pos, q = _split((positions, charges), 3)
        self.n = len(pos)
        dev = torch.device("cuda", self.ctx.device)
        self._torch, self._dev = torch, dev
        d_pos = torch.from_numpy(pos).to(dev)
        self._q = torch.from_numpy(q).to(dev)
        self._pot = torch.empty(self.n, dtype=torch.float64, device=dev)
        self._fld = torch.empty(self.n, 3, dtype=torch.float64, device=dev)
        opts = LfmmSolveOpts(int(N), int(tree_depth), int(max_leaf), PRECISION[precision], 1e-8)
        self.handle = ctypes.c_void_p()
        torch.cuda.synchronize(dev)
        vp = ctypes.c_void_p
        self.ctx.check(self.ctx.lib.lfmm3d_plan_create(self.ctx.handle, self.n, vp(d_pos.data_ptr()),
                                                       vp(self._q.data_ptr()), ctypes.byref(opts),
                                                       ctypes.byref(self.handle)), "lfmm3d_plan_create")

    def execute(self, charges):
        """(potentials, forces) for new charges at the plan's positions."""
        torch = self._torch
        q = np.ascontiguousarray(np.asarray(charges, dtype=np.float64).reshape(-1))
        if len(q) != self.n:
            raise ValueError("charges differ in length from the plan's positions")
        self._q.copy_(torch.from_numpy(q))
        torch.cuda.synchronize(self._dev)
        vp = ctypes.c_void_p
        self.ctx.check(self.ctx.lib.lfmm3d_plan_execute(self.handle, vp(self._q.data_ptr()),
                                                        vp(self._pot.data_ptr()), vp(self._fld.data_ptr())),
                       "lfmm3d_plan_execute")
        torch.cuda.ExternalStream(self.ctx.stream, device=self._dev).synchronize()
        return self._pot.cpu().numpy(), self._fld.cpu().numpy()

    def close(self):
        if self.handle:
            self.ctx.lib.lfmm3d_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchPlan3d(Plan3d):
    """A batch of independent problems solved repeatedly with new charges: the
    forest of their trees and a CUDA graph of the FMM passes over all of them
    are built once (lfmm3d_plan_create_batch); ``execute(charges)`` takes and
    returns the problems' values concatenated in input order."""

    def __init__(self, problems, N: int, tree_depth: int = FMM_AUTO, max_leaf: int = 64, precision: str = "mixed",
                 ctx: Context | None = None):
        import torch
        self.ctx = ctx or default_context()
        parts = [_split((p, c), 3) for p, c in problems]
        self.offsets = np.zeros(len(parts) + 1, dtype=np.uint64)
        self.offsets[1:] = np.cumsum([len(p) for p, _ in parts])
        pos = np.ascontiguousarray(np.concatenate([p for p, _ in parts]))
        q = np.ascontiguousarray(np.concatenate([c for _, c in parts]))
        self.n = len(pos)
        dev = torch.device("cuda", self.ctx.device)
        self._torch, self._dev = torch, dev
        d_pos = torch.from_numpy(pos).to(dev)
        self._q = torch.from_numpy(q).to(dev)
        self._pot = torch.empty(self.n, dtype=torch.float64, device=dev)
        self._fld = torch.empty(self.n, 3, dtype=torch.float64, device=dev)
        opts = LfmmSolveOpts(int(N), int(tree_depth), int(max_leaf), PRECISION[precision], 1e-8)
        self.handle = ctypes.c_void_p()
        torch.cuda.synchronize(dev)
        vp = ctypes.c_void_p
        self.ctx.check(self.ctx.lib.lfmm3d_plan_create_batch(self.ctx.handle, len(parts),
                                                             self.offsets.ctypes.data_as(vp), vp(d_pos.data_ptr()),
                                                             vp(self._q.data_ptr()), ctypes.byref(opts),
                                                             ctypes.byref(self.handle)), "lfmm3d_plan_create_batch")

