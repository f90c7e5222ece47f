"""ctypes bindings for the two CPU checkers.  TEST INFRASTRUCTURE.

* ``Oracle`` -- the C restatement of the reference FMM (oracle/*.c, built by
  ``make -C oracle oracle`` into ``oracle/_build/libfmm_oracle.so``).
* ``Reference`` -- the reference's own CPU FMM compiled from its sources
  (``make -C oracle ref`` into ``oracle/_ref/libfmmref.so``), present only
  where the reference sources were available at build time.

Only tests/, ``__graft_entry__.smoke()``, the fixture generator and bench.py's
CPU legs import this module: it is the checker and the CPU baseline, never the
thing measured on the GPU.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libfmm_oracle.so"
REF_SO = HERE / "_ref" / "libfmmref.so"
REF_GPU_SO = HERE / "_ref" / "libfmmref_gpu.so"
AUTO = 2**31 - 1  # the reference's FMM_AUTO (std::numeric_limits<int>::max())

_P = ctypes.c_void_p
_SZ = ctypes.c_size_t
_I = ctypes.c_int
_D = ctypes.c_double


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _f64(a, shape_last=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a


def build(which=("oracle",)):
    """Compile the checkers (``make -C oracle <targets>``)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", str(HERE), *which], check=True)


class Oracle:
    """The C restatement (FP64), with the tree exposed for the integer tests."""

    def __init__(self, path: Path = ORACLE_SO):
        if not Path(path).exists():
            build(("oracle",))
        L = ctypes.CDLL(str(path))
        self.lib = L
        L.orc_fmm3d.argtypes = [_SZ, _P, _P, _SZ, _P, _I, _I, _D, _P, _P]
        L.orc_fmm2d.argtypes = [_SZ, _P, _P, _SZ, _P, _I, _I, _D, _P, _P]
        L.orc_fmm3d_run.argtypes = [_SZ, _P, _P, _SZ, _P, _I, _I, _D, _P, _P, ctypes.POINTER(_I)]
        L.orc_fmm3d_run.restype = _P
        L.orc_fmm2d_run.argtypes = [_SZ, _P, _P, _SZ, _P, _I, _I, _D, _P, _P, ctypes.POINTER(_I)]
        L.orc_fmm2d_run.restype = _P
        L.orc_run_free.argtypes = [_P]
        L.orc_run_expansions.argtypes = [_P, _I, _P, _P]
        L.orc_run_order.argtypes = [_P]
        L.orc_run_depth.argtypes = [_P]
        L.orc_direct3d.argtypes = [_SZ, _P, _P, _SZ, _P, _P, _P]
        L.orc_direct2d.argtypes = [_SZ, _P, _P, _SZ, _P, _P, _P]
        L.orc_wignerd.argtypes = [_I, _D, _P]
        L.orc_op3d.argtypes = [_I, _I, _P, _D, _D, _D, _P]
        L.orc_table_angles.argtypes = [_D, _D, ctypes.POINTER(_D), ctypes.POINTER(_D)]
        L.orc_direction_key_counts.argtypes = [ctypes.POINTER(_I)] * 3
        L.orc_tree_create.argtypes = [_I, _SZ, _P, _P, _I]
        L.orc_tree_create.restype = _P
        L.orc_tree_destroy.argtypes = [_P]
        L.orc_tree_level_size.argtypes = [_P, _I]
        L.orc_tree_level_size.restype = _SZ
        L.orc_tree_targets_num.argtypes = [_P]
        L.orc_tree_targets_num.restype = _SZ
        L.orc_tree_geometry.argtypes = [_P, _P, _P]
        L.orc_tree_cells.argtypes = [_P, _I, _P, _P, _P, _P, _P, _P, _P]
        L.orc_tree_list_counts.argtypes = [_P, _I, _I, _P, _P]
        L.orc_tree_lists.argtypes = [_P, _I, _I, _P, _P]
        L.orc_tree_positions.argtypes = [_P, _P]
        L.orc_tree_particles.argtypes = [_P, _P, _P]
        L.orc_set_threads.argtypes = [_I]

    def set_threads(self, n: int):
        self.lib.orc_set_threads(int(n))

    # ---- full solves -------------------------------------------------
    def fmm3d(self, src, q, targets=None, N=AUTO, depth=AUTO, eps=1e-8):
        src = _f64(src).reshape(-1, 3); q = _f64(q)
        nt = 0 if targets is None else len(targets)
        tgt = None if targets is None else _f64(targets).reshape(-1, 3)
        nout = nt if nt else len(src)
        pot = np.zeros(nout); fld = np.zeros((nout, 3))
        st = self.lib.orc_fmm3d(len(src), _ptr(src), _ptr(q), nt, _ptr(tgt), int(N), int(depth), float(eps),
                                _ptr(pot), _ptr(fld))
        if st:
            raise RuntimeError(f"oracle fmm3d failed with status {st}")
        return pot, fld

    def fmm3d_vec(self, src, q3, targets=None, N=AUTO, depth=AUTO, eps=1e-8):
        """Vector charges (reference FastMultipole3d<Vector3d>,
        cpu/multipole3d.cpp:414-853): the field sum q x d / r^3 written as
        e_x x E^(x) + e_y x E^(y) + e_z x E^(z), E^(c) the field of this
        oracle's scalar FMM for the charges' component c (the reference sums
        the same cross products pairwise in the near field and from its three
        expansions' gradients in the far field).  Each particle's charge must
        be zero in all components or in none, so that the three scalar solves
        split sources and targets alike (the reference's zero rule)."""
        q3 = _f64(q3).reshape(-1, 3)
        z = q3 == 0
        if np.any(z.any(axis=1) != z.all(axis=1)):
            raise ValueError("a charge with some zero components: the scalar solves would split it differently")
        E = [self.fmm3d(src, np.ascontiguousarray(q3[:, c]), targets, N, depth, eps)[1] for c in range(3)]
        return np.stack([E[1][:, 2] - E[2][:, 1], E[2][:, 0] - E[0][:, 2], E[0][:, 1] - E[1][:, 0]], axis=1)

    def fmm2d(self, src, q, targets=None, N=AUTO, depth=AUTO, eps=1e-8):
        src = _f64(src).reshape(-1, 2); q = _f64(q)
        nt = 0 if targets is None else len(targets)
        tgt = None if targets is None else _f64(targets).reshape(-1, 2)
        nout = nt if nt else len(src)
        pot = np.zeros(nout); fld = np.zeros((nout, 2))
        st = self.lib.orc_fmm2d(len(src), _ptr(src), _ptr(q), nt, _ptr(tgt), int(N), int(depth), float(eps),
                                _ptr(pot), _ptr(fld))
        if st:
            raise RuntimeError(f"oracle fmm2d failed with status {st}")
        return pot, fld

    def run3d(self, src, q, targets=None, N=AUTO, depth=AUTO, eps=1e-8):
        """Solve and keep the per-level expansions: returns (pot, field, outer, inner)
        with outer[L], inner[L] complex arrays of shape (cells, ncoef)."""
        return self._run(3, src, q, targets, N, depth, eps)

    def run2d(self, src, q, targets=None, N=AUTO, depth=AUTO, eps=1e-8):
        return self._run(2, src, q, targets, N, depth, eps)

    def _run(self, dim, src, q, targets, N, depth, eps):
        src = _f64(src).reshape(-1, dim); q = _f64(q)
        nt = 0 if targets is None else len(targets)
        tgt = None if targets is None else _f64(targets).reshape(-1, dim)
        nout = nt if nt else len(src)
        pot = np.zeros(nout); fld = np.zeros((nout, dim))
        st = _I(0)
        fn = self.lib.orc_fmm3d_run if dim == 3 else self.lib.orc_fmm2d_run
        h = fn(len(src), _ptr(src), _ptr(q), nt, _ptr(tgt), int(N), int(depth), float(eps), _ptr(pot), _ptr(fld),
               ctypes.byref(st))
        if st.value or not h:
            raise RuntimeError(f"oracle run failed with status {st.value}")
        try:
            D = self.lib.orc_run_depth(h)
            outer, inner = [], []
            for L in range(D):
                m = self.lib.orc_tree_level_size(h, L)
                nc = dim == 3 and (lambda N_: N_ * (N_ + 1) // 2)(self.lib.orc_run_order(h)) or self.lib.orc_run_order(h)
                o = np.zeros(m * nc * 2); i_ = np.zeros(m * nc * 2)
                self.lib.orc_run_expansions(h, L, _ptr(o), _ptr(i_))
                outer.append(o.view(np.complex128).reshape(m, nc))
                inner.append(i_.view(np.complex128).reshape(m, nc))
        finally:
            self.lib.orc_run_free(h)
        return pot, fld, outer, inner

    # ---- direct sums -------------------------------------------------
    def direct3d(self, src, q, targets):
        src = _f64(src).reshape(-1, 3); q = _f64(q); tgt = _f64(targets).reshape(-1, 3)
        pot = np.zeros(len(tgt)); fld = np.zeros((len(tgt), 3))
        self.lib.orc_direct3d(len(src), _ptr(src), _ptr(q), len(tgt), _ptr(tgt), _ptr(pot), _ptr(fld))
        return pot, fld

    def direct2d(self, src, q, targets):
        src = _f64(src).reshape(-1, 2); q = _f64(q); tgt = _f64(targets).reshape(-1, 2)
        pot = np.zeros(len(tgt)); fld = np.zeros((len(tgt), 2))
        self.lib.orc_direct2d(len(src), _ptr(src), _ptr(q), len(tgt), _ptr(tgt), _ptr(pot), _ptr(fld))
        return pot, fld

    # ---- special functions -------------------------------------------
    def wignerd(self, N, theta):
        out = np.zeros(N * (N + 1) * (4 * N - 1) // 6)
        self.lib.orc_wignerd(int(N), float(theta), _ptr(out))
        return out

    def op3d(self, op, N, a, p0):
        """op: 0 = M2M, 1 = M2L, 2 = L2L; a complex (Nx2,), p0 displacement."""
        a = np.ascontiguousarray(a, dtype=np.complex128)
        b = np.zeros_like(a)
        st = self.lib.orc_op3d(int(op), int(N), _ptr(a), float(p0[0]), float(p0[1]), float(p0[2]), _ptr(b))
        if st:
            raise RuntimeError("angle outside the reference's direction tables")
        return b

    def table_angles(self, theta, phi):
        a, b = _D(), _D()
        st = self.lib.orc_table_angles(float(theta), float(phi), ctypes.byref(a), ctypes.byref(b))
        return st, a.value, b.value

    def direction_key_counts(self):
        a, b, c = _I(), _I(), _I()
        self.lib.orc_direction_key_counts(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    # ---- tree ----------------------------------------------------------
    def tree(self, dim, pts, q, depth, halved=None):
        pts = _f64(pts).reshape(-1, dim); q = _f64(q)
        h = self.lib.orc_tree_create(dim, len(pts), _ptr(pts), _ptr(q), int(depth))
        if not h:
            raise RuntimeError("oracle tree build failed")
        try:
            return _export_tree(self.lib, "orc_tree_", h, dim, depth, len(pts), halved)
        finally:
            self.lib.orc_tree_destroy(h)


def _export_tree(L, prefix, h, dim, depth, n, halved):
    """Read a tree handle into numpy arrays (shared by both checkers)."""
    g = lambda name: getattr(L, prefix + name)
    targets_num = g("targets_num")(h)
    if halved is None:
        halved = targets_num == 0
    levels = []
    for lvl in range(depth):
        m = g("level_size")(h, lvl)
        code = np.zeros(m, np.uint64)
        sb, se, tb, te, par = (np.zeros(m, np.int64) for _ in range(5))
        cen = np.zeros((m, dim))
        g("cells")(h, lvl, _ptr(code), _ptr(sb), _ptr(se), _ptr(tb), _ptr(te), _ptr(par), _ptr(cen))
        nc = np.zeros(m, np.int64); nf = np.zeros(m, np.int64)
        leaf = lvl == depth - 1
        if prefix == "orc_tree_":
            g("list_counts")(h, lvl, int(halved and leaf), _ptr(nc), _ptr(nf))
            close = np.zeros(int(nc.sum()), np.int64); far = np.zeros(int(nf.sum()), np.int64)
            g("lists")(h, lvl, int(halved and leaf), _ptr(close), _ptr(far))
        else:
            g("list_counts")(h, lvl, _ptr(nc), _ptr(nf))
            close = np.zeros(int(nc.sum()), np.int64); far = np.zeros(int(nf.sum()), np.int64)
            g("lists")(h, lvl, _ptr(close), _ptr(far))
        levels.append(dict(code=code, sb=sb, se=se, tb=tb, te=te, parent=par, center=cen,
                           close_off=np.concatenate([[0], np.cumsum(nc)]), close=close,
                           far_off=np.concatenate([[0], np.cumsum(nf)]), far=far))
    pos = np.zeros(n, np.int64)
    g("positions")(h, _ptr(pos))
    return dict(levels=levels, positions=pos, targets_num=targets_num)


class Reference:
    """The reference's own CPU FMM (unmodified sources), for pinning the oracle
    and as the CPU baseline."""

    def __init__(self, path: Path = REF_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built (needs the reference sources; make -C oracle ref)")
        L = ctypes.CDLL(str(path))
        self.lib = L
        L.ref_fmm3d.argtypes = [_SZ, _P, _P, _I, _I, _D, _P, _P]
        L.ref_fmm3d_st.argtypes = [_SZ, _P, _P, _SZ, _P, _I, _I, _D, _P, _P]
        L.ref_fmm3d_vec.argtypes = [_SZ, _P, _P, _I, _I, _D, _P]
        L.ref_fmm3d_vec_st.argtypes = [_SZ, _P, _P, _SZ, _P, _I, _I, _D, _P]
        L.ref_fmm2d.argtypes = [_SZ, _P, _P, _I, _I, _D, _P, _P]
        L.ref_fmm2d_st.argtypes = [_SZ, _P, _P, _SZ, _P, _I, _I, _D, _P, _P]
        L.ref_wignerd.argtypes = [_I, _D, _P]
        L.ref_set_threads.argtypes = [_I]
        for d in ("3d", "2d"):
            getattr(L, f"ref_tree{d}_build").argtypes = [_SZ, _P, _P, _I]
            getattr(L, f"ref_tree{d}_build").restype = _P
            getattr(L, f"ref_tree{d}_free").argtypes = [_P]
            getattr(L, f"ref_tree{d}_level_size").argtypes = [_P, _I]
            getattr(L, f"ref_tree{d}_level_size").restype = _SZ
            getattr(L, f"ref_tree{d}_targets_num").argtypes = [_P]
            getattr(L, f"ref_tree{d}_targets_num").restype = _SZ
            getattr(L, f"ref_tree{d}_cells").argtypes = [_P, _I, _P, _P, _P, _P, _P, _P, _P]
            getattr(L, f"ref_tree{d}_list_counts").argtypes = [_P, _I, _P, _P]
            getattr(L, f"ref_tree{d}_lists").argtypes = [_P, _I, _P, _P]
            getattr(L, f"ref_tree{d}_positions").argtypes = [_P, _P]

    def set_threads(self, n: int):
        self.lib.ref_set_threads(int(n))

    def fmm3d(self, src, q, targets=None, N=AUTO, depth=AUTO, eps=1e-8):
        src = _f64(src).reshape(-1, 3); q = _f64(q)
        if targets is None:
            pot = np.zeros(len(src)); fld = np.zeros((len(src), 3))
            self.lib.ref_fmm3d(len(src), _ptr(src), _ptr(q), int(N), int(depth), float(eps), _ptr(pot), _ptr(fld))
        else:
            tgt = _f64(targets).reshape(-1, 3)
            pot = np.zeros(len(tgt)); fld = np.zeros((len(tgt), 3))
            self.lib.ref_fmm3d_st(len(src), _ptr(src), _ptr(q), len(tgt), _ptr(tgt), int(N), int(depth), float(eps),
                                  _ptr(pot), _ptr(fld))
        return pot, fld

    def fmm3d_vec(self, src, q3, targets=None, N=AUTO, depth=AUTO, eps=1e-8):
        src = _f64(src).reshape(-1, 3); q3 = _f64(q3).reshape(-1, 3)
        if targets is None:
            fld = np.zeros((len(src), 3))
            self.lib.ref_fmm3d_vec(len(src), _ptr(src), _ptr(q3), int(N), int(depth), float(eps), _ptr(fld))
        else:
            tgt = _f64(targets).reshape(-1, 3)
            fld = np.zeros((len(tgt), 3))
            self.lib.ref_fmm3d_vec_st(len(src), _ptr(src), _ptr(q3), len(tgt), _ptr(tgt), int(N), int(depth),
                                      float(eps), _ptr(fld))
        return fld

    def fmm2d(self, src, q, targets=None, N=AUTO, depth=AUTO, eps=1e-8):
        src = _f64(src).reshape(-1, 2); q = _f64(q)
        if targets is None:
            pot = np.zeros(len(src)); fld = np.zeros((len(src), 2))
            self.lib.ref_fmm2d(len(src), _ptr(src), _ptr(q), int(N), int(depth), float(eps), _ptr(pot), _ptr(fld))
        else:
            tgt = _f64(targets).reshape(-1, 2)
            pot = np.zeros(len(tgt)); fld = np.zeros((len(tgt), 2))
            self.lib.ref_fmm2d_st(len(src), _ptr(src), _ptr(q), len(tgt), _ptr(tgt), int(N), int(depth), float(eps),
                                  _ptr(pot), _ptr(fld))
        return pot, fld

    def wignerd(self, N, theta):
        out = np.zeros(N * (N + 1) * (4 * N - 1) // 6)
        self.lib.ref_wignerd(int(N), float(theta), _ptr(out))
        return out

    def tree(self, dim, pts, q, depth):
        pts = _f64(pts).reshape(-1, dim); q = _f64(q)
        d = f"{dim}d"
        h = getattr(self.lib, f"ref_tree{d}_build")(len(pts), _ptr(pts), _ptr(q), int(depth))
        try:
            return _export_tree(self.lib, f"ref_tree{d}_", h, dim, depth, len(pts), None)
        finally:
            getattr(self.lib, f"ref_tree{d}_free")(h)


class ReferenceGPU:
    """The reference's own CUDA FMM (unmodified sources, built for sm_100a by
    ``make -C oracle ref-gpu``; allocations zero-filled by the link, see
    ref_gpu_wrapper.cu).  Timed as a comparison point; its outputs are not a
    parity oracle (its M2L sums uninitialised work arrays)."""

    def __init__(self, path: Path = REF_GPU_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built (needs the reference sources; make -C oracle ref-gpu)")
        L = ctypes.CDLL(str(path))
        self.lib = L
        for f in ("ref_gpu_fmm3d", "ref_gpu_fmm2d"):
            getattr(L, f).argtypes = [_SZ, _P, _P, _I, _I, _D, _P, _P, _P]
            getattr(L, f).restype = _I
        L.ref_gpu_set_verbose.argtypes = [_I]

    def _solve(self, fn, dim, src, q, N, depth, eps):
        src = _f64(src).reshape(-1, dim); q = _f64(q)
        pot = np.zeros(len(src)); fld = np.zeros((len(src), dim)); sec = np.zeros(1)
        rc = fn(len(src), _ptr(src), _ptr(q), int(N), int(depth), float(eps), _ptr(pot), _ptr(fld), _ptr(sec))
        if rc != 0:
            raise RuntimeError(f"reference GPU solve failed (status {rc})")
        return pot, fld, float(sec[0])

    def fmm3d(self, src, q, N=AUTO, depth=AUTO, eps=1e-8):
        """(potential, field, seconds of the reference's constructor)"""
        return self._solve(self.lib.ref_gpu_fmm3d, 3, src, q, N, depth, eps)

    def fmm2d(self, src, q, N=AUTO, depth=AUTO, eps=1e-8):
        return self._solve(self.lib.ref_gpu_fmm2d, 2, src, q, N, depth, eps)


def rel_l2(x, ref):
    x = np.asarray(x); ref = np.asarray(ref)
    return float(np.linalg.norm((x - ref).ravel()) / np.linalg.norm(ref.ravel()))
