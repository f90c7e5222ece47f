"""ctypes binding of ``liblfmm.so`` (the C ABI in ``include/lfmm.h``).

The shared library is the product: every solve runs in its CUDA kernels.
Loading fails loudly when the library is missing; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "liblfmm.so"

AUTO = 2147483647
PRECISION = {"fp64": 0, "mixed": 1}
STATUS = {0: "OK", -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_OOM", -4: "ERR_DEVICE", -5: "ERR_UNSUPPORTED"}

# Every symbol include/lfmm.h declares (checked by the CPU tests).
EXPORTS = [
    "lfmm_create", "lfmm_destroy", "lfmm_last_error", "lfmm_version", "lfmm_stream", "lfmm_check",
    "lfmm_debug_raise_flags",
    "lfmm3d_solve", "lfmm3d_solve_device", "lfmm3d_solve_ex", "lfmm3d_solve_ex_device",
    "lfmm3d_solve_levels", "lfmm3d_solve_levels_device",
    "lfmm3d_solve_vector", "lfmm3d_solve_vector_device",
    "lfmm2d_solve", "lfmm2d_solve_device", "lfmm2d_solve_ex", "lfmm2d_solve_ex_device",
    "lfmm3d_direct", "lfmm3d_direct_device", "lfmm2d_direct", "lfmm2d_direct_device",
    "lfmm3d_direct_device_noalloc",
    "lfmm_tree_build", "lfmm_tree_level", "lfmm_tree_list_sizes", "lfmm_tree_lists", "lfmm_tree_positions",
    "lfmm_tree_build_adaptive", "lfmm2d_tree_build_adaptive", "lfmm_tree_adaptive_cells",
    "lfmm_tree_adaptive_lists",
    "lfmm_wignerd_slot",
    "lfmm_mlp_forward", "lfmm_mlp_grad", "lfmm_mlp_adam",
    "lfmm3d_features", "lfmm3d_leaf_features", "lfmm3d_solve_learned", "lfmm3d_solve_learned_device",
    "lfmm3d_solve_batch", "lfmm3d_solve_batch_device", "lfmm3d_solve_batch_learned_device",
    "lfmm3d_plan_create", "lfmm3d_plan_create_batch", "lfmm3d_plan_execute", "lfmm3d_plan_destroy",
]


class LfmmOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("verbose", ctypes.c_int), ("timing", ctypes.c_int)]


class LfmmStats(ctypes.Structure):
    _fields_ = [
        ("order_N", ctypes.c_int), ("depth", ctypes.c_int),
        ("n_particles", ctypes.c_size_t), ("n_cells", ctypes.c_size_t), ("n_leaves", ctypes.c_size_t),
        ("targets_num", ctypes.c_size_t), ("n_far_pairs", ctypes.c_size_t), ("n_close_pairs", ctypes.c_size_t),
        ("n_p2p_pairs", ctypes.c_size_t), ("n_m2p", ctypes.c_size_t), ("n_w", ctypes.c_size_t),
        ("n_x", ctypes.c_size_t),
        ("ms_tree", ctypes.c_float), ("ms_upward", ctypes.c_float), ("ms_m2l", ctypes.c_float),
        ("ms_l2l", ctypes.c_float), ("ms_leaves", ctypes.c_float), ("ms_total", ctypes.c_float),
        ("ms_m2l_kernel", ctypes.c_float), ("n_m2l_kernel", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LfmmSolveOpts(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("tree_depth", ctypes.c_int), ("max_leaf", ctypes.c_int),
                ("precision", ctypes.c_int), ("eps", ctypes.c_double)]


class LfmmLearnedInfo(ctypes.Structure):
    _fields_ = [("order_N", ctypes.c_int), ("predicted_N", ctypes.c_int), ("fallback", ctypes.c_int),
                ("predicted_error", ctypes.c_double), ("checked_error", ctypes.c_double),
                ("checked_error_field", ctypes.c_double), ("fp64_resolved", ctypes.c_int),
                ("predicted_error_field", ctypes.c_double), ("judged_error", ctypes.c_double),
                ("max_leaf", ctypes.c_int), ("order_groups", ctypes.c_int),
                ("checked_targets", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LfmmError(RuntimeError):
    pass


_lock = threading.Lock()
_lib = None


def load(path: Path | str = LIB_PATH):
    """Load the library (no GPU needed just to load it)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not Path(path).exists():
            raise LfmmError(f"{path} is not built: run `python -m laplace_fmm_b200.build`")
        L = ctypes.CDLL(str(path))
        P, SZ, I, D = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_double
        L.lfmm_create.argtypes = [ctypes.POINTER(P), ctypes.POINTER(LfmmOptions)]
        L.lfmm_destroy.argtypes = [P]
        L.lfmm_destroy.restype = None
        L.lfmm_last_error.argtypes = [P]
        L.lfmm_last_error.restype = ctypes.c_char_p
        L.lfmm_stream.argtypes = [P]
        L.lfmm_stream.restype = P
        L.lfmm_check.argtypes = [P]
        L.lfmm_debug_raise_flags.argtypes = [P, ctypes.c_uint]
        solve = [P, SZ, P, P, SZ, P, I, I, D, I, P, P, ctypes.POINTER(LfmmStats)]
        for f in ("lfmm3d_solve", "lfmm3d_solve_device", "lfmm2d_solve", "lfmm2d_solve_device"):
            getattr(L, f).argtypes = solve
        for f in ("lfmm3d_solve_ex", "lfmm3d_solve_ex_device", "lfmm2d_solve_ex", "lfmm2d_solve_ex_device"):
            getattr(L, f).argtypes = [P, SZ, P, P, SZ, P, ctypes.POINTER(LfmmSolveOpts), P, P,
                                      ctypes.POINTER(LfmmStats)]
        for f in ("lfmm3d_solve_levels", "lfmm3d_solve_levels_device"):
            getattr(L, f).argtypes = [P, SZ, P, P, SZ, P, ctypes.POINTER(LfmmSolveOpts), P, I, P, P,
                                      ctypes.POINTER(LfmmStats)]
        for f in ("lfmm3d_solve_vector", "lfmm3d_solve_vector_device"):
            getattr(L, f).argtypes = [P, SZ, P, P, SZ, P, ctypes.POINTER(LfmmSolveOpts), P,
                                      ctypes.POINTER(LfmmStats)]
        for f in ("lfmm3d_direct", "lfmm3d_direct_device", "lfmm2d_direct", "lfmm2d_direct_device",
                  "lfmm3d_direct_device_noalloc"):
            getattr(L, f).argtypes = [P, SZ, P, P, SZ, P, P, P]
        L.lfmm_tree_build.argtypes = [P, I, SZ, P, P, SZ, P, I, P, P]
        L.lfmm_tree_level.argtypes = [P, I, P, P, P, P, P, P, P]
        L.lfmm_tree_list_sizes.argtypes = [P, I, P, P]
        L.lfmm_tree_lists.argtypes = [P, I, P, P]
        L.lfmm_tree_positions.argtypes = [P, P]
        L.lfmm3d_leaf_features.argtypes = [P, SZ, P, P, SZ, P, I, I, P, I, P]
        L.lfmm_tree_build_adaptive.argtypes = [P, SZ, P, P, SZ, P, I, I, P, P, P]
        L.lfmm2d_tree_build_adaptive.argtypes = [P, SZ, P, P, SZ, P, I, I, P, P, P]
        L.lfmm_tree_adaptive_cells.argtypes = [P, P, P, P, P, P, P, P, P, P]
        L.lfmm_tree_adaptive_lists.argtypes = [P, I, P, P]
        L.lfmm_wignerd_slot.argtypes = [P, I, ctypes.POINTER(D), P]
        L.lfmm_mlp_forward.argtypes = [P, P, I, P, P]
        L.lfmm_mlp_grad.argtypes = [P, P, I, P, P, P, P, P, ctypes.POINTER(ctypes.c_float)]
        F = ctypes.c_float
        L.lfmm_mlp_adam.argtypes = [P, P, P, P, P, I, F, F, F, F]
        L.lfmm3d_features.argtypes = [P, SZ, P, P, SZ, P, ctypes.POINTER(LfmmSolveOpts), P, SZ, P,
                                      ctypes.POINTER(SZ)]
        for f in ("lfmm3d_solve_learned", "lfmm3d_solve_learned_device"):
            getattr(L, f).argtypes = [P, SZ, P, P, SZ, P, ctypes.POINTER(LfmmSolveOpts), P, D, I, P, P,
                                      ctypes.POINTER(LfmmLearnedInfo), ctypes.POINTER(LfmmStats)]
        L.lfmm3d_solve_batch_learned_device.argtypes = [P, I, P, P, P, ctypes.POINTER(LfmmSolveOpts), P, D, I, P, P,
                                                         ctypes.POINTER(LfmmLearnedInfo), ctypes.POINTER(LfmmStats)]
        L.lfmm3d_plan_create.argtypes = [P, SZ, P, P, ctypes.POINTER(LfmmSolveOpts), ctypes.POINTER(P)]
        L.lfmm3d_plan_create_batch.argtypes = [P, I, P, P, P, ctypes.POINTER(LfmmSolveOpts), ctypes.POINTER(P)]
        L.lfmm3d_plan_execute.argtypes = [P, P, P, P]
        L.lfmm3d_plan_destroy.argtypes = [P]
        L.lfmm3d_plan_destroy.restype = None
        for f in ("lfmm3d_solve_batch", "lfmm3d_solve_batch_device"):
            getattr(L, f).argtypes = [P, I, P, P, P, ctypes.POINTER(LfmmSolveOpts), P, P, ctypes.POINTER(LfmmStats)]
        _lib = L
        return L


class Context:
    """One solver context (CUDA stream + device arena + rotation tables)."""

    def __init__(self, device: int = 0, timing: bool = False):
        self.lib = load()
        self.handle = ctypes.c_void_p()
        opt = LfmmOptions(device, 0, 1 if timing else 0)
        st = self.lib.lfmm_create(ctypes.byref(self.handle), ctypes.byref(opt))
        if st != 0:
            raise LfmmError(f"lfmm_create failed ({STATUS.get(st, st)}): no usable CUDA device {device}?")
        self.device = device

    def check(self, st: int, what: str):
        if st != 0:
            msg = self.lib.lfmm_last_error(self.handle).decode()
            raise LfmmError(f"{what}: {STATUS.get(st, st)}: {msg}")

    @property
    def stream(self) -> int:
        return self.lib.lfmm_stream(self.handle)

    def close(self):
        if self.handle:
            self.lib.lfmm_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default: dict[int, Context] = {}


def default_context(device: int = 0) -> Context:
    with _lock:
        ctx = _default.get(device)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _default[device] = ctx
    return ctx
