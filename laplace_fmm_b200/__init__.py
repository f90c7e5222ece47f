"""B200-native (sm_100a) Laplace fast multipole method.

The compute path is ``liblfmm.so`` (hand-written CUDA kernels behind the C ABI
in ``include/lfmm.h``); this package is the host-side mirror of the
reference's solver classes over that ABI.
"""
from ._lib import AUTO, Context, LfmmError, default_context, load  # noqa: F401
from .fmm import (FMM_AUTO, FastMultipole, FastMultipole3d, InteractionType, compute_exact,  # noqa: F401
                  cuda_clear_math_constants, cuda_copy_math_constants, init_math_constants,
                  particle2d_dtype, particle3d_dtype, solve_batch, Plan3d, BatchPlan3d)

__all__ = ["FastMultipole3d", "FastMultipole", "compute_exact", "InteractionType", "FMM_AUTO", "Context",
           "default_context", "LfmmError", "init_math_constants", "cuda_copy_math_constants",
           "cuda_clear_math_constants", "particle3d_dtype", "particle2d_dtype", "solve_batch", "Plan3d", "BatchPlan3d"]
