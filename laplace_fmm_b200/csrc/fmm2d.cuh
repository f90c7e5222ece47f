// 2D Laplace FMM on the device (complex Taylor / Laurent expansions, FP64).
#pragma once
#include "fmm3d.cuh"

namespace lfmm {

// Device buffers; pot (n_out), field (n_out x 2: re, im).
int fmm2d_solve_device(Context& ctx, const ParticleInput& in, int N, int depth, double* pot, double* field,
                       SolveStats* stats);

} // namespace lfmm
