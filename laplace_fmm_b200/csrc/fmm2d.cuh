// 2D Laplace FMM on the device (complex Taylor / Laurent expansions, FP64).
#pragma once
#include "fmm3d.cuh"

namespace lfmm {

// Device buffers; pot (n_out), field (n_out x 2: re, im).
int fmm2d_solve_device(Context& ctx, const ParticleInput& in, int N, int depth, double* pot, double* field,
                       SolveStats* stats);

// Adaptive quadtree (cells split while they hold more than max_leaf
// particles, at most depth levels) with U / V / W / X lists; FP64.
int fmm2d_solve_adaptive(Context& ctx, const ParticleInput& in, int N, int depth, int max_leaf, double* pot,
                         double* field, SolveStats* stats);

} // namespace lfmm
