// 3D rotation-based Laplace FMM on the device (plain FP64 form).
#pragma once
#include "tree.cuh"

namespace lfmm {

struct SolveStats {
	int N = 0, depth = 0;
	size_t n_particles = 0, n_cells = 0, n_leaves = 0, targets_num = 0;
	size_t n_far_pairs = 0, n_close_pairs = 0, n_p2p_pairs = 0;
	float ms_tree = 0, ms_upward = 0, ms_m2l = 0, ms_l2l = 0, ms_leaves = 0, ms_total = 0;
};

// Solve on device-resident inputs; pot (n_out) and field (n_out x 3) are
// device pointers, n_out = nt if nt > 0 else ns.  N = number of degrees
// (order p + 1), depth = uniform tree depth (levels), both already resolved.
int fmm3d_solve_device(Context& ctx, const ParticleInput& in, int N, int depth, double* pot, double* field,
                       SolveStats* stats, DevTree* tree_out = nullptr, double2** inner_out = nullptr,
                       double2** outer_out = nullptr);

// Mixed-precision form (FP32 scaled expansions below level 4, FP32 near field
// with FP64 tile accumulation); same arguments.
int fmm3d_solve_mixed(Context& ctx, const ParticleInput& in, int N, int depth, double* pot, double* field,
                      SolveStats* stats);

// Dense FP64 M2L operators [343][MT][MT] for cell size h (h = 1: the
// level-independent scaled operators), cached in the context.
double* m2l_ops_fp64(Context& ctx, int N, double h);
float* m2l_ops_fp32(Context& ctx, int N);

} // namespace lfmm
