// 3D rotation-based Laplace FMM on the device (plain FP64 form).
#pragma once
#include "tree.cuh"

namespace lfmm {

struct SolveStats {
	int N = 0, depth = 0;
	size_t n_particles = 0, n_cells = 0, n_leaves = 0, targets_num = 0;
	size_t n_far_pairs = 0, n_close_pairs = 0, n_p2p_pairs = 0;
	size_t n_m2p = 0, n_w = 0, n_x = 0;
	float ms_tree = 0, ms_upward = 0, ms_m2l = 0, ms_l2l = 0, ms_leaves = 0, ms_total = 0;
	float ms_m2l_kernel = 0;     // inside the M2L GEMMs (3D: tensor-core launches; 2D: every level's)
	int n_m2l_kernel = 0;        // those launches
};

// Solve on device-resident inputs; pot (n_out) and field (n_out x 3) are
// device pointers, n_out = nt if nt > 0 else ns.  N = number of degrees
// (order p + 1), depth = uniform tree depth (levels), both already resolved.
int fmm3d_solve_device(Context& ctx, const ParticleInput& in, int N, int depth, double* pot, double* field,
                       SolveStats* stats, DevTree* tree_out = nullptr, double2** inner_out = nullptr,
                       double2** outer_out = nullptr);

// Scaled-expansion solver on the adaptive-form tree (max_leaf = 0: uniform
// depth `depth`; > 0: adaptive, at most `depth` levels): precision 0 = FP64,
// 1 = mixed (FP32 expansions / near field, FP64 M2L on levels 2-3, FP64 tile
// sums and self term).  N <= 18.
// Vector charges (in.srcq: 3 doubles per source): field = sum q x d / r^3.
int fmm3d_solve_vector(Context& ctx, const ParticleInput& in, int N, int depth, int max_leaf, int precision,
                       double* field, SolveStats* stats);
// level_N (optional, depth entries): the M2L order of each level, the
// degrees of the source multipoles its M2L uses (0 or >= N: N); honoured on
// the tensor-core (mixed-form FP32) levels, whose expansions keep N degrees.
int fmm3d_solve_scaled(Context& ctx, const ParticleInput& in, int N, int depth, int max_leaf, int precision,
                       double* pot, double* field, SolveStats* stats, DevTree* tree_out = nullptr,
                       const int* level_N = nullptr);
// The same on a tree built by tree_build_adaptive (phase events 0 and 1, the
// tree build, are the caller's when timing).
int fmm3d_scaled_on_tree(Context& ctx, const DevTree& t, int N, int precision, double* pot, double* field,
                         SolveStats* stats, const int* level_N = nullptr);

// Dense FP64 M2L operators [343][MT][MT] for cell size h (h = 1: the
// level-independent scaled operators), cached in the context.
double* m2l_ops_fp64(Context& ctx, int N, double h);
float* m2l_ops_fp32(Context& ctx, int N);

} // namespace lfmm
