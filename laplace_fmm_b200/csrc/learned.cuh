// Learned order selection: MLP forward (mlp.cu), per-leaf features and the
// learned solve (learned.cu).
#pragma once
#include "../../include/lfmm.h"
#include "fmm3d.cuh"

namespace lfmm {

// Y[n][14] = MLP(X[n][16]) on ctx.stream (device pointers).
int mlp_forward_device(Context& ctx, const float* params, int n, const float* X, float* Y);

// Tree (adaptive form: max_leaf > 0 splits, 0 = uniform depth), order from
// the network for tolerance tol, solve on that tree, optional sampled check
// (check_targets outputs) with the fixed-order rerun on a miss.  Device
// pointers; synchronises.
int solve_learned_device(Context& ctx, const ParticleInput& in, int depth, int max_leaf, int precision,
                         const float* params, double tol, int check_targets, double* pot, double* field,
                         lfmm_learned_info* info, SolveStats* stats);

// The same for a forest of in.nprob problems (hoff: host offsets): one order
// for the batch (the highest any problem needs), samples and check per
// problem (checked errors: the largest over the problems).
int solve_learned_batch_device(Context& ctx, const ParticleInput& in, const size_t* hoff, int depth, int max_leaf,
                               int precision, const float* params, double tol, int check_targets, double* pot,
                               double* field, lfmm_learned_info* info, SolveStats* stats);

// The threshold network's inputs [K][16] for candidate leaf-size thresholds
// cand[K] (K <= 8) at order N (host buffer).
int leaf_features_host(Context& ctx, const ParticleInput& in, int depth, int N, const int* cand, int K, float* feats);

// Per-leaf features [n_leaves][16] and the leaf of every input particle
// (host buffers; either may be null).
int features_tree(Context& ctx, const ParticleInput& in, int depth, int max_leaf, float* feats_host, size_t cap,
                  int32_t* leaf_of_host, size_t* n_leaves);

} // namespace lfmm
