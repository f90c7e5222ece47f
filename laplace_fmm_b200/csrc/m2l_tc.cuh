// tcgen05 (5th-generation tensor core) form of the direction-grouped M2L
// GEMM, FP32 data in TF32 with a hi + lo split on both operands:
//   T B ~= T_hi B_hi + T_hi B_lo + T_lo B_hi      (FP32 accumulation in TMEM)
// which keeps ~21 bits of each product, FP32-level accuracy.
#pragma once
#include "m2l_gemm.cuh"

namespace lfmm {

// Device flag: an mbarrier wait gave up (the kernel returned early).
constexpr unsigned DEV_ERR_TIMEOUT = 8u;

// Rows of the padded operator (output coefficients): 128 or 256 (two M=128
// MMAs); K blocks of 32 inputs (128 bytes of TF32).
inline int m2l_tc_halves(int N) { return N * (N + 1) <= 128 ? 1 : 2; }
inline int m2l_tc_kblocks(int N) { return (N * (N + 1) + 31) / 32; }
inline bool m2l_tc_supported(int N) { return N * (N + 1) <= 256 && N >= 2; }

// Operators in the tensor-core layout: per direction, per K block, hi then lo,
// (128 * halves) rows of 128 bytes, 128-byte swizzled (16-byte chunk c of row
// r at chunk c ^ (r & 7)); built from the FP64 scaled operators; cached.
const uint4* m2l_ops_tc(Context& ctx, int N);

// loc = sum over slots of T_dir mult[src] for every cell of the level (FP32).
int m2l_gemm_tc(Context& ctx, const M2LPlan& plan, const uint4* ops_tc, const float* mult, float* loc, int N);

} // namespace lfmm
