// tcgen05 (5th-generation tensor core) form of the direction-grouped M2L
// GEMM for the FP32 levels, FP16 (or TF32) with a hi + lo split of both operands:
//   D = B T^T ~= B_hi T_hi + (B_hi T_lo + B_lo T_hi)
// with D[targets][output coefficients], B the gathered source multipoles and
// T the offset's operator.  The three products of each far slot are summed
// in a fresh TMEM accumulator and added to FP32 registers after the slot (one
// tensor-core FP32 chain across 189 slots would keep only ~1e-5 relative
// accuracy).  B is stored by the producers into tensor memory and read from
// there by the MMAs; shared memory holds only the operator stages.
#pragma once
#include "m2l_gemm.cuh"

namespace lfmm {

// Device flag: an mbarrier wait gave up (the kernel returned early).
constexpr unsigned DEV_ERR_TIMEOUT = 8u;

// Operator rows (MMA N) = m2l_padded(N); K blocks of 32 inputs (128 bytes of TF32).
inline int m2l_tc_kblocks(int N) { return (m2l_padded(N) + 31) / 32; }
inline bool m2l_tc_supported(int N) { return N >= 7 && N <= 18; }
// Output columns on the full-accuracy path (drained to FP32 after every slot,
// hi/lo corrections): all of them up to N = 12, the coefficients of degree
// < 12 (156 reals, padded to 160) above; the higher degrees accumulate in
// tensor memory from the hi products alone (their terms are at the
// truncation-error level).
inline int m2l_tc_drained(int N) { return m2l_padded(N) <= 160 ? m2l_padded(N) : 160; }

// Operators in the tensor-core layout: per (direction, K block): the hi rows
// of all m2l_padded(N) output columns, then, for the K blocks of the drained
// columns' source degrees, the lo rows of the m2l_tc_drained(N) drained
// columns; rows of 128 bytes, 128-byte swizzled (16-byte chunk c of row r
// stored at chunk c ^ (r & 7)); built from the FP64 scaled operators, cached
// per context.  The context's operand type (Context::m2l_f16): TF32 pairs,
// K blocks of 32 inputs, or FP16 pairs of the operators scaled by a power of
// two (*t_inv: its inverse), K blocks of 64 inputs.
const uint4* m2l_ops_tc(Context& ctx, int N, float* t_inv = nullptr);
size_t tc16_ops_bytes(int ndir, int N);

// loc = sum over slots of T_dir mult[src] for every cell of the level (FP32).
// n_src in (0, N): the level's M2L order, the degrees of the sources it uses
// (the nearest offsets use n_src degrees, the farther ones the truncation
// rule's fewer, never below the corrected K blocks); 0: N.  ops and t_inv from
// m2l_ops_tc (the context's operand type).
int m2l_gemm_tc(Context& ctx, const M2LPlan& plan, const uint4* ops, const float* mult, float* loc, int N,
                int n_src = 0, float t_inv = 1.f);

// The same engine for the level-to-level shifts, whose scaled operators are
// one per child octant:
//   TC_M2M  targets = the level's non-leaf cells (one class), 8 slots = the
//           child octants, vtab[cell][8] = child (next level) or -1, and
//           dst[cell] = sum_o T_o src[child_o];
//   TC_L2L  targets = the level's cells grouped by octant (class = octant),
//           1 slot = the parent (previous level), dst[cell] += T_class src[parent]
//           with T's diagonal taken out of the operators and applied in FP32:
//           ops holds the 8 operators (tc_ops_bytes(8, N)) and then the
//           diagonal as float [8][m2l_padded(N)].
enum { TC_M2L = 0, TC_M2M = 1, TC_L2L = 2 };
// src_cells: the cells of src (the children's level for M2M, the parents'
// for L2L); an index outside it is skipped and reported as DEV_ERR_RANGE.
int shift_gemm_tc(Context& ctx, int mode, const M2LPlan& plan, const uint4* ops, const float* src, float* dst, int N,
                  size_t src_cells);
// FP64 operators [ndir][m2l_padded(N)][m2l_padded(N)] -> the tensor-core layout
// at out (tc_ops_bytes(ndir, N) bytes, 16-byte aligned).
size_t tc_ops_bytes(int ndir, int N);
int tc_ops_convert(Context& ctx, const double* ops64, int ndir, int N, void* out);

} // namespace lfmm
