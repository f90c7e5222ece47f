// Direction-grouped M2L as dense GEMMs.
//
// For a target cell at level L and a far offset d (in cells), the rotation-
// based M2L (rotate to the z-axis of d, z-translate, rotate back; reference
// cpu/multipole3d.cpp:152-190) is one fixed real linear map T_{L,d} of the
// 2 * N(N+1)/2 expansion reals.  A target's V list holds at most one source
// per d, and the 189 offsets a target can have depend only on its octant in
// its parent.  So targets are grouped by octant into tiles of 64; for each of
// the octant's 189 offsets the tile gathers its sources' multipoles as the
// columns of B and accumulates C += T_d B, C staying on chip across all
// offsets.
#pragma once
#include "tree.cuh"

namespace lfmm {

constexpr int M2L_SLOTS = 189;    // far offsets per octant class
constexpr int M2L_SLOTS2 = 27;    // 2D: far offsets per quadrant class
constexpr int M2L_TILE = 64;      // targets per GEMM tile

// Offsets of each octant class: slot -> direction id (dx+3)*49+(dy+3)*7+(dz+3)
// and direction id -> slot (-1 when not a far offset of that octant).
struct M2LSlots {
	int16_t slot_dir[8][M2L_SLOTS];
	int16_t dir_slot[8][343];
};
const M2LSlots& m2l_slots();

struct M2LPlan {
	int32_t* vtab = nullptr;     // [cells of level][189] source (level-local) or -1
	int32_t* order = nullptr;    // cells of the level grouped by octant
	uint32_t* oct_count = nullptr; // [8] cells per octant (device)
	size_t cells = 0;
};

// Padded operator size for N degrees: 2 N(N+1)/2 rounded up to 16.
inline int m2l_padded(int N) { return ((N * (N + 1) + 15) / 16) * 16; }
inline bool m2l_gemm_supported(int N) { return m2l_padded(N) <= 352; }

int m2l_plan_build(Context& ctx, const DevTree& t, int L, M2LPlan& plan);

// loc[c] = sum_slots T[dir] mult[src]   for every cell c of the level
// (real = double: plain form; float: mixed form).  ops: [343][MT][MT].
template <typename real>
int m2l_gemm(Context& ctx, const M2LPlan& plan, const real* ops, const real* mult, real* loc, int N);

// 2D (FP64, expansions [cell][N] complex): the quadrant classes' 27 far
// slots, the dense operators [49][MT][MT] (MT = 2N rounded up to 16) of cell
// size h, and the GEMM.
int m2l_plan_build2d(Context& ctx, const DevTree& t, int L, M2LPlan& plan);
double* m2l_ops2d(Context& ctx, int N, double h);
int m2l_gemm2d(Context& ctx, const M2LPlan& plan, const double* ops, const double* mult, double* loc, int N);
// The same M2L through the Hankel factorisation (the default 2D engine):
// the per-offset tables of cell size h and the launch (N <= 32).
double2* m2l_tab2d(Context& ctx, int N, double h);
int m2l_hankel2d(Context& ctx, const M2LPlan& plan, const double2* tab, const double2* mult, double2* loc, int N);

} // namespace lfmm
