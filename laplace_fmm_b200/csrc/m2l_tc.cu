// tcgen05 M2L engine (m2l_tc.cuh).  One CTA per work item (a tile of 128
// targets of one octant class and a share of its far slots); D[128 targets][NC
// coefficients] in TMEM.  Operands are hi / lo pairs: FP16 for the M2L (the
// default; operators and each level's multipoles scaled by exact powers of
// two), TF32 for the M2M / L2L shifts and the LFMM_M2L_TYPE=tf32 M2L.  Warp roles:
//   warps 0-3  producers, one target row per thread.  FP16 with TMA (the
//              default M2L): the sources are split once per level into staged
//              FP16 hi / lo rows (stage_f16_kernel); per K block lanes 0-7 of
//              each warp gather the warp's rows with tile::gather4 copies
//              straight into the stage's 128-byte swizzled rows, and lane 0
//              arrives with the warp's byte count.  Otherwise thread t loads
//              target t's source K block (staged FP16 rows, or the FP32
//              multipole it splits into TF32 hi / lo), stores hi into TMEM
//              lane t (read by two MMAs from tensor memory) and lo into the
//              stage's shared memory as a swizzled row (read by one).  Warp
//              0's lane 0 (thread 0) also starts the bulk copy of the
//              operator block (hi and lo rows, stored pre-swizzled).
//   warp 4     TMEM owner; lane 0 issues the MMAs (M = 128, K steps of 32
//              bytes): main = B_hi T_hi (fresh per slot), corr += B_hi T_lo +
//              B_lo T_hi.
//   warps 5-12 epilogue: after each slot, add main to FP32 registers (warp w
//              reads TMEM lanes 32 (w % 4) .. +31, half of the columns each).
// TMEM: main, the high-degree columns and the corrections (TcCfg), and, when
// two or more fit, the stages' B_hi blocks (32 columns each); else B_hi sits in
// shared memory beside B_lo.  The two accumulators stay apart: each
// tensor-core accumulate rounds at its accumulator's ulp, and the corrections
// summed into main (measured) doubled the mixed form's error on clustered
// sets.  Stages (full: 128 producer arrivals, or 4 with TMA, plus the copies'
// bytes; empty: MMA commit): two to three; one main accumulator (full: MMA
// commit after the slot; empty: 256 epilogue arrivals).  Every wait is
// bounded; on expiry the kernel sets DEV_ERR_TIMEOUT, waits (bounded) for its
// copies and MMAs in flight, frees TMEM and returns.
#include "m2l_tc.cuh"
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>
#include "fmm3d.cuh"
#include <mutex>
#include <cstring>
#include <cmath>

namespace lfmm {

namespace {

__constant__ int16_t c_tc_slot_dir[8][M2L_SLOTS];

constexpr int TC_M = 128;                 // targets per tile
constexpr int NSTAGE_MAX = 3;
constexpr int EPI_WARP0 = 5, EPI_WARPS = 8;
constexpr int TC_THREADS = (EPI_WARP0 + EPI_WARPS) * 32;
constexpr uint32_t TMEM_COLS = 512;
constexpr int WAIT_LIMIT = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Round to TF32 (nearest, ties away); the low 13 bits of the cvt result are
// not specified, so they are cleared to make the value exact as an FP32.
__device__ __forceinline__ uint32_t tf32_rna(float x)
{
	uint32_t r;
	asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
	return r & 0xffffe000u;
}

// K-major operand, 128-byte swizzle, 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr)
{
	uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
	d |= (uint64_t)1u << 16;
	d |= (uint64_t)(1024u >> 4) << 32;
	d |= (uint64_t)1u << 46;
	d |= (uint64_t)2u << 61;
	return d;
}

// Instruction descriptor: D FP32, A and B both TF32 (kind::tf32) or both FP16
// (kind::f16), K-major, M = TC_M, N = n (a multiple of 16 in [16, 256]).
template <bool F16>
__host__ __device__ constexpr uint32_t idesc_of(int n)
{
	return (1u << 4) | ((F16 ? 0u : 2u) << 7) | ((F16 ? 0u : 2u) << 10) | ((uint32_t)(n >> 3) << 17) |
	       ((uint32_t)(TC_M >> 4) << 24);
}

// D (+)= A B^T, one K step (32 bytes of each row: 8 TF32 or 16 FP16 inputs),
// A read from tensor memory (M lanes x 8 columns)
template <bool F16>
__device__ __forceinline__ void mma_ta(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
	if constexpr (F16)
		asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		             "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n"
		             :: "r"(d_tmem), "r"(a_tmem), "l"(b), "r"(idesc), "r"(accumulate));
	else
		asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		             "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n"
		             :: "r"(d_tmem), "r"(a_tmem), "l"(b), "r"(idesc), "r"(accumulate));
}

// the same with A in shared memory
template <bool F16>
__device__ __forceinline__ void mma_ss(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
	if constexpr (F16)
		asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
		             :: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
	else
		asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		             "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
		             :: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
	asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}

// Wait for the phase of the given parity; gives up after WAIT_LIMIT polls, or
// at once when *abort is set (abort == nullptr: a draining wait).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort)
{
	for (int it = 0; it < WAIT_LIMIT; ++it) {
		uint32_t ok;
		asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
		if (ok) return true;
		if (abort && *abort) return false;
	}
	return false;
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}

// Rows y0..y3 of a 2D tensor map (box: one row of 64 FP16 = 128 bytes, 128-byte
// swizzle) from column x into 4 consecutive 128-byte rows at dst.
__device__ __forceinline__ void gather4_g2s(uint32_t dst, const CUtensorMap* map, int x, int y0, int y1, int y2, int y3,
                                            uint32_t bar)
{
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
	             " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
	             :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3),
	                "r"(bar)
	             : "memory");
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
	             :: "r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}

// TMEM -> registers, 32 lanes x 16 (or 8) consecutive columns, the wait inside
// the same asm so the values are complete when it returns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
	uint32_t r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
	             "tcgen05.wait::ld.sync.aligned;"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	               "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
	               "=r"(r[15])
	             : "r"(taddr) : "memory");
#pragma unroll
	for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v)
{
	uint32_t r[8];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n\t"
	             "tcgen05.wait::ld.sync.aligned;"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
	             : "r"(taddr) : "memory");
#pragma unroll
	for (int j = 0; j < 8; ++j) v[j] = __uint_as_float(r[j]);
}

// registers -> TMEM, 32 lanes x 16 consecutive columns (the thread's own lane)
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* r)
{
	asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
	             :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
	                "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
	             : "memory");
}

// acc[0 .. W) += TMEM columns [col, col + W) of this warp's 32 lanes
template <int W>
__device__ __forceinline__ void tmem_accumulate(uint32_t taddr, float (&acc)[W])
{
#pragma unroll
	for (int c = 0; c + 16 <= W; c += 16) {
		float v[16];
		tmem_ld16(taddr + c, v);
#pragma unroll
		for (int j = 0; j < 16; ++j) acc[c + j] += v[j];
	}
#pragma unroll
	for (int c = W / 16 * 16; c < W; c += 8) {
		float v[8];
		tmem_ld8(taddr + c, v);
#pragma unroll
		for (int j = 0; j < 8; ++j) acc[c + j] += v[j];
	}
}

// Far slots of the farther offsets run truncated (tc_trunc): fewer K blocks of
// source degrees and the same number of output columns, so the operator copy,
// the gathers and the MMAs of such a slot shrink together.
//
// Column split of the NC output coefficients (triangular (n, m) order, so a
// degree is a prefix): columns [0, NA) are the low degrees, whose MMA result
// is drained to FP32 registers after every slot and which get the hi/lo
// correction products; columns [NA, NC) are the high degrees, accumulated
// across all slots in tensor memory from B_hi T_hi alone.  A coefficient of
// degree >= 12 scales its term by at most (sqrt(3)/2)^12 ~ 0.18 at the target
// and carries what is left of the far field beyond that degree (the
// truncation error of a 12-degree expansion, ~1e-5 relative here), so the
// TF32 rounding (2^-11) and the tensor-core accumulation (~1e-5 relative) of
// those columns stay near 1e-9 of the result.  The corrections are applied to
// the source degrees of the same range only (K blocks [0, KBC)), for the same
// reason.  NA = NC keeps every column on the full path (low orders).
//
// TMEM columns: P = main of the drained columns [0, NA), fresh per slot;
// Q = the high-degree columns [NA, NC), one accumulator over all slots;
// C = corrections of the drained columns [NC, NC + NA), over all slots; the
// stages' B_hi blocks (32 columns each) after C when two or more fit, else
// B_hi goes to shared memory beside B_lo.  Shared memory per K block:
// operator hi rows (NC x 128 bytes), then, for K blocks below KBC, the lo rows
// of the drained columns (NA x 128 bytes) and the sources' lo block.
//
// TMEM_HI = false keeps the sources' hi parts in shared memory (the L2L
// mode: one slot of few K blocks per tile leaves the TMEM stores' waits exposed).
// F16: the operands are FP16 hi / lo pairs (kind::f16, twice the TF32 rate;
// the same 11-bit significands, the range kept by exact power-of-two scales of
// the operators and of each level's multipoles): a 128-byte row holds 64
// inputs instead of 32, so a K block covers 64 inputs with the same bytes,
// descriptors and TMEM columns.
template <int NC, int NA, bool TMEM_HI = true, bool F16 = false>
struct TcCfg {
	static constexpr int EPB = F16 ? 64 : 32;           // inputs per 128-byte row (K block)
	static constexpr int UPB = EPB / 32;                // 32-input gather units per K block
	static constexpr int KB = (NC + EPB - 1) / EPB;     // K blocks
	static constexpr int KBC = (NA + EPB - 1) / EPB;    // K blocks with corrections
	static constexpr int HI_BYTES = NC * 128;           // operator hi rows of a K block
	static constexpr int LO_BYTES = NA * 128;           // operator lo rows (drained columns) of a K block
	static constexpr int A_BYTES = TC_M * 128;          // one 32-wide K block of the multipoles (hi or lo)
	static constexpr size_t DIR_BYTES = (size_t)KB * HI_BYTES + (size_t)KBC * LO_BYTES;
	static constexpr uint32_t Q_COL = NA, C_COL = NC;
	static constexpr int FREE = (int)TMEM_COLS - NC - NA;
	static constexpr bool HI_TMEM = TMEM_HI && FREE >= 64; // B_hi in TMEM (else in shared memory)
	static constexpr int STAGE = HI_BYTES + LO_BYTES + (HI_TMEM ? 1 : 2) * A_BYTES;
	static constexpr int NSTAGE = HI_TMEM ? (FREE / 32 < NSTAGE_MAX ? FREE / 32 : NSTAGE_MAX)
	                                      : ((227 * 1024 - 1024) / STAGE >= 3 ? 3 : 2);
	static constexpr int HALF = NA / 2;                 // drained columns per epilogue warp
	static constexpr int HQ = (NC - NA) / 2;            // high-degree columns per epilogue warp
	static constexpr int SMEM = NSTAGE * STAGE + 1024;
	static __host__ __device__ __forceinline__ size_t op_off(int kb)
	{ return (size_t)kb * HI_BYTES + (size_t)(kb < KBC ? kb : KBC) * LO_BYTES; }
	static __host__ __device__ __forceinline__ uint32_t op_bytes(int kb)
	{ return (uint32_t)(HI_BYTES + (kb < KBC ? LO_BYTES : 0)); }
	static __device__ __forceinline__ uint32_t hi_col(uint32_t s) { return (uint32_t)(NC + NA) + 32u * s; }
	// K steps (32 bytes of a row each) of K block kb holding inputs below NC
	static __host__ __device__ __forceinline__ int ksteps(int kb)
	{ const int left = NC - kb * EPB; return left >= EPB ? 4 : (left + EPB / 4 - 1) / (EPB / 4); }
	static_assert(NC % 16 == 0 && NC >= 16 && NC <= 352, "operator rows");
	static_assert(NA % 16 == 0 && NA >= 16 && NA <= NC && NA <= 256 && NC - NA <= 256, "MMA N");
	static_assert(NC + NA <= (int)TMEM_COLS, "TMEM columns");
	static_assert(HALF % 8 == 0 && HQ % 8 == 0, "epilogue column split");
	static_assert(SMEM <= 227 * 1024, "shared memory");
};

// K blocks of the far slots by squared offset length |d|^2 (0 .. 27, in cell
// sizes): a slot of a far offset converges faster (worst-case ratio
// sqrt(3) / |d|) and reaches the truncation error of the nearest offsets
// with fewer degrees, so its M2L runs on the first kb[|d|^2] K blocks of
// source degrees and the same number of output columns (never fewer than the
// corrected ones).
struct TcTrunc {
	uint8_t kb[28];
};

__device__ __forceinline__ int dir_d2(int dir)
{
	const int dx = dir / 49 - 3, dy = (dir / 7) % 7 - 3, dz = dir % 7 - 3;
	return dx * dx + dy * dy + dz * dz;
}

// A persistent grid (about one block per SM) taking work items from a
// counter: item w is tile w / S and slot split w % S.  With S > 1 split s
// handles slots [s*SLOTS/S, (s+1)*SLOTS/S) and writes part[s][cell][R]; else
// loc[cell][R].  Tensor memory is allocated once per block; the barriers are
// initialised afresh for every item (every copy, MMA and arrival of the
// previous item has completed by then).
// MODE picks the operator of a (class, slot) and the store:
//   TC_M2L    189 far slots, operator c_tc_slot_dir[class][slot], loc = sum;
//   TC_M2M    8 slots (child octants), operator = slot, loc = sum;
//   TC_L2L    1 slot (the parent), operator = class (the child's octant)
//             without its diagonal, loc += sum + diag[class] * parent (the
//             diagonal, 2^-(n+1) on degree n, applied exactly in FP32: through
//             the TF32 split the dominant coefficients would lose 2^-22 per level).
// The K blocks of a slot are fed from the highest degrees down, so the
// dominant low-degree products enter each FP32 accumulator last, when the
// accumulator's own rounding has least left to act on.
// The exponent e of the FP16 multipole scale 2^e for a level whose largest
// magnitude has the float bits mb: 2^e mb in [2^14, 2^15).
__host__ __device__ __forceinline__ int f16_exponent(uint32_t mb)
{
	const int e = mb ? 14 - ((int)((mb >> 23) & 255u) - 127) : 0;
	return e < -126 ? -126 : (e > 126 ? 126 : e);
}

// The M2L's FP16 sources: each cell's multipole (R floats) x 2^e split into
// FP16 hi and lo (the residual), as rows of KB blocks of 64 (hi; zero past
// R) and of KBC blocks (lo), FP16 pairs with the lower input in the low half.
// One thread per (cell, 8 inputs).
__global__ void stage_f16_kernel(const float* __restrict__ mult, size_t cells, int R, int KB, int KBC,
                                 const unsigned* __restrict__ bmax, uint4* __restrict__ hi, uint4* __restrict__ lo)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= cells * (size_t)KB * 8) return;
	const size_t cell = i / ((size_t)KB * 8);
	const int c = (int)(i % ((size_t)KB * 8));
	const float sc = __uint_as_float((uint32_t)(127 + f16_exponent(*bmax)) << 23);
	const float2* row = reinterpret_cast<const float2*>(mult + cell * (size_t)R);
	uint32_t h[4], l[4];
#pragma unroll
	for (int q = 0; q < 4; ++q) {
		const int k = c * 8 + 2 * q;                 // R is even: a pair is in or out
		const float2 x = k < R ? row[k / 2] : make_float2(0.f, 0.f);
		const float x0 = x.x * sc, x1 = x.y * sc;
		const __half h0 = __float2half_rn(x0), h1 = __float2half_rn(x1);
		const __half l0 = __float2half_rn(x0 - __half2float(h0)), l1 = __float2half_rn(x1 - __half2float(h1));
		h[q] = (uint32_t)__half_as_ushort(h0) | ((uint32_t)__half_as_ushort(h1) << 16);
		l[q] = (uint32_t)__half_as_ushort(l0) | ((uint32_t)__half_as_ushort(l1) << 16);
	}
	hi[i] = make_uint4(h[0], h[1], h[2], h[3]);
	if (c < KBC * 8) lo[cell * (size_t)KBC * 8 + c] = make_uint4(l[0], l[1], l[2], l[3]);
}

// F16 (M2L only): the sources come split already (stage_f16_kernel): shi /
// slo hold each source cell's multipole scaled by 2^e, with e such that the
// level's largest magnitude (*bmax, the bits of a positive float) lands in
// [2^14, 2^15), as FP16 hi / lo rows of KB (lo: KBC) blocks of 64; the
// results are scaled by 2^-e t_inv (t_inv: the inverse of the operators'
// scale); both exact.
// TMA (with F16): the producers gather the staged rows with tile::gather4
// (tm_hi / tm_lo: the staged hi / lo arrays, one row per source cell and a
// zero row zero_row for targets without a source in the slot) straight into
// the stage's swizzled A rows; the MMAs read both A parts from shared memory.
template <int NC, int NA, int SLOTS, int MODE, bool PERSIST, bool F16, bool TMA>
__global__ void __launch_bounds__(TC_THREADS, 1)
m2l_tc_kernel(const uint8_t* __restrict__ ops, const float* __restrict__ mult, float* __restrict__ loc,
              const int32_t* __restrict__ vtab, const int32_t* __restrict__ order,
              const uint32_t* __restrict__ oct_count, int R, float* __restrict__ part, size_t cells,
              const float* __restrict__ diag, unsigned* flags, const TcTrunc trunc, size_t src_cells, int ndir,
              unsigned* __restrict__ work, int S, unsigned total, const unsigned* __restrict__ bmax, float t_inv,
              const uint4* __restrict__ shi, const uint4* __restrict__ slo,
              const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo, int zero_row)
{
	static_assert(!F16 || MODE == TC_M2L, "FP16 operands: M2L only");
	static_assert(!TMA || F16, "TMA row gathers: FP16 staged sources only");
	using C = TcCfg<NC, NA, MODE != TC_L2L && !TMA, F16>;
	constexpr int UPB = C::UPB;
	extern __shared__ uint8_t dsm[];
	constexpr int NSTAGE = C::NSTAGE;
	constexpr int KB = C::KB, KBC = C::KBC;
	__shared__ uint64_t full_bar[NSTAGE_MAX], empty_bar[NSTAGE_MAX];
	__shared__ uint64_t tfull_bar, tempty_bar, drain_bar;
	__shared__ uint32_t tmem_sh;
	__shared__ int32_t tgt[TC_M];
	__shared__ uint32_t active_mask[(SLOTS + 31) / 32];
	__shared__ int16_t active[SLOTS];
	__shared__ uint8_t active_kb[SLOTS];     // K blocks of each active slot
	__shared__ int s_nactive, s_oct, s_n, s_abort;
	__shared__ uint32_t s_start, s_work;

	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	uint8_t* base = dsm + ((1024u - (smem_u32(dsm) & 1023u)) & 1023u);
	volatile int* abort = &s_abort;
	if (tid == 0) s_abort = 0;
	if (warp == 4) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		             :: "r"(smem_u32(&tmem_sh)), "r"(TMEM_COLS));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
	}
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	const uint32_t tmem = tmem_sh;
	// the FP16 outputs' scale 2^-e t_inv
	float out_scale = 1.f;
	if constexpr (F16) out_scale = __uint_as_float((uint32_t)(127 - f16_exponent(*bmax)) << 23) * t_inv;

	for (int round = 0;; ++round) {
	uint32_t witem;
	if constexpr (PERSIST) {
		if (tid == 0) s_work = *abort ? total : atomicAdd(work, 1u);
		__syncthreads();
		witem = s_work;
	} else {
		if (round > 0) break;         // one item per block: item = block
		witem = blockIdx.x;
	}
	if (witem >= total) break;
	const int sidx = (int)(witem % (uint32_t)S);
	const int slot0 = sidx * SLOTS / S, slot1 = (sidx + 1) * SLOTS / S;
	float* out = S > 1 ? part + (size_t)sidx * cells * R : loc;

	if (tid == 0) {
		// this item's (octant, tile): tiles of each octant class in turn
		uint32_t b = witem / (uint32_t)S, start = 0;
		int oct = -1, nn = 0;
		for (int o = 0; o < 8; ++o) {
			const uint32_t cnt = oct_count[o];
			const uint32_t tiles = (cnt + TC_M - 1) / TC_M;
			if (b < tiles) { oct = o; start += b * TC_M; nn = (int)min((uint32_t)TC_M, cnt - b * TC_M); break; }
			b -= tiles; start += cnt;
		}
		s_oct = oct; s_n = nn; s_start = start; s_nactive = 0;
	}
	if (tid < (SLOTS + 31) / 32) active_mask[tid] = 0u;
	__syncthreads();
	if (s_oct < 0) {
		__syncthreads();    // every thread has read s_oct before the next item rewrites it
		continue;
	}
	const int oct = s_oct;
	if (tid < TC_M) tgt[tid] = tid < s_n ? order[s_start + tid] : -1;
	if (tid == 0) {
		for (int s = 0; s < NSTAGE; ++s) {
			mbar_init(smem_u32(&full_bar[s]), TMA ? 4 : TC_M);    // TMA: one arrival per producer warp
			mbar_init(smem_u32(&empty_bar[s]), 1);
		}
		mbar_init(smem_u32(&tfull_bar), 1);
		mbar_init(smem_u32(&tempty_bar), EPI_WARPS * 32);
		mbar_init(smem_u32(&drain_bar), 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
	// slots in which at least one target of the tile has a source
	if (warp < 4) {
		const int myt = tgt[tid];
		const int32_t* row = vtab + (size_t)(myt >= 0 ? myt : 0) * SLOTS;
		for (int s = slot0; s < slot1; ++s) {
			const unsigned any = __ballot_sync(0xffffffffu, myt >= 0 && row[s] >= 0);
			if (lane == 0 && any) atomicOr(&active_mask[s >> 5], 1u << (s & 31));
		}
	}
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	if (tid == 0) {
		int n = 0;
		for (int s = slot0; s < slot1; ++s)
			if (active_mask[s >> 5] & (1u << (s & 31))) {
				int kb = KB;
				if (MODE == TC_M2L) kb = min(KB, max(KBC, (int)trunc.kb[dir_d2(c_tc_slot_dir[oct][s])]));
				active_kb[n] = (uint8_t)kb;
				active[n++] = (int16_t)s;
			}
		s_nactive = n;
	}
	__syncthreads();
	const int nact = s_nactive;

	if (warp < 4) {
		// ---- producers: one target row each; thread 0 also copies the operator.
		// The source block of the next iteration is loaded while the current
		// one is split and stored (the gathers hit L2 and their latency is
		// comparable with one K block of MMAs).
		const int myt = tgt[tid];
		uint32_t it = 0;
		// the gather of 32-input unit g (inputs [32 g, 32 g + 32)) of slot
		// active[j] into w: TF32, the 32 multipole floats (bits); F16, the staged
		// hi words (w[0, 16)) and, in corrected K blocks, lo words (w[16, 32))
		auto gather = [&](int j, int g, uint32_t (&w)[32]) {
			const int slot = active[j];
			int src = myt >= 0 ? vtab[(size_t)myt * SLOTS + slot] : -1;
			if (src >= 0 && (size_t)src >= src_cells) {    // a source outside the level: skipped, reported
				atomicOr(flags, DEV_ERR_RANGE);
				src = -1;
			}
			if constexpr (F16) {
				const bool corr = g / UPB < KBC;
				const uint4* hp = shi + (size_t)(src >= 0 ? src : 0) * (KB * 8) + g * 4;
				const uint4* lp = slo + (size_t)(src >= 0 ? src : 0) * (KBC * 8) + g * 4;
#pragma unroll
				for (int q = 0; q < 4; ++q) {
					const uint4 a = src >= 0 ? hp[q] : make_uint4(0u, 0u, 0u, 0u);
					const uint4 b = src >= 0 && corr ? lp[q] : make_uint4(0u, 0u, 0u, 0u);
					w[4 * q] = a.x; w[4 * q + 1] = a.y; w[4 * q + 2] = a.z; w[4 * q + 3] = a.w;
					w[16 + 4 * q] = b.x; w[16 + 4 * q + 1] = b.y; w[16 + 4 * q + 2] = b.z; w[16 + 4 * q + 3] = b.w;
				}
			} else {
				const float2* mp = reinterpret_cast<const float2*>(mult + (size_t)(src >= 0 ? src : 0) * R);
#pragma unroll
				for (int q = 0; q < 16; ++q) {
					const int k = g * 32 + 2 * q;            // R is even: a pair is in or out
					const float2 x = (src >= 0 && k < R) ? mp[g * 16 + q] : make_float2(0.f, 0.f);
					w[2 * q] = __float_as_uint(x.x); w[2 * q + 1] = __float_as_uint(x.y);
				}
			}
		};
		// the high-degree columns accumulate over slots of different widths:
		// they start at zero (every MMA into them accumulates)
		if constexpr (NC > NA) {
			uint32_t z[16];
#pragma unroll
			for (int e = 0; e < 16; ++e) z[e] = 0u;
			const uint32_t qa = tmem + ((uint32_t)(warp * 32) << 16) + C::Q_COL;
#pragma unroll
			for (int c = 0; c < NC - NA; c += 16) tmem_st16(qa + (uint32_t)c, z);
			asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
			asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
		}
		if constexpr (TMA) {
			// per slot each lane finds its row's source cell (or the zero row);
			// per K block lane 0 arrives with the warp's byte count (warp 0:
			// and the operator's) and lanes 0-7 gather the warp's 32 rows, four
			// per tile::gather4, hi (and lo in corrected blocks)
			for (int j = 0; j < nact; ++j) {
				const int slot = active[j];
				int dir = c_tc_slot_dir[oct][slot];
				if (dir < 0 || dir >= ndir) {               // an operator outside the set: reported
					if (tid == 0) atomicOr(flags, DEV_ERR_RANGE);
					dir = 0;
				}
				int src = myt >= 0 ? vtab[(size_t)myt * SLOTS + slot] : -1;
				if (src >= 0 && (size_t)src >= src_cells) {  // a source outside the level: skipped, reported
					atomicOr(flags, DEV_ERR_RANGE);
					src = -1;
				}
				const int y = src >= 0 ? src : zero_row;
				const int l4 = (4 * lane) & 31;
				const int y0 = __shfl_sync(0xffffffffu, y, l4), y1 = __shfl_sync(0xffffffffu, y, l4 + 1);
				const int y2 = __shfl_sync(0xffffffffu, y, l4 + 2), y3 = __shfl_sync(0xffffffffu, y, l4 + 3);
				const int kbs = active_kb[j];
				const uint32_t hi_bytes = (uint32_t)min(NC, C::EPB * kbs) * 128u;
				bool ok = true;
				for (int kq = 0; kq < kbs; ++kq, ++it) {
					const int kb = kbs - 1 - kq;
					const bool corr = kb < KBC;
					const uint32_t st = it % NSTAGE;
					uint8_t* stage = base + st * C::STAGE;
					const bool got = it < NSTAGE || mbar_wait(smem_u32(&empty_bar[st]), ((it / NSTAGE) - 1) & 1u, abort);
					if (!__all_sync(0xffffffffu, got)) {
						ok = false;
						break;
					}
					const uint32_t fb = smem_u32(&full_bar[st]);
					if (lane == 0) {
						uint32_t bytes = 32u * 128u * (corr ? 2u : 1u);
						if (warp == 0) bytes += hi_bytes + (corr ? (uint32_t)C::LO_BYTES : 0u);
						mbar_arrive_expect_tx(fb, bytes);
						if (warp == 0) {
							const uint8_t* blk = ops + (size_t)dir * C::DIR_BYTES + C::op_off(kb);
							bulk_g2s(smem_u32(stage), blk, hi_bytes, fb);
							if (corr) bulk_g2s(smem_u32(stage + C::HI_BYTES), blk + C::HI_BYTES, C::LO_BYTES, fb);
						}
					}
					__syncwarp();
					if (lane < 8) {
						const uint32_t row = (uint32_t)(32 * warp + 4 * lane) * 128u;
						uint8_t* a_lo = stage + C::HI_BYTES + C::LO_BYTES;
						gather4_g2s(smem_u32(a_lo + C::A_BYTES) + row, &tm_hi, kb * C::EPB, y0, y1, y2, y3, fb);
						if (corr) gather4_g2s(smem_u32(a_lo) + row, &tm_lo, kb * C::EPB, y0, y1, y2, y3, fb);
					}
				}
				if (!ok) {
					*abort = 1;
					atomicOr(flags, DEV_ERR_TIMEOUT);
					break;
				}
			}
		} else {
			uint32_t nxt[32];
			if (nact > 0) gather(0, (active_kb[0] - 1) * UPB, nxt);
			for (int j = 0; j < nact; ++j) {
				const int slot = active[j];
				int dir = MODE == TC_M2L ? c_tc_slot_dir[oct][slot] : MODE == TC_M2M ? slot : oct;
				if (dir < 0 || dir >= ndir) {                   // an operator outside the set: reported
					if (tid == 0) atomicOr(flags, DEV_ERR_RANGE);
					dir = 0;
				}
				const int kbs = active_kb[j];
				const uint32_t hi_bytes = (uint32_t)min(NC, C::EPB * kbs) * 128u;    // the slot's output columns
				bool ok = true;
				for (int kq = 0; kq < kbs; ++kq, ++it) {
					const int kb = kbs - 1 - kq;                 // highest degrees first
					const bool corr = kb < KBC;
					const uint32_t st = it % NSTAGE;
					uint8_t* stage = base + st * C::STAGE;
					// lo (corrected K blocks only) to the stage's swizzled row tid;
					// hi to TMEM columns [hi_col(st), +32) of lane tid (or to the row after lo's)
					const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + C::hi_col(st);
					uint8_t* rl = stage + C::HI_BYTES + C::LO_BYTES + tid * 128;
					uint8_t* rh = rl + C::A_BYTES;
					for (int u = 0; u < UPB; ++u) {
						uint32_t v[32];
	#pragma unroll
						for (int q = 0; q < 32; ++q) v[q] = nxt[q];
						if (u + 1 < UPB) gather(j, kb * UPB + u + 1, nxt);
						else if (kq + 1 < kbs) gather(j, (kb - 1) * UPB, nxt);
						else if (j + 1 < nact) gather(j + 1, (active_kb[j + 1] - 1) * UPB, nxt);
						if (u == 0) {
							// the TMEM stores below are warp-collective: the warp gives up as one
							const bool got = it < NSTAGE || mbar_wait(smem_u32(&empty_bar[st]), ((it / NSTAGE) - 1) & 1u, abort);
							if (!__all_sync(0xffffffffu, got)) {
								ok = false;
								break;
							}
							asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
							if (tid == 0) {
								// the hi rows of the slot's output columns, and the lo rows
								const uint8_t* blk = ops + (size_t)dir * C::DIR_BYTES + C::op_off(kb);
								mbar_expect_tx(smem_u32(&full_bar[st]), hi_bytes + (corr ? (uint32_t)C::LO_BYTES : 0u));
								bulk_g2s(smem_u32(stage), blk, hi_bytes, smem_u32(&full_bar[st]));
								if (corr)
									bulk_g2s(smem_u32(stage + C::HI_BYTES), blk + C::HI_BYTES, C::LO_BYTES,
									         smem_u32(&full_bar[st]));
							}
						}
						if constexpr (F16) {
							// unit u: 16 words of FP16 pairs each, hi to TMEM columns [16 u, +16),
							// lo to chunks [4 u, +4)
							const uint32_t* h = v;
							const uint32_t* l = v + 16;
							if constexpr (C::HI_TMEM) tmem_st16(ta + 16u * u, h);
	#pragma unroll
							for (int c = 0; c < 4; ++c) {
								const int pc = (4 * u + c) ^ (tid & 7);
								if (corr)
									*reinterpret_cast<uint4*>(rl + pc * 16) =
										make_uint4(l[4 * c], l[4 * c + 1], l[4 * c + 2], l[4 * c + 3]);
								if constexpr (!C::HI_TMEM)
									*reinterpret_cast<uint4*>(rh + pc * 16) =
										make_uint4(h[4 * c], h[4 * c + 1], h[4 * c + 2], h[4 * c + 3]);
							}
						} else {
	#pragma unroll
							for (int hf = 0; hf < 2; ++hf) {
								uint32_t h[16], l[16];
	#pragma unroll
								for (int e = 0; e < 16; ++e) {
									const float x = __uint_as_float(v[16 * hf + e]);
									h[e] = tf32_rna(x);
									l[e] = tf32_rna(x - __uint_as_float(h[e]));
								}
								if constexpr (C::HI_TMEM) tmem_st16(ta + 16u * hf, h);
	#pragma unroll
								for (int c = 0; c < 4; ++c) {
									const int pc = (4 * hf + c) ^ (tid & 7);
									if (corr)
										*reinterpret_cast<uint4*>(rl + pc * 16) =
											make_uint4(l[4 * c], l[4 * c + 1], l[4 * c + 2], l[4 * c + 3]);
									if constexpr (!C::HI_TMEM)
										*reinterpret_cast<uint4*>(rh + pc * 16) =
											make_uint4(h[4 * c], h[4 * c + 1], h[4 * c + 2], h[4 * c + 3]);
								}
							}
						}
					}
					if (!ok) break;
					asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
					if constexpr (C::HI_TMEM) {
						asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
						asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
					}
					mbar_arrive(smem_u32(&full_bar[st]));
				}
				if (!ok) {
					*abort = 1;
					atomicOr(flags, DEV_ERR_TIMEOUT);
					break;
				}
			}
		}
		// the operator copies still in flight land before the block exits
		if (tid == 0)
			for (uint32_t i = it > NSTAGE ? it - NSTAGE : 0; i < it; ++i)
				mbar_wait(smem_u32(&full_bar[i % NSTAGE]), (i / NSTAGE) & 1u, nullptr);
	} else if (warp == 4) {
		// ---- MMA issue (one thread)
		if (lane == 0) {
			uint32_t it = 0;
			bool ok = true;
			for (int j = 0; j < nact && ok; ++j) {
				if (j > 0 && !mbar_wait(smem_u32(&tempty_bar), (j - 1) & 1u, abort)) { ok = false; break; }
				asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
				const int kbs = active_kb[j];
				const int nq = min(NC, C::EPB * kbs) - NA;  // the slot's high-degree columns
				const uint32_t idq = nq > 0 ? idesc_of<F16>(nq) : 0u;
				constexpr uint32_t IDA = idesc_of<F16>(NA);
				for (int kq = 0; kq < kbs; ++kq, ++it) {
					const int kb = kbs - 1 - kq;
					const int k0 = 4 - C::ksteps(kb);           // the K steps past NC hold only padding
					const uint32_t st = it % NSTAGE;
					if (!mbar_wait(smem_u32(&full_bar[st]), (it / NSTAGE) & 1u, abort)) { ok = false; break; }
					asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
					const uint32_t sb = smem_u32(base + st * C::STAGE);
					const uint32_t op_hi = sb, op_lo = sb + C::HI_BYTES, a_lo = sb + C::HI_BYTES + C::LO_BYTES;
					const uint32_t a_hi_t = tmem + C::hi_col(st), a_hi_s = a_lo + C::A_BYTES;
					for (int kk = k0; kk < 4; ++kk) {
						const int ks = 3 - kk;
						const uint32_t first = kq == 0 && kk == k0;         // first MMA of the slot
						const uint64_t bh = desc_sw128(op_hi + ks * 32);
						const uint64_t bq = desc_sw128(op_hi + NA * 128 + ks * 32);
						if constexpr (C::HI_TMEM) {
							const uint32_t ah = a_hi_t + 8u * ks;
							mma_ta<F16>(tmem, ah, bh, IDA, !first);
							if (nq > 0) mma_ta<F16>(tmem + C::Q_COL, ah, bq, idq, 1u);
						} else {
							const uint64_t ah = desc_sw128(a_hi_s + ks * 32);
							mma_ss<F16>(tmem, ah, bh, IDA, !first);
							if (nq > 0) mma_ss<F16>(tmem + C::Q_COL, ah, bq, idq, 1u);
						}
						if (kb < KBC) {
							// the first correction of the tile: highest corrected block, its
							// first K step, slot 0
							const uint32_t cfirst = j == 0 && kb == KBC - 1 && kk == k0;
							const uint64_t bl = desc_sw128(op_lo + ks * 32), al = desc_sw128(a_lo + ks * 32);
							if constexpr (C::HI_TMEM) mma_ta<F16>(tmem + C::C_COL, a_hi_t + 8u * ks, bl, IDA, !cfirst);
							else mma_ss<F16>(tmem + C::C_COL, desc_sw128(a_hi_s + ks * 32), bl, IDA, !cfirst);
							mma_ss<F16>(tmem + C::C_COL, al, bh, IDA, 1u);
						}
					}
					mma_commit(smem_u32(&empty_bar[st]));
				}
				if (ok) mma_commit(smem_u32(&tfull_bar));
			}
			if (!ok) {
				*abort = 1;
				atomicOr(flags, DEV_ERR_TIMEOUT);
			}
			// every MMA issued above has completed once this commit arrives
			mma_commit(smem_u32(&drain_bar));
			mbar_wait(smem_u32(&drain_bar), 0u, nullptr);
		}
		__syncwarp();
	} else {
		// ---- epilogue: per slot, the drained columns' main -> FP32 registers;
		// at the end the corrections and the high-degree columns
		constexpr int W = C::HALF, WQ = C::HQ;
		const int quarter = warp & 3, half = (warp - EPI_WARP0) >> 2;
		const uint32_t lanes = (uint32_t)(quarter * 32) << 16;
		const uint32_t taddr = tmem + lanes + (uint32_t)(half * W);
		float acc[W];
#pragma unroll
		for (int c = 0; c < W; ++c) acc[c] = 0.f;
		bool ok = true;
		for (int j = 0; j < nact; ++j) {
			// the TMEM loads below are warp-collective: the warp gives up as one
			const bool got = mbar_wait(smem_u32(&tfull_bar), j & 1u, abort);
			if (!__all_sync(0xffffffffu, got)) { ok = false; break; }
			asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
			tmem_accumulate<W>(taddr, acc);
			asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
			mbar_arrive(smem_u32(&tempty_bar));
		}
		if (!ok) {
			*abort = 1;
			atomicOr(flags, DEV_ERR_TIMEOUT);
		} else {
			if (nact > 0) tmem_accumulate<W>(taddr + C::C_COL, acc);
			const int tg = tgt[quarter * 32 + lane];
			bool store = tg >= 0 && !*abort;
			if (store && (size_t)tg >= cells) {             // a target outside the level: skipped, reported
				atomicOr(flags, DEV_ERR_RANGE);
				store = false;
			}
			const float* xs = nullptr;
			const float* dg = nullptr;
			if (MODE == TC_L2L && store) {
				const int par = vtab[tg];
				if (par < 0 || (size_t)par >= src_cells) {
					atomicOr(flags, DEV_ERR_RANGE);
					store = false;
				} else {
					xs = mult + (size_t)par * R;
					dg = diag + oct * NC;
				}
			}
			if (store) {
				const int c0 = half * W;
				float* o = out + (size_t)tg * R + c0;
				const int lim = R - c0;
#pragma unroll
				for (int c = 0; c < W; ++c)
					if (c < lim) {
						if (MODE == TC_L2L) o[c] += acc[c] + dg[c0 + c] * xs[c0 + c];
						else if constexpr (F16) o[c] = acc[c] * out_scale;
						else o[c] = acc[c];
					}
			}
			if constexpr (WQ > 0) {
				// high-degree columns [NA + half WQ, +WQ): read once (every lane of
				// the warp takes part in the loads), stored where the target exists
				const int c0 = NA + half * WQ;
				const uint32_t qa = tmem + lanes + (uint32_t)c0;
#pragma unroll
				for (int c = 0; c < WQ; c += 8) {
					float v[8];
					if (nact > 0) tmem_ld8(qa + c, v);
					else {
#pragma unroll
						for (int e = 0; e < 8; ++e) v[e] = 0.f;
					}
					if (store) {
						float* o = out + (size_t)tg * R + c0 + c;
#pragma unroll
						for (int e = 0; e < 8; ++e)
							if (c0 + c + e < R) {
								if (MODE == TC_L2L) o[e] += v[e] + dg[c0 + c + e] * xs[c0 + c + e];
								else if constexpr (F16) o[e] = v[e] * out_scale;
								else o[e] = v[e];
							}
					}
				}
			}
		}
	}
	// the item's TMEM reads, copies and MMAs are complete: the next item may
	// re-initialise the barriers and overwrite the accumulators
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	}
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	if (warp == 4)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TMEM_COLS));
}
__global__ void tc_split_reduce_kernel(const float* __restrict__ part, float* __restrict__ loc, size_t n, int S)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	float s = part[i];
	for (int k = 1; k < S; ++k) s += part[(size_t)k * n + i];
	loc[i] = s;
}

// FP64 scaled operators [ndir][NC][NC] -> per (direction, K block): the hi
// rows of every output column, then (K blocks below KBC) the lo rows of the
// drained columns [0, NA); rows of 32 TF32 values, 16-byte chunk c of row r
// at c ^ (r & 7).  One thread per (direction, K block, row, value).
__global__ void build_tc_ops_kernel(const double* __restrict__ ops64, int ndir, int NC, int NA, int R, int KB,
                                    uint32_t* __restrict__ out)
{
	const size_t total = (size_t)ndir * KB * NC * 32;
	const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= total) return;
	const int j = (int)(e % 32);
	size_t rest = e / 32;
	const int row = (int)(rest % NC); rest /= NC;
	const int kb = (int)(rest % KB);
	const int dir = (int)(rest / KB);
	const int KBC = (NA + 31) / 32;
	const int k = kb * 32 + j;
	const double v = (row < R && k < R) ? ops64[((size_t)dir * NC + row) * NC + k] : 0.0;
	const uint32_t hi = tf32_rna((float)v);
	const uint32_t lo = tf32_rna((float)(v - (double)__uint_as_float(hi)));
	const size_t dir_words = ((size_t)KB * NC + (size_t)KBC * NA) * 32;
	const size_t blk = (size_t)dir * dir_words + ((size_t)kb * NC + (size_t)min(kb, KBC) * NA) * 32;
	const size_t in_row = (size_t)(((j >> 2) ^ (row & 7)) * 4) + (j & 3);
	out[blk + (size_t)row * 32 + in_row] = hi;
	if (kb < KBC && row < NA) out[blk + (size_t)NC * 32 + (size_t)row * 32 + in_row] = lo;
}

// The FP16 layout of the same: FP64 operators x scale -> per (direction, K
// block of 64 inputs): the hi rows of every output column, then (K blocks
// below KBC) the lo rows of the drained columns; FP16 pairs (the lower input
// in the low half), 16-byte chunk c (8 inputs) of row r at c ^ (r & 7).  One
// thread per (direction, K block, row, input pair).
__global__ void build_tc16_ops_kernel(const double* __restrict__ ops64, int ndir, int NC, int NA, int R, int KB,
                                      double scale, uint32_t* __restrict__ out)
{
	const size_t total = (size_t)ndir * KB * NC * 32;
	const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= total) return;
	const int jp = (int)(e % 32);
	size_t rest = e / 32;
	const int row = (int)(rest % NC); rest /= NC;
	const int kb = (int)(rest % KB);
	const int dir = (int)(rest / KB);
	const int KBC = (NA + 63) / 64;
	const int k = kb * 64 + 2 * jp;
	const double* src = ops64 + ((size_t)dir * NC + row) * NC;
	const double v0 = (row < R && k < R) ? src[k] * scale : 0.0;
	const double v1 = (row < R && k + 1 < R) ? src[k + 1] * scale : 0.0;
	const __half h0 = __float2half_rn((float)v0), h1 = __float2half_rn((float)v1);
	const __half l0 = __float2half_rn((float)(v0 - (double)__half2float(h0)));
	const __half l1 = __float2half_rn((float)(v1 - (double)__half2float(h1)));
	const size_t dir_words = ((size_t)KB * NC + (size_t)KBC * NA) * 32;
	const size_t blk = (size_t)dir * dir_words + ((size_t)kb * NC + (size_t)min(kb, KBC) * NA) * 32;
	const size_t in_row = (size_t)(((jp >> 2) ^ (row & 7)) * 4) + (jp & 3);
	out[blk + (size_t)row * 32 + in_row] = (uint32_t)__half_as_ushort(h0) | ((uint32_t)__half_as_ushort(h1) << 16);
	if (kb < KBC && row < NA)
		out[blk + (size_t)NC * 32 + (size_t)row * 32 + in_row] =
			(uint32_t)__half_as_ushort(l0) | ((uint32_t)__half_as_ushort(l1) << 16);
}

// *out = max |x| over x[0, n) as the bits of a non-negative double (out zeroed before)
__global__ void absmax64_kernel(const double* __restrict__ x, size_t n, unsigned long long* __restrict__ out)
{
	unsigned long long m = 0;
	for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
		m = max(m, (unsigned long long)__double_as_longlong(fabs(x[i])));
	for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
	if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// K blocks per far slot by |d|^2 for order N and KB K blocks: the offsets
// with |d|^2 < 8 (|d| = 2, sqrt 5, sqrt 6: worst-case ratios 0.87 to 0.71)
// keep every degree; the farther classes [8, 9], [10, 13], [14, 19], [20, 27]
// (ratios 0.61 down to 0.33) drop 3, 4, 5, 6 degrees, never below the
// corrected columns (the kernel's floor).  Measured on the 16.8M-particle
// clustered set at N = 16: potential 3.31e-7 -> 3.27e-7, field 6.47e-7 ->
// 6.44e-7 against the FP64 direct sum, M2L kernel 99.4 -> 73.4 ms; one
// degree off the |d|^2 = 5, 6 class already raised the field to 6.99e-7.
TcTrunc tc_trunc(int N, int KB, int EPB)
{
	TcTrunc t;
	for (int d2 = 0; d2 < 28; ++d2) {
		const int r = d2 < 8 ? 0 : d2 < 10 ? 3 : d2 < 14 ? 4 : d2 < 20 ? 5 : 6;
		const int Nd = std::max(1, N - r);
		t.kb[d2] = (uint8_t)std::min(KB, (Nd * (Nd + 1) + EPB - 1) / EPB);
	}
	return t;
}

// *out = max |x| over x[0, n) as the bits of a positive float (out zeroed
// before the launch): the FP16 M2L's multipole scale.
__global__ void absmax_kernel(const float* __restrict__ x, size_t n, unsigned* __restrict__ out)
{
	unsigned m = 0;
	for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
		m = max(m, __float_as_uint(fabsf(x[i])));
	for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
	if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// A 2D tensor map over rows of cols FP16 values (row pitch cols * 2 bytes),
// read one row of 64 values (128 bytes, 128-byte swizzle) at a time: the
// staged sources for the TMA row gathers.  cuTensorMapEncodeTiled comes from
// the driver through the runtime's entry-point query.
int row_map(Context& ctx, CUtensorMap* m, const void* base, uint64_t cols, uint64_t rows)
{
	static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
	static std::once_flag once;
	std::call_once(once, [] {
		void* fn = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) ==
		        cudaSuccess && q == cudaDriverEntryPointSuccess)
			encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
		else
			cudaGetLastError();
	});
	if (!encode) { ctx.last_error = "tensor-core M2L: cuTensorMapEncodeTiled unavailable"; return ERR_CUDA; }
	const cuuint64_t dims[2] = {cols, rows};
	const cuuint64_t strides[1] = {cols * 2};
	const cuuint32_t box[2] = {64, 1};
	const cuuint32_t estr[2] = {1, 1};
	const CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
	                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
	                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS) { ctx.last_error = "tensor-core M2L: tensor map encoding failed"; return ERR_CUDA; }
	return OK;
}

// persistent: about one block per SM taking items from the counter; else one
// block per item (the hardware's block scheduler hands them out).
template <int NC, int NA, int SLOTS = M2L_SLOTS, int MODE = TC_M2L, bool F16 = false, bool TMA = false>
int run_tc(Context& ctx, const M2LPlan& plan, const uint4* ops, const float* mult, float* loc, int R, int S, float* part,
           bool timed, size_t src_cells, const float* diag = nullptr, int n_src = 0, bool persistent = true,
           const unsigned* bmax = nullptr, float t_inv = 1.f, const uint4* shi = nullptr, const uint4* slo = nullptr,
           const CUtensorMap* maps = nullptr)
{
	using C = TcCfg<NC, NA, MODE != TC_L2L && !TMA, F16>;
	CUtensorMap m_hi, m_lo;
	std::memset(&m_hi, 0, sizeof(m_hi));
	std::memset(&m_lo, 0, sizeof(m_lo));
	if (maps) { m_hi = maps[0]; m_lo = maps[1]; }
	const unsigned tiles = (unsigned)(plan.cells / TC_M + 8);
	const unsigned total = tiles * (unsigned)S;
	unsigned* work = static_cast<unsigned*>(ctx.arena.take(sizeof(unsigned)));
	if (!work) { ctx.last_error = "tensor-core M2L: allocation failed"; return ERR_OOM; }
	LFMM_CUDA(ctx, cudaMemsetAsync(work, 0, sizeof(unsigned), ctx.stream));
	const unsigned grid = persistent ? std::min(total, (unsigned)ctx.num_sms) : total;
	timed = timed && ctx.timing && ctx.kev_used + 2 <= 32;
	if (timed) LFMM_CUDA(ctx, cudaEventRecord(ctx.kev[ctx.kev_used], ctx.stream));
	const TcTrunc tr =
		tc_trunc(n_src > 0 ? n_src : R > 0 ? (int)std::lround((std::sqrt(4.0 * R + 1.0) - 1.0) / 2.0) : 0, C::KB,
		         C::EPB);
	if (persistent)
		m2l_tc_kernel<NC, NA, SLOTS, MODE, true, F16, TMA><<<grid, TC_THREADS, C::SMEM, ctx.stream>>>(
			reinterpret_cast<const uint8_t*>(ops), mult, loc, plan.vtab, plan.order, plan.oct_count, R, part,
			plan.cells, diag, ctx.dev_flags, tr, src_cells, MODE == TC_M2L ? 343 : 8, work, S, total, bmax, t_inv,
			shi, slo, m_hi, m_lo, (int)src_cells);
	else
		m2l_tc_kernel<NC, NA, SLOTS, MODE, false, F16, TMA><<<grid, TC_THREADS, C::SMEM, ctx.stream>>>(
			reinterpret_cast<const uint8_t*>(ops), mult, loc, plan.vtab, plan.order, plan.oct_count, R, part,
			plan.cells, diag, ctx.dev_flags, tr, src_cells, MODE == TC_M2L ? 343 : 8, work, S, total, bmax, t_inv,
			shi, slo, m_hi, m_lo, (int)src_cells);
	if (timed) {
		LFMM_CUDA(ctx, cudaEventRecord(ctx.kev[ctx.kev_used + 1], ctx.stream));
		ctx.kev_used += 2;
	}
	if (S > 1) {
		const size_t n = plan.cells * (size_t)R;
		tc_split_reduce_kernel<<<div_up(n, 256), 256, 0, ctx.stream>>>(part, loc, n, S);
	}
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

// The work-item shape and the grid: the slot split S (items per tile, each
// taking 189 / S of the far slots, partials added in fixed order) and the
// launch (persistent blocks taking items from a counter, or one block per
// item).  Without tuning: the smallest power of two S that gives about two
// waves of items, one block per item.  With tuning, the first level of each
// (operator rows, log2 tiles) pair times the 8 pairs S = 1, 2, 4, 8 x
// {persistent, one block per item} with CUDA events and keeps the fastest
// for the context (stored as S | 16 for persistent; the chosen pair runs
// last, so the level's result always comes from it).
template <int NC, int NA, bool F16, bool TMA>
int launch_tc(Context& ctx, const M2LPlan& plan, const uint4* ops, const float* mult, float* loc, int R, int n_src,
              float t_inv)
{
	using C = TcCfg<NC, NA, !TMA, F16>;
	LFMM_CUDA(ctx, cudaFuncSetAttribute(m2l_tc_kernel<NC, NA, M2L_SLOTS, TC_M2L, true, F16, TMA>,
	                                    cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
	LFMM_CUDA(ctx, cudaFuncSetAttribute(m2l_tc_kernel<NC, NA, M2L_SLOTS, TC_M2L, false, F16, TMA>,
	                                    cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
	unsigned* bmax = nullptr;
	uint4 *shi = nullptr, *slo = nullptr;
	CUtensorMap maps[2];
	if (F16) {
		// the level's largest multipole magnitude (the sources' scale), then
		// the sources split once into FP16 hi / lo rows, and a zero row after
		// them (the TMA gathers' row for a target without a source)
		const size_t rows = plan.cells + 1;
		bmax = static_cast<unsigned*>(ctx.arena.take(sizeof(unsigned)));
		shi = static_cast<uint4*>(ctx.arena.take(rows * (size_t)C::KB * 128));
		slo = static_cast<uint4*>(ctx.arena.take(rows * (size_t)C::KBC * 128));
		if (!bmax || !shi || !slo) { ctx.last_error = "tensor-core M2L: allocation failed"; return ERR_OOM; }
		LFMM_CUDA(ctx, cudaMemsetAsync(shi + plan.cells * (size_t)C::KB * 8, 0, (size_t)C::KB * 128, ctx.stream));
		LFMM_CUDA(ctx, cudaMemsetAsync(slo + plan.cells * (size_t)C::KBC * 8, 0, (size_t)C::KBC * 128, ctx.stream));
		if (TMA) {
			if (int st = row_map(ctx, &maps[0], shi, (uint64_t)C::KB * 64, rows)) return st;
			if (int st = row_map(ctx, &maps[1], slo, (uint64_t)C::KBC * 64, rows)) return st;
		}
		LFMM_CUDA(ctx, cudaMemsetAsync(bmax, 0, sizeof(unsigned), ctx.stream));
		const size_t n = plan.cells * (size_t)R;
		absmax_kernel<<<(unsigned)std::min<size_t>(div_up(n, 256), 8 * (size_t)ctx.num_sms), 256, 0, ctx.stream>>>(
			mult, n, bmax);
		const size_t chunks = plan.cells * (size_t)C::KB * 8;
		stage_f16_kernel<<<div_up(chunks, 256), 256, 0, ctx.stream>>>(mult, plan.cells, R, C::KB, C::KBC, bmax, shi,
		                                                              slo);
	}
	const unsigned tiles = (unsigned)(plan.cells / TC_M + 8);
	int S = 1;
	while (S < 8 && tiles * S < 2u * (unsigned)ctx.num_sms) S *= 2;
	int bucket = 0;
	while ((1u << bucket) < tiles && bucket < 32) ++bucket;
	static_assert(NC / 16 < Context::SPLIT_ROWS, "autotuner table");
	int& tuned = ctx.m2l_split[F16 ? (TMA ? 2 : 1) : 0][NC / 16][bucket];
	const bool tune = ctx.tune_m2l && tuned == 0;
	bool pers = false;
	if (ctx.tune_m2l && !tune) { S = tuned & 15; pers = (tuned & 16) != 0; }
	// the tuner tries splits up to 8 where their partials fit in 1 GiB (a level
	// that large has tiles enough for S = 1; only the launch is tuned there)
	const int maxS = sizeof(float) * 8 * plan.cells * (size_t)R <= ((size_t)1 << 30) ? 8 : 1;
	float* part = nullptr;
	if ((tune && maxS > 1) || S > 1) {
		part = static_cast<float*>(ctx.arena.take(sizeof(float) * (tune ? maxS : S) * plan.cells * (size_t)R));
		if (!part) {
			ctx.last_error = "tensor-core M2L: allocation failed";
			return ERR_OOM;
		}
	}
	if (tune) {
		cudaEvent_t e0, e1;
		LFMM_CUDA(ctx, cudaEventCreate(&e0));
		LFMM_CUDA(ctx, cudaEventCreate(&e1));
		float best = 1e30f;
		int bestS = S;
		bool bestP = true;
		for (int mode = 0; mode < 2; ++mode)
			for (int cand = 1; cand <= maxS; cand *= 2) {
				LFMM_CUDA(ctx, cudaEventRecord(e0, ctx.stream));
				int st = run_tc<NC, NA, M2L_SLOTS, TC_M2L, F16, TMA>(ctx, plan, ops, mult, loc, R, cand, part, false,
				                                                     plan.cells, nullptr, n_src, mode == 0, bmax, t_inv,
				                                                     shi, slo, TMA ? maps : nullptr);
				if (st) return st;
				LFMM_CUDA(ctx, cudaEventRecord(e1, ctx.stream));
				LFMM_CUDA(ctx, cudaEventSynchronize(e1));
				float ms = 0.f;
				LFMM_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
				if (ms < best) { best = ms; bestS = cand; bestP = mode == 0; }
			}
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		tuned = bestS | (bestP ? 16 : 0);
		S = bestS;
		pers = bestP;
	}
	return run_tc<NC, NA, M2L_SLOTS, TC_M2L, F16, TMA>(ctx, plan, ops, mult, loc, R, S, part, true, plan.cells,
	                                                   nullptr, n_src, pers, bmax, t_inv, shi, slo,
	                                                   TMA ? maps : nullptr);
}

// M2M (8 slots, stored) or L2L (1 slot, added) of one level: S = 1.
template <int NC, int NA>
int launch_shift_tc(Context& ctx, int mode, const M2LPlan& plan, const uint4* ops, const float* src, float* dst, int R,
                    size_t src_cells)
{
	using C = TcCfg<NC, NA>;
	using CL = TcCfg<NC, NA, false>;
	if (mode == TC_M2M) {
		LFMM_CUDA(ctx, cudaFuncSetAttribute(m2l_tc_kernel<NC, NA, 8, TC_M2M, false, false, false>,
		                                    cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
		return run_tc<NC, NA, 8, TC_M2M>(ctx, plan, ops, src, dst, R, 1, nullptr, false, src_cells, nullptr, 0,
		                                 false);
	}
	LFMM_CUDA(ctx, cudaFuncSetAttribute(m2l_tc_kernel<NC, NA, 1, TC_L2L, false, false, false>,
	                                    cudaFuncAttributeMaxDynamicSharedMemorySize, CL::SMEM));
	// the diagonal [8][NC] follows the 8 operators
	const float* diag = reinterpret_cast<const float*>(reinterpret_cast<const uint8_t*>(ops) + 8 * C::DIR_BYTES);
	return run_tc<NC, NA, 1, TC_L2L>(ctx, plan, ops, src, dst, R, 1, nullptr, false, src_cells, diag, 0, false);
}

std::mutex g_upload_mu;
bool g_uploaded[64] = {};

int upload_slot_dirs(Context& ctx)
{
	std::lock_guard<std::mutex> lock(g_upload_mu);
	if (ctx.device < 0 || ctx.device >= 64) { ctx.last_error = "device index above 63"; return ERR_ARG; }
	if (!g_uploaded[ctx.device]) {
		const M2LSlots& S = m2l_slots();
		LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_tc_slot_dir, S.slot_dir, sizeof(S.slot_dir)));
		g_uploaded[ctx.device] = true;
	}
	return OK;
}

} // namespace

const uint4* m2l_ops_tc(Context& ctx, int N, float* t_inv)
{
	const bool f16 = ctx.m2l_f16 != 0;
	const int prec = f16 ? 4 : 3;
	for (auto& e : ctx.opcache)
		if (e.N == N && e.prec == prec) {
			e.stamp = ++ctx.opcache_clock;
			if (t_inv) *t_inv = e.aux;
			return static_cast<const uint4*>(e.ptr);
		}
	const double* d = m2l_ops_fp64(ctx, N, 1.0);
	if (!d) return nullptr;
	const int NC = m2l_padded(N), R = N * (N + 1), NA = m2l_tc_drained(N);
	const int KB = f16 ? (NC + 63) / 64 : m2l_tc_kblocks(N);
	OpCacheEntry e;
	e.N = N; e.prec = prec; e.h = 1.0; e.stamp = ++ctx.opcache_clock;
	double scale = 1.0;
	if (f16) {
		// the largest operator magnitude scaled into [2^14, 2^15)
		unsigned long long* mx = static_cast<unsigned long long*>(ctx.arena.take(sizeof(unsigned long long)));
		if (!mx) { ctx.last_error = "tensor-core operators: allocation failed"; return nullptr; }
		const size_t n = (size_t)343 * NC * NC;
		unsigned long long hb = 0;
		if (cudaMemsetAsync(mx, 0, sizeof(hb), ctx.stream) != cudaSuccess) { cudaGetLastError(); return nullptr; }
		absmax64_kernel<<<(unsigned)std::min<size_t>(div_up(n, 256), 8 * (size_t)ctx.num_sms), 256, 0, ctx.stream>>>(
			d, n, mx);
		if (cudaMemcpyAsync(&hb, mx, sizeof(hb), cudaMemcpyDeviceToHost, ctx.stream) != cudaSuccess ||
		    cudaStreamSynchronize(ctx.stream) != cudaSuccess) {
			cudaGetLastError();
			ctx.last_error = "tensor-core operators: scale reduction failed";
			return nullptr;
		}
		double m;
		std::memcpy(&m, &hb, sizeof(m));
		const int ex = m > 0.0 ? std::ilogb(m) : 0;
		scale = std::ldexp(1.0, 14 - ex);
		e.aux = (float)std::ldexp(1.0, ex - 14);
	}
	e.bytes = f16 ? tc16_ops_bytes(343, N) : tc_ops_bytes(343, N);
	if (cudaMalloc(&e.ptr, e.bytes) != cudaSuccess) {
		cudaGetLastError();
		ctx.last_error = "tensor-core operators: out of memory";
		return nullptr;
	}
	const size_t threads = (size_t)343 * KB * NC * 32;
	if (f16)
		build_tc16_ops_kernel<<<div_up(threads, 256), 256, 0, ctx.stream>>>(d, 343, NC, NA, R, KB, scale,
		                                                                    static_cast<uint32_t*>(e.ptr));
	else
		build_tc_ops_kernel<<<div_up(threads, 256), 256, 0, ctx.stream>>>(d, 343, NC, NA, R, KB,
		                                                                  static_cast<uint32_t*>(e.ptr));
	if (cudaGetLastError() != cudaSuccess) {
		cudaFree(e.ptr);
		ctx.last_error = "tensor-core operators: launch failed";
		return nullptr;
	}
	ctx.opcache.push_back(e);
	if (t_inv) *t_inv = e.aux;
	return static_cast<const uint4*>(e.ptr);
}

size_t tc16_ops_bytes(int ndir, int N)
{
	const int NC = m2l_padded(N), NA = m2l_tc_drained(N);
	const size_t KB = (size_t)(NC + 63) / 64, KBC = (size_t)(NA + 63) / 64;
	return (size_t)ndir * (KB * NC + KBC * NA) * 128;
}

size_t tc_ops_bytes(int ndir, int N)
{
	const int NC = m2l_padded(N), NA = m2l_tc_drained(N);
	const size_t KB = (size_t)m2l_tc_kblocks(N), KBC = (size_t)(NA + 31) / 32;
	return (size_t)ndir * (KB * NC + KBC * NA) * 128;
}

int tc_ops_convert(Context& ctx, const double* ops64, int ndir, int N, void* out)
{
	const int NC = m2l_padded(N), R = N * (N + 1), KB = m2l_tc_kblocks(N), NA = m2l_tc_drained(N);
	const size_t threads = (size_t)ndir * KB * NC * 32;
	build_tc_ops_kernel<<<div_up(threads, 256), 256, 0, ctx.stream>>>(ops64, ndir, NC, NA, R, KB,
	                                                                 static_cast<uint32_t*>(out));
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

// The (operator rows, drained columns) pairs built: every order 7 <= N <= 18.
#define LFMM_TC_ORDERS(X) X(64, 64) X(80, 80) X(96, 96) X(112, 112) X(144, 144) X(160, 160) \
	X(192, 160) X(224, 160) X(240, 160) X(272, 160) X(320, 160) X(352, 160)

int shift_gemm_tc(Context& ctx, int mode, const M2LPlan& plan, const uint4* ops, const float* src, float* dst, int N,
                  size_t src_cells)
{
	if (mode != TC_M2M && mode != TC_L2L) { ctx.last_error = "tensor-core shift: bad mode"; return ERR_ARG; }
	const int R = N * (N + 1), NC = m2l_padded(N), NA = m2l_tc_drained(N);
#define LFMM_TC_SHIFT(nc, na) if (NC == nc && NA == na) return launch_shift_tc<nc, na>(ctx, mode, plan, ops, src, dst, R, src_cells);
	LFMM_TC_ORDERS(LFMM_TC_SHIFT)
#undef LFMM_TC_SHIFT
	ctx.last_error = "tensor-core shift: unsupported order";
	return ERR_UNSUPPORTED;
}

int m2l_gemm_tc(Context& ctx, const M2LPlan& plan, const uint4* ops, const float* mult, float* loc, int N, int n_src,
                float t_inv)
{
	if (int st = upload_slot_dirs(ctx)) return st;
	const int R = N * (N + 1), NC = m2l_padded(N), NA = m2l_tc_drained(N);
	const int ns = n_src > 0 && n_src < N ? n_src : 0;
#define LFMM_TC_M2L(nc, na)                                                                                   \
	if (NC == nc && NA == na)                                                                                 \
		return !ctx.m2l_f16 ? launch_tc<nc, na, false, false>(ctx, plan, ops, mult, loc, R, ns, 1.f)          \
		       : ctx.m2l_tma ? launch_tc<nc, na, true, true>(ctx, plan, ops, mult, loc, R, ns, t_inv)          \
		                     : launch_tc<nc, na, true, false>(ctx, plan, ops, mult, loc, R, ns, t_inv);
	LFMM_TC_ORDERS(LFMM_TC_M2L)
#undef LFMM_TC_M2L
	ctx.last_error = "tensor-core M2L: unsupported order";
	return ERR_UNSUPPORTED;
}

} // namespace lfmm
