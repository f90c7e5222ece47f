// Direction-grouped M2L GEMMs (see m2l_gemm.cuh), SIMT register-tiled form
// for FP64 (plain) and FP32.
#include "m2l_gemm.cuh"
#include "m2l_tc.cuh"
#include "fmm3d.cuh"
#include "primitives.cuh"
#include <mutex>
#include <cstdlib>

namespace lfmm {

namespace {

__constant__ int16_t c_slot_dir[8][M2L_SLOTS];
__constant__ int16_t c_dir_slot[8][343];

__device__ __forceinline__ void coords3(uint64_t code, int* c)
{ c[0] = (int)compact3(code >> 2); c[1] = (int)compact3(code >> 1); c[2] = (int)compact3(code); }

// Fill the V table of level L: slot of each far source in the target's
// octant class; the candidates are the children of the parent's close cells
// and of the parent (reference cpu/morton_tree.cpp:147-208).
__global__ void vtab_kernel(DevTree t, int L, int32_t* __restrict__ vtab, unsigned* flags)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	size_t m = t.lsize[L];
	if (c >= m) return;
	size_t off = t.loff[L], poff = t.loff[L - 1];
	int me[3];
	coords3(t.code[off + c], me);
	int oct = ((me[0] & 1) << 2) | ((me[1] & 1) << 1) | (me[2] & 1);
	int32_t* row = vtab + c * M2L_SLOTS;
	int32_t p = t.parent[off + c];
	int npc = t.close_cnt[poff + p];
	const int32_t* pl = t.close_idx + (poff + p) * t.close_stride;
	for (int e = 0; e <= npc; ++e) {
		int32_t pn = e < npc ? pl[e] : p;
		for (uint32_t k = t.beg[poff + pn]; k < t.end[poff + pn]; ++k) {
			if (k == c) continue;
			int o[3];
			coords3(t.code[off + k], o);
			int dx = o[0] - me[0], dy = o[1] - me[1], dz = o[2] - me[2];
			if (max(max(abs(dx), abs(dy)), abs(dz)) <= 1) continue;
			int slot = c_dir_slot[oct][(dx + 3) * 49 + (dy + 3) * 7 + (dz + 3)];
			if (slot < 0) { atomicOr(flags, DEV_ERR_DIRECTION); continue; }
			row[slot] = (int32_t)k;
		}
	}
}

__global__ void count_oct_kernel(DevTree t, int L, uint32_t* __restrict__ oct_count)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= t.lsize[L]) return;
	int me[3];
	coords3(t.code[t.loff[L] + c], me);
	int oct = ((me[0] & 1) << 2) | ((me[1] & 1) << 1) | (me[2] & 1);
	atomicAdd(&oct_count[oct], 1u);
}

__global__ void scatter_oct_kernel(DevTree t, int L, uint32_t* __restrict__ oct_count, int32_t* __restrict__ order)
{
	__shared__ uint32_t base[8];
	if (threadIdx.x < 8) {
		uint32_t a = 0;
		for (int o = 0; o < (int)threadIdx.x; ++o) a += oct_count[o];
		base[threadIdx.x] = a;
	}
	__syncthreads();
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= t.lsize[L]) return;
	int me[3];
	coords3(t.code[t.loff[L] + c], me);
	int oct = ((me[0] & 1) << 2) | ((me[1] & 1) << 1) | (me[2] & 1);
	uint32_t pos = atomicAdd(&oct_count[8 + oct], 1u);
	order[base[oct] + pos] = (int32_t)c;
}

// C[MT x 64] = sum over the octant's offsets of T_dir[MT x MT] * B[MT x 64];
// 256 threads, thread (ty, tx) owns rows ty + 16 i and columns tx + 16 j.
// blockIdx.y = split s of S: slots [s*189/S, (s+1)*189/S); with S > 1 the
// partial sums go to part[s][cell][R] and a fixed-order reduction follows.
template <typename real, int TM, int TN>
__global__ void __launch_bounds__(256) m2l_gemm_kernel(const real* __restrict__ ops, const real* __restrict__ mult,
                                                       real* __restrict__ loc, const int32_t* __restrict__ vtab,
                                                       const int32_t* __restrict__ order,
                                                       const uint32_t* __restrict__ oct_count, int R,
                                                       real* __restrict__ part, size_t cells)
{
	const int S = gridDim.y, sidx = blockIdx.y;
	const int slot0 = sidx * M2L_SLOTS / S, slot1 = (sidx + 1) * M2L_SLOTS / S;
	if (S > 1) loc = part + (size_t)sidx * cells * R;
	constexpr int MT = 16 * TM;
	constexpr int BN = 16 * TN;
	constexpr int BK = 16;
	__shared__ real As[BK][MT];
	__shared__ real Bs[BK][BN];
	__shared__ int32_t src[BN];
	__shared__ int32_t tgt[BN];
	__shared__ int s_oct, s_n;
	const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
	if (tid == 0) {
		// locate this block's (octant, tile)
		uint32_t b = blockIdx.x, start = 0;
		int oct = -1, nn = 0;
		for (int o = 0; o < 8; ++o) {
			uint32_t cnt = oct_count[o];
			uint32_t tiles = (cnt + BN - 1) / BN;
			if (b < tiles) { oct = o; start += b * BN; nn = (int)min((uint32_t)BN, cnt - b * BN); break; }
			b -= tiles; start += cnt;
		}
		s_oct = oct; s_n = nn;
		tgt[0] = (int32_t)start;
	}
	__syncthreads();
	const int oct = s_oct, nt = s_n;
	if (oct < 0) return;
	const uint32_t start = (uint32_t)tgt[0];
	__syncthreads();
	if (tid < BN) tgt[tid] = tid < nt ? order[start + tid] : -1;
	// per-offset partial sums in `real`, carried across offsets in FP64
	double acc[TM][TN];
	real part_[TM][TN];
#pragma unroll
	for (int i = 0; i < TM; ++i)
#pragma unroll
		for (int j = 0; j < TN; ++j) acc[i][j] = 0.0;
	__syncthreads();
	for (int slot = slot0; slot < slot1; ++slot) {
		int mine = -1;
		if (tid < BN && tgt[tid] >= 0) mine = vtab[(size_t)tgt[tid] * M2L_SLOTS + slot];
		if (tid < BN) src[tid] = mine;
		if (!__syncthreads_or(mine >= 0)) continue;
		if constexpr (sizeof(real) == sizeof(float)) {
#pragma unroll
			for (int i = 0; i < TM; ++i)
#pragma unroll
				for (int j = 0; j < TN; ++j) part_[i][j] = real(0);
		}
		const real* A = ops + (size_t)c_slot_dir[oct][slot] * MT * MT;
		for (int k0 = 0; k0 < MT; k0 += BK) {
			for (int idx = tid; idx < BK * MT; idx += 256) {
				int k = idx & (BK - 1), r = idx / BK;
				As[k][r] = A[(size_t)r * MT + k0 + k];
			}
			for (int idx = tid; idx < BK * BN; idx += 256) {
				int k = idx & (BK - 1), c = idx / BK;
				int s = src[c];
				int kk = k0 + k;
				Bs[k][c] = (s >= 0 && kk < R) ? mult[(size_t)s * R + kk] : real(0);
			}
			__syncthreads();
#pragma unroll
			for (int k = 0; k < BK; ++k) {
				real a[TM], b[TN];
#pragma unroll
				for (int i = 0; i < TM; ++i) a[i] = As[k][ty + 16 * i];
#pragma unroll
				for (int j = 0; j < TN; ++j) b[j] = Bs[k][tx + 16 * j];
#pragma unroll
				for (int i = 0; i < TM; ++i)
#pragma unroll
					for (int j = 0; j < TN; ++j) {
						if constexpr (sizeof(real) == sizeof(double)) acc[i][j] = fma((double)a[i], (double)b[j], acc[i][j]);
						else part_[i][j] = fma(a[i], b[j], part_[i][j]);
					}
			}
			__syncthreads();
		}
		if constexpr (sizeof(real) == sizeof(float)) {
#pragma unroll
			for (int i = 0; i < TM; ++i)
#pragma unroll
				for (int j = 0; j < TN; ++j) acc[i][j] += (double)part_[i][j];
		}
	}
#pragma unroll
	for (int j = 0; j < TN; ++j) {
		int c = tx + 16 * j;
		int tg = c < BN ? tgt[c] : -1;
		if (tg < 0) continue;
#pragma unroll
		for (int i = 0; i < TM; ++i) {
			int r = ty + 16 * i;
			if (r < R) loc[(size_t)tg * R + r] = (real)acc[i][j];
		}
	}
}

template <typename real>
__global__ void split_reduce_kernel(const real* __restrict__ part, real* __restrict__ loc, size_t n, int S)
{
	size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	real s = part[i];
	for (int k = 1; k < S; ++k) s += part[(size_t)k * n + i];
	loc[i] = s;
}

template <typename real, int TM>
void launch_gemm(dim3 grid, cudaStream_t s, const real* ops, const real* mult, real* loc, const M2LPlan& p, int R,
                 real* part)
{
	m2l_gemm_kernel<real, TM, 4><<<grid, 256, 0, s>>>(ops, mult, loc, p.vtab, p.order, p.oct_count, R, part, p.cells);
}

} // namespace

const M2LSlots& m2l_slots()
{
	static M2LSlots S;
	static std::once_flag once;
	std::call_once(once, [] {
		for (int o = 0; o < 8; ++o) {
			for (int d = 0; d < 343; ++d) S.dir_slot[o][d] = -1;
			int ox = (o >> 2) & 1, oy = (o >> 1) & 1, oz = o & 1;
			int s = 0;
			for (int dx = -2 - ox; dx <= 3 - ox; ++dx)
				for (int dy = -2 - oy; dy <= 3 - oy; ++dy)
					for (int dz = -2 - oz; dz <= 3 - oz; ++dz) {
						if (std::max(std::max(std::abs(dx), std::abs(dy)), std::abs(dz)) <= 1) continue;
						int id = (dx + 3) * 49 + (dy + 3) * 7 + (dz + 3);
						S.slot_dir[o][s] = (int16_t)id;
						S.dir_slot[o][id] = (int16_t)s;
						++s;
					}
		}
	});
	return S;
}

int m2l_plan_build(Context& ctx, const DevTree& t, int L, M2LPlan& plan)
{
	static bool uploaded = false;
	if (!uploaded) {
		const M2LSlots& S = m2l_slots();
		LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_slot_dir, S.slot_dir, sizeof(S.slot_dir)));
		LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_dir_slot, S.dir_slot, sizeof(S.dir_slot)));
		uploaded = true;
	}
	size_t m = t.lsize[L];
	plan.cells = m;
	plan.vtab = static_cast<int32_t*>(ctx.arena.take(sizeof(int32_t) * m * M2L_SLOTS));
	plan.order = static_cast<int32_t*>(ctx.arena.take(sizeof(int32_t) * 2 * m));
	plan.oct_count = static_cast<uint32_t*>(ctx.arena.take(sizeof(uint32_t) * 16));
	if (!plan.vtab || !plan.order || !plan.oct_count) { ctx.last_error = "m2l plan: allocation failed"; return ERR_OOM; }
	cudaStream_t s = ctx.stream;
	LFMM_CUDA(ctx, cudaMemsetAsync(plan.vtab, 0xff, sizeof(int32_t) * m * M2L_SLOTS, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(plan.oct_count, 0, sizeof(uint32_t) * 16, s));
	count_oct_kernel<<<div_up(m, 256), 256, 0, s>>>(t, L, plan.oct_count);
	scatter_oct_kernel<<<div_up(m, 256), 256, 0, s>>>(t, L, plan.oct_count, plan.order);
	vtab_kernel<<<div_up(m, 128), 128, 0, s>>>(t, L, plan.vtab, ctx.dev_flags);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

template <typename real>
int m2l_gemm(Context& ctx, const M2LPlan& plan, const real* ops, const real* mult, real* loc, int N)
{
	const int R = N * (N + 1);
	const int MT = m2l_padded(N);
	const unsigned tiles = (unsigned)(plan.cells / M2L_TILE + 8);
	// spread the offsets of few tiles over several blocks (>= ~2 blocks per SM)
	int S = 1;
	while (S < 8 && tiles * S < 296) S *= 2;
	real* part = nullptr;
	if (S > 1) {
		part = static_cast<real*>(ctx.arena.take(sizeof(real) * (size_t)S * plan.cells * R));
		if (!part) S = 1;
	}
	dim3 grid(tiles, S);
	cudaStream_t s = ctx.stream;
	switch (MT / 16) {
	case 1: launch_gemm<real, 1>(grid, s, ops, mult, loc, plan, R, part); break;
	case 2: launch_gemm<real, 2>(grid, s, ops, mult, loc, plan, R, part); break;
	case 3: launch_gemm<real, 3>(grid, s, ops, mult, loc, plan, R, part); break;
	case 4: launch_gemm<real, 4>(grid, s, ops, mult, loc, plan, R, part); break;
	case 5: launch_gemm<real, 5>(grid, s, ops, mult, loc, plan, R, part); break;
	case 6: launch_gemm<real, 6>(grid, s, ops, mult, loc, plan, R, part); break;
	case 7: launch_gemm<real, 7>(grid, s, ops, mult, loc, plan, R, part); break;
	case 8: launch_gemm<real, 8>(grid, s, ops, mult, loc, plan, R, part); break;
	case 9: launch_gemm<real, 9>(grid, s, ops, mult, loc, plan, R, part); break;
	case 10: launch_gemm<real, 10>(grid, s, ops, mult, loc, plan, R, part); break;
	case 11: launch_gemm<real, 11>(grid, s, ops, mult, loc, plan, R, part); break;
	case 12: launch_gemm<real, 12>(grid, s, ops, mult, loc, plan, R, part); break;
	default: ctx.last_error = "m2l gemm: order too large"; return ERR_UNSUPPORTED;
	}
	if (S > 1) {
		size_t nel = plan.cells * (size_t)R;
		split_reduce_kernel<real><<<div_up(nel, 256), 256, 0, s>>>(part, loc, nel, S);
	}
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

template int m2l_gemm<double>(Context&, const M2LPlan&, const double*, const double*, double*, int);
template int m2l_gemm<float>(Context&, const M2LPlan&, const float*, const float*, float*, int);

// ======================================================================
// tcgen05 form (m2l_tc.cuh).  One CTA (128 threads) per tile of 128 targets
// of one octant class; D = T B accumulates in TMEM (lanes = output rows,
// columns = targets; two 128-row halves when the operator has > 128 rows).
// Per (offset, K block of 32 inputs): the operator block (hi, lo; stored
// pre-swizzled) is copied in with cp.async, the 128 gathered source columns
// are split into TF32 hi / lo and written in the 128-byte-swizzled K-major
// layout, then one thread issues 4 k-steps x 3 products x halves MMAs
// (M=128, N=128, K=8) and commits them to the stage's mbarrier.  Two stages
// alternate; every mbarrier wait is bounded and sets a device flag on expiry.
namespace {

constexpr int TC_BN = 128;
constexpr int TC_THREADS = 128;
constexpr uint32_t TC_IDESC = (1u << 4)        // D: FP32
                            | (2u << 7)        // A: TF32
                            | (2u << 10)       // B: TF32
                            | ((uint32_t)(TC_BN >> 3) << 17)   // N
                            | ((uint32_t)(128 >> 4) << 24);    // M

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
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
	uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
	d |= (uint64_t)1u << 16;
	d |= (uint64_t)(1024u >> 4) << 32;
	d |= (uint64_t)1u << 46;
	d |= (uint64_t)2u << 61;
	return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate)
{
	asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
	             "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
	             :: "r"(d_tmem), "l"(a), "l"(b), "r"(TC_IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
	for (int it = 0; it < (1 << 20); ++it) {
		uint32_t ok;
		asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
		if (ok) return true;
	}
	return false;
}

template <int MH, int KB>
__global__ void __launch_bounds__(TC_THREADS, 1) m2l_tc_kernel(const uint4* __restrict__ ops, const float* __restrict__ mult,
                                                               float* __restrict__ loc, const int32_t* __restrict__ vtab,
                                                               const int32_t* __restrict__ order,
                                                               const uint32_t* __restrict__ oct_count, int R, unsigned* flags)
{
	constexpr int HALF = 128 * 128;                 // bytes of one 128-row half (128 B rows)
	constexpr int A_BYTES = 2 * MH * HALF;          // hi halves, then lo halves
	constexpr int B_BYTES = 2 * TC_BN * 128;        // hi, then lo
	constexpr int STAGE = A_BYTES + B_BYTES;
	// two accumulators: main (hi x hi) and correction (hi x lo + lo x hi).  The
	// tensor core aligns each product to the largest addend before adding, so
	// the small corrections keep their bits only if summed on their own.
	constexpr uint32_t TMEM_COLS = MH == 1 ? 256 : 512;
	constexpr uint32_t CORR = MH * TC_BN;     // column offset of the correction accumulator
	extern __shared__ uint8_t dsm[];
	__shared__ uint64_t bars[2];
	__shared__ uint32_t tmem_sh;
	__shared__ int32_t tgt[TC_BN];
	__shared__ int s_oct, s_n;
	__shared__ uint32_t s_start;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	uint8_t* base = dsm + ((1024u - (smem_u32(dsm) & 1023u)) & 1023u);
	if (tid == 0) {
		uint32_t b = blockIdx.x, start = 0;
		int oct = -1, nn = 0;
		for (int o = 0; o < 8; ++o) {
			uint32_t cnt = oct_count[o];
			uint32_t tiles = (cnt + TC_BN - 1) / TC_BN;
			if (b < tiles) { oct = o; start += b * TC_BN; nn = (int)min((uint32_t)TC_BN, cnt - b * TC_BN); break; }
			b -= tiles; start += cnt;
		}
		s_oct = oct; s_n = nn; s_start = start;
	}
	__syncthreads();
	if (s_oct < 0) return;
	const int oct = s_oct;
	tgt[tid] = tid < s_n ? order[s_start + tid] : -1;
	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		             :: "r"(smem_u32(&tmem_sh)), "r"(TMEM_COLS));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
	}
	if (tid == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&bars[0])));
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&bars[1])));
		asm volatile("fence.mbarrier_init.release.cluster;");
	}
	asm volatile("tcgen05.fence::before_thread_sync;");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;");
	const uint32_t tmem = tmem_sh;
	const int myt = tgt[tid];
	uint32_t it = 0;
	bool ok = true;
	for (int slot = 0; slot < M2L_SLOTS; ++slot) {
		const int s_ = myt >= 0 ? vtab[(size_t)myt * M2L_SLOTS + slot] : -1;
		if (!__syncthreads_or(s_ >= 0)) continue;
		const int dir = c_slot_dir[oct][slot];
		for (int kb = 0; kb < KB; ++kb) {
			const uint32_t st = it & 1u;
			uint8_t* sA = base + st * STAGE;
			uint8_t* sB = sA + A_BYTES;
			if (it >= 2 && !mbar_wait(smem_u32(&bars[st]), ((it >> 1) - 1) & 1u)) ok = false;
			if (!__syncthreads_and(ok)) { ok = false; break; }
			const uint4* gA = ops + ((size_t)dir * KB + kb) * (A_BYTES / 16);
			const uint32_t sa = smem_u32(sA);
			for (int c = tid; c < A_BYTES / 16; c += TC_THREADS)
				asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(sa + 16u * c), "l"(gA + c) : "memory");
			asm volatile("cp.async.commit_group;" ::: "memory");
			{
				float v[32];
				if (s_ >= 0) {
					const float2* p = reinterpret_cast<const float2*>(mult + (size_t)s_ * R + kb * 32);
#pragma unroll
					for (int j = 0; j < 16; ++j) {
						const int k = kb * 32 + 2 * j;
						float2 w = k < R ? p[j] : make_float2(0.f, 0.f);   // R is even: pairs stay in range
						v[2 * j] = w.x; v[2 * j + 1] = w.y;
					}
				} else {
#pragma unroll
					for (int j = 0; j < 32; ++j) v[j] = 0.f;
				}
				uint8_t* rh = sB + tid * 128;
				uint8_t* rl = sB + TC_BN * 128 + tid * 128;
#pragma unroll
				for (int c = 0; c < 8; ++c) {
					uint32_t h[4], l[4];
#pragma unroll
					for (int e = 0; e < 4; ++e) {
						const float x = v[4 * c + e];
						h[e] = tf32_rna(x);
						l[e] = tf32_rna(x - __uint_as_float(h[e]));
					}
					const int pc = c ^ (tid & 7);
					*reinterpret_cast<uint4*>(rh + pc * 16) = make_uint4(h[0], h[1], h[2], h[3]);
					*reinterpret_cast<uint4*>(rl + pc * 16) = make_uint4(l[0], l[1], l[2], l[3]);
				}
			}
			asm volatile("cp.async.wait_all;" ::: "memory");
			asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
			asm volatile("tcgen05.fence::before_thread_sync;");
			__syncthreads();
			asm volatile("tcgen05.fence::after_thread_sync;");
			if (tid == 0) {
				const uint32_t sb = smem_u32(sB);
#pragma unroll
				for (int ks = 0; ks < 4; ++ks) {
					const uint64_t bh = umma_desc_sw128(sb + ks * 32);
					const uint64_t bl = umma_desc_sw128(sb + TC_BN * 128 + ks * 32);
#pragma unroll
					for (int h = 0; h < MH; ++h) {
						const uint64_t ah = umma_desc_sw128(sa + h * HALF + ks * 32);
						const uint64_t al = umma_desc_sw128(sa + MH * HALF + h * HALF + ks * 32);
						const uint32_t d = tmem + (uint32_t)(h * TC_BN);
						const uint32_t first = (it == 0 && ks == 0) ? 0u : 1u;
						mma_tf32(d, ah, bh, first);
						mma_tf32(d + CORR, ah, bl, first);
						mma_tf32(d + CORR, al, bh, 1u);
					}
				}
				asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
				             :: "r"(smem_u32(&bars[st])) : "memory");
			}
			++it;
		}
		if (!ok) break;
	}
	if (ok && it > 0 && !mbar_wait(smem_u32(&bars[(it - 1) & 1u]), ((it - 1) >> 1) & 1u)) ok = false;
	ok = __syncthreads_and(ok);
	asm volatile("tcgen05.fence::after_thread_sync;");
	if (!ok) {
		if (tid == 0) atomicOr(flags, DEV_ERR_TIMEOUT);
		// give the other stage's MMAs a bounded chance to drain before freeing TMEM
		if (it > 1) mbar_wait(smem_u32(&bars[it & 1u]), ((it >> 1) - 1) & 1u);
	} else {
#pragma unroll
		for (int h = 0; h < MH; ++h) {
			for (int cc = 0; cc < TC_BN / 16; ++cc) {
				uint32_t r[16], rc[16];
				if (it > 0) {
					const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(h * TC_BN + cc * 16);
					asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
					             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
					               "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
					               "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
					             : "r"(ta));
					asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
					             : "=r"(rc[0]), "=r"(rc[1]), "=r"(rc[2]), "=r"(rc[3]), "=r"(rc[4]), "=r"(rc[5]), "=r"(rc[6]),
					               "=r"(rc[7]), "=r"(rc[8]), "=r"(rc[9]), "=r"(rc[10]), "=r"(rc[11]), "=r"(rc[12]),
					               "=r"(rc[13]), "=r"(rc[14]), "=r"(rc[15])
					             : "r"(ta + CORR));
					asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
				} else {
#pragma unroll
					for (int j = 0; j < 16; ++j) { r[j] = 0u; rc[j] = 0u; }
				}
				const int row = h * 128 + warp * 32 + lane;
				if (row < R) {
#pragma unroll
					for (int j = 0; j < 16; ++j) {
						const int tg = tgt[cc * 16 + j];
						if (tg >= 0) loc[(size_t)tg * R + row] = __uint_as_float(r[j]) + __uint_as_float(rc[j]);
					}
				}
			}
		}
	}
	asm volatile("tcgen05.fence::before_thread_sync;");
	__syncthreads();
	if (warp == 0)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TMEM_COLS));
}

// FP64 scaled operators -> tensor-core layout (see m2l_tc.cuh)
__global__ void build_tc_ops_kernel(const double* __restrict__ ops64, int MT, int R, int MH, int KB,
                                    uint32_t* __restrict__ out)
{
	const size_t rows = (size_t)MH * 128;
	const size_t total = (size_t)343 * KB * 2 * rows * 32;
	size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= total) return;
	const int j = (int)(e % 32);
	size_t rest = e / 32;
	const int row = (int)(rest % rows); rest /= rows;
	const int x = (int)(rest % 2); rest /= 2;
	const int kb = (int)(rest % KB);
	const int dir = (int)(rest / KB);
	const int k = kb * 32 + j;
	const double v = (row < R && k < R) ? ops64[((size_t)dir * MT + row) * MT + k] : 0.0;
	const uint32_t hi = tf32_rna((float)v);
	const uint32_t lo = tf32_rna((float)(v - (double)__uint_as_float(hi)));
	const int h = row / 128, r = row % 128;
	const size_t off = (size_t)h * 16384 + (size_t)r * 128 + (size_t)(((j >> 2) ^ (r & 7)) * 16) + (size_t)(j & 3) * 4;
	const size_t blk = ((size_t)dir * KB + kb) * 2 + x;
	out[(blk * rows * 128 + off) / 4] = x == 0 ? hi : lo;
}

template <int MH, int KB>
int launch_tc(Context& ctx, const M2LPlan& plan, const uint4* ops, const float* mult, float* loc, int R)
{
	constexpr int STAGE = 2 * MH * 16384 + 2 * TC_BN * 128;
	const int smem = 2 * STAGE + 1024;
	static bool attr = false;
	if (!attr) {
		LFMM_CUDA(ctx, cudaFuncSetAttribute(m2l_tc_kernel<MH, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
		attr = true;
	}
	const unsigned grid = (unsigned)(plan.cells / TC_BN + 8);
	m2l_tc_kernel<MH, KB><<<grid, TC_THREADS, smem, ctx.stream>>>(ops, mult, loc, plan.vtab, plan.order, plan.oct_count,
	                                                              R, ctx.dev_flags);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

} // namespace

const uint4* m2l_ops_tc(Context& ctx, int N)
{
	for (auto& e : ctx.opcache)
		if (e.N == N && e.prec == 2) { e.stamp = ++ctx.opcache_clock; return static_cast<const uint4*>(e.ptr); }
	double* d = m2l_ops_fp64(ctx, N, 1.0);
	if (!d) return nullptr;
	const int MT = m2l_padded(N), R = N * (N + 1), MH = m2l_tc_halves(N), KB = m2l_tc_kblocks(N);
	const size_t words = (size_t)343 * KB * 2 * MH * 128 * 32;
	OpCacheEntry e;
	e.N = N; e.prec = 2; e.h = 1.0; e.bytes = words * 4; e.stamp = ++ctx.opcache_clock;
	if (cudaMalloc(&e.ptr, e.bytes) != cudaSuccess) { cudaGetLastError(); ctx.last_error = "tc operators: out of memory"; return nullptr; }
	build_tc_ops_kernel<<<div_up(words, 256), 256, 0, ctx.stream>>>(d, MT, R, MH, KB, static_cast<uint32_t*>(e.ptr));
	ctx.opcache.push_back(e);
	return static_cast<const uint4*>(e.ptr);
}

int m2l_gemm_tc(Context& ctx, const M2LPlan& plan, const uint4* ops, const float* mult, float* loc, int N)
{
	const int R = N * (N + 1), MH = m2l_tc_halves(N), KB = m2l_tc_kblocks(N);
	if (MH == 1 && KB == 1) return launch_tc<1, 1>(ctx, plan, ops, mult, loc, R);
	if (MH == 1 && KB == 2) return launch_tc<1, 2>(ctx, plan, ops, mult, loc, R);
	if (MH == 1 && KB == 3) return launch_tc<1, 3>(ctx, plan, ops, mult, loc, R);
	if (MH == 1 && KB == 4) return launch_tc<1, 4>(ctx, plan, ops, mult, loc, R);
	if (MH == 2 && KB == 5) return launch_tc<2, 5>(ctx, plan, ops, mult, loc, R);
	if (MH == 2 && KB == 6) return launch_tc<2, 6>(ctx, plan, ops, mult, loc, R);
	ctx.last_error = "tensor-core M2L: unsupported order";
	return ERR_UNSUPPORTED;
}

} // namespace lfmm
