// Direction-grouped M2L GEMMs (see m2l_gemm.cuh), SIMT register-tiled form
// for FP64 (plain) and FP32.
#include "m2l_gemm.cuh"
#include "fmm3d.cuh"
#include "primitives.cuh"
#include <mutex>
#include <cstdlib>

namespace lfmm {

namespace {

__constant__ int16_t c_slot_dir[8][M2L_SLOTS];
__constant__ int16_t c_dir_slot[8][343];
// 2D: 4 child classes x 27 far offsets, direction id (dx + 3) * 7 + (dy + 3)
__constant__ int16_t c_slot_dir2[4][M2L_SLOTS2];
__constant__ int16_t c_dir_slot2[4][49];

template <int DIM> struct GemmDim;
template <> struct GemmDim<3> {
	static constexpr int SLOTS = M2L_SLOTS, CLASSES = 8;
	__device__ static int dir(int cls, int slot) { return c_slot_dir[cls][slot]; }
};
template <> struct GemmDim<2> {
	static constexpr int SLOTS = M2L_SLOTS2, CLASSES = 4;
	__device__ static int dir(int cls, int slot) { return c_slot_dir2[cls][slot]; }
};

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

// ---- 2D: quadrant classes, slot table, dense complex M2L operators ----------

__device__ __forceinline__ void coords2g(uint64_t code, int* c) { c[0] = (int)compact2(code >> 1); c[1] = (int)compact2(code); }

__global__ void count_cls2_kernel(DevTree t, int L, uint32_t* __restrict__ cnt)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= t.lsize[L]) return;
	int me[2];
	coords2g(t.code[t.loff[L] + c], me);
	atomicAdd(&cnt[((me[0] & 1) << 1) | (me[1] & 1)], 1u);
}

__global__ void scatter_cls2_kernel(DevTree t, int L, uint32_t* __restrict__ cnt, int32_t* __restrict__ order)
{
	__shared__ uint32_t base[4];
	if (threadIdx.x < 4) {
		uint32_t a = 0;
		for (int o = 0; o < (int)threadIdx.x; ++o) a += cnt[o];
		base[threadIdx.x] = a;
	}
	__syncthreads();
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= t.lsize[L]) return;
	int me[2];
	coords2g(t.code[t.loff[L] + c], me);
	const int cls = ((me[0] & 1) << 1) | (me[1] & 1);
	order[base[cls] + atomicAdd(&cnt[8 + cls], 1u)] = (int32_t)c;
}

// The 2D far list (children of the parent's close cells and of the parent
// that are not adjacent, reference cpu/morton_tree.cpp:147-208) as slots.
__global__ void vtab2_kernel(DevTree t, int L, int32_t* __restrict__ vtab, unsigned* flags)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	size_t m = t.lsize[L];
	if (c >= m) return;
	size_t off = t.loff[L], poff = t.loff[L - 1];
	int me[2];
	coords2g(t.code[off + c], me);
	const int cls = ((me[0] & 1) << 1) | (me[1] & 1);
	int32_t* row = vtab + c * M2L_SLOTS2;
	int32_t p = t.parent[off + c];
	int npc = t.close_cnt[poff + p];
	const int32_t* pl = t.close_idx + (poff + p) * t.close_stride;
	for (int e = 0; e <= npc; ++e) {
		int32_t pn = e < npc ? pl[e] : p;
		for (uint32_t k = t.beg[poff + pn]; k < t.end[poff + pn]; ++k) {
			if (k == c) continue;
			int o[2];
			coords2g(t.code[off + k], o);
			int dx = o[0] - me[0], dy = o[1] - me[1];
			if (max(abs(dx), abs(dy)) <= 1) continue;
			int slot = (abs(dx) <= 3 && abs(dy) <= 3) ? c_dir_slot2[cls][(dx + 3) * 7 + (dy + 3)] : -1;
			if (slot < 0) { atomicOr(flags, DEV_ERR_DIRECTION); continue; }
			row[slot] = (int32_t)k;
		}
	}
}

// Dense 2D M2L for offset d (cells of size h, z0 = d h = source - target),
// complex coefficients as 2 x 2 real blocks of [MT][MT] (reference
// cpu/multipole.cpp:66-84): b_0 += a_0 conj(log(-z0)) + sum_{j>=1} (-1)^j a_j / z0^j,
// b_i += -a_0 / (i z0^i) + sum_{j>=1} (-1)^j C(i+j-1, j-1) a_j / z0^(i+j).
__global__ void m2l_ops2d_kernel(int N, int MT, double h, double* __restrict__ ops)
{
	const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= (size_t)49 * N * N) return;
	const int j = (int)(e % N), i = (int)((e / N) % N), d = (int)(e / ((size_t)N * N));
	const int dx = d / 7 - 3, dy = d % 7 - 3;
	if (max(abs(dx), abs(dy)) <= 1) return;
	const double zx = dx * h, zy = dy * h;
	double cr, ci;
	if (i == 0 && j == 0) {
		cr = log(sqrt(zx * zx + zy * zy));
		ci = -atan2(-zy, -zx);
	} else {
		// 1 / z0^k, k = i + j
		const double r2 = zx * zx + zy * zy;
		const double ix = zx / r2, iy = -zy / r2;
		double px = 1.0, py = 0.0;
		for (int k = 0; k < i + j; ++k) { const double nx = px * ix - py * iy; py = px * iy + py * ix; px = nx; }
		double f;
		if (i == 0) f = (j & 1) ? -1.0 : 1.0;
		else if (j == 0) f = -1.0 / i;
		else {
			double b = 1.0;                          // C(i + j - 1, j - 1)
			for (int k = 1; k <= j - 1; ++k) b = b * (double)(i + k) / (double)k;
			f = ((j & 1) ? -1.0 : 1.0) * b;
		}
		cr = f * px; ci = f * py;
	}
	double* T = ops + (size_t)d * MT * MT;
	T[(size_t)(2 * i) * MT + 2 * j] = cr;
	T[(size_t)(2 * i) * MT + 2 * j + 1] = -ci;
	T[(size_t)(2 * i + 1) * MT + 2 * j] = ci;
	T[(size_t)(2 * i + 1) * MT + 2 * j + 1] = cr;
}

// The same operator factored through one real Hankel matrix shared by every
// offset and level: T = diag(post) H diag(pre) plus the log term, with
// H[i][j] = (i+j-1)! (H[0][0] = 0), pre_0 = -1, pre_j = (-1)^j / ((j-1)! z0^j),
// post_i = 1 / (i! z0^i) and b_0 += a_0 conj(log(-z0)).  The per-offset
// vectors of one level: tab[d] = pre[0..N), post[0..N), log term.
__constant__ double c_fact[64];        // k!

__global__ void m2l2d_tab_kernel(int N, double h, double2* __restrict__ tab)
{
	const int W = 2 * N + 1;
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= 49 * W) return;
	const int d = e / W, k = e - d * W;
	const int dx = d / 7 - 3, dy = d % 7 - 3;
	if (max(abs(dx), abs(dy)) <= 1) { tab[e] = make_double2(0.0, 0.0); return; }
	const double zx = dx * h, zy = dy * h;
	if (k == 2 * N) { tab[e] = make_double2(log(sqrt(zx * zx + zy * zy)), -atan2(-zy, -zx)); return; }
	const int p = k < N ? k : k - N;           // power of 1 / z0
	if (k == 0) { tab[e] = make_double2(-1.0, 0.0); return; }
	const double r2 = zx * zx + zy * zy;
	const double ix = zx / r2, iy = -zy / r2;
	double px = 1.0, py = 0.0;
	for (int q = 0; q < p; ++q) { const double nx = px * ix - py * iy; py = px * iy + py * ix; px = nx; }
	const double f = k < N ? ((p & 1) ? -1.0 : 1.0) / c_fact[p - 1] : 1.0 / c_fact[p];
	tab[e] = make_double2(f * px, f * py);
}

// Block of 128 threads per (quadrant class, tile of 64 targets) and slot
// range; thread (ty, tx) owns rows ty + 4 r (r < TM) of targets tx and tx + 32.
// Per slot: W = pre (.) a (gathered sources), S = H W, b += post (.) S.
template <int TM>
__global__ void __launch_bounds__(128) m2l2d_hankel_kernel(const double2* __restrict__ tab,
                                                           const double2* __restrict__ mult, double2* __restrict__ loc,
                                                           const int32_t* __restrict__ vtab,
                                                           const int32_t* __restrict__ order,
                                                           const uint32_t* __restrict__ cls_count, int N,
                                                           double2* __restrict__ part, size_t cells)
{
	const int S = gridDim.y, sidx = blockIdx.y;
	const int slot0 = sidx * M2L_SLOTS2 / S, slot1 = (sidx + 1) * M2L_SLOTS2 / S;
	if (S > 1) loc = part + (size_t)sidx * cells * N;
	__shared__ double Wr[32][65], Wi[32][65];
	__shared__ double sH[64];
	__shared__ double2 spost[32];
	__shared__ double2 slg;
	__shared__ int32_t src[64], tgt[64];
	__shared__ int s_cls, s_n;
	__shared__ uint32_t s_start;
	const int tid = threadIdx.x, ty = tid >> 5, tx = tid & 31;
	if (tid == 0) {
		uint32_t b = blockIdx.x, start = 0;
		int cls = -1, nn = 0;
		for (int o = 0; o < 4; ++o) {
			const uint32_t cnt = cls_count[o], tiles = (cnt + 63) / 64;
			if (b < tiles) { cls = o; start += b * 64; nn = (int)min(64u, cnt - b * 64); break; }
			b -= tiles; start += cnt;
		}
		s_cls = cls; s_n = nn; s_start = start;
	}
	if (tid < 64) sH[tid] = tid == 0 ? 0.0 : c_fact[tid - 1];
	__syncthreads();
	const int cls = s_cls;
	if (cls < 0) return;
	if (tid < 64) tgt[tid] = tid < s_n ? order[s_start + tid] : -1;
	double ar[TM][2], ai[TM][2];
#pragma unroll
	for (int r = 0; r < TM; ++r) { ar[r][0] = ar[r][1] = ai[r][0] = ai[r][1] = 0.0; }
	__syncthreads();
	for (int slot = slot0; slot < slot1; ++slot) {
		int mine = -1;
		if (tid < 64 && tgt[tid] >= 0) mine = vtab[(size_t)tgt[tid] * M2L_SLOTS2 + slot];
		if (tid < 64) src[tid] = mine;
		if (!__syncthreads_or(mine >= 0)) continue;
		const double2* T = tab + (size_t)c_slot_dir2[cls][slot] * (2 * N + 1);
		if (tid < N) spost[tid] = T[N + tid];
		if (tid == 0) slg = T[2 * N];
		for (int idx = tid; idx < 64 * N; idx += 128) {
			const int c = idx / N, k = idx - c * N;
			const int s = src[c];
			const double2 a = s >= 0 ? mult[(size_t)s * N + k] : make_double2(0.0, 0.0);
			const double2 p = T[k];
			Wr[k][c] = a.x * p.x - a.y * p.y;
			Wi[k][c] = a.x * p.y + a.y * p.x;
		}
		__syncthreads();
		double sr[TM][2], si[TM][2];
#pragma unroll
		for (int r = 0; r < TM; ++r) { sr[r][0] = sr[r][1] = si[r][0] = si[r][1] = 0.0; }
		for (int k = 0; k < N; ++k) {
			const double br0 = Wr[k][tx], br1 = Wr[k][tx + 32], bi0 = Wi[k][tx], bi1 = Wi[k][tx + 32];
#pragma unroll
			for (int r = 0; r < TM; ++r) {
				const double hk = sH[ty + 4 * r + k];
				sr[r][0] = fma(hk, br0, sr[r][0]); sr[r][1] = fma(hk, br1, sr[r][1]);
				si[r][0] = fma(hk, bi0, si[r][0]); si[r][1] = fma(hk, bi1, si[r][1]);
			}
		}
#pragma unroll
		for (int r = 0; r < TM; ++r) {
			const int i = ty + 4 * r;
			if (i < N) {
				const double2 p = spost[i];
#pragma unroll
				for (int j = 0; j < 2; ++j) {
					ar[r][j] += p.x * sr[r][j] - p.y * si[r][j];
					ai[r][j] += p.x * si[r][j] + p.y * sr[r][j];
				}
			}
		}
		if (ty == 0) {                         // b_0 += a_0 lg, a_0 = -W[0]
			const double2 lg = slg;
#pragma unroll
			for (int j = 0; j < 2; ++j) {
				const double a0r = -Wr[0][tx + 32 * j], a0i = -Wi[0][tx + 32 * j];
				ar[0][j] += a0r * lg.x - a0i * lg.y;
				ai[0][j] += a0r * lg.y + a0i * lg.x;
			}
		}
		__syncthreads();
	}
#pragma unroll
	for (int j = 0; j < 2; ++j) {
		const int tg = tgt[tx + 32 * j];
		if (tg < 0) continue;
#pragma unroll
		for (int r = 0; r < TM; ++r) {
			const int i = ty + 4 * r;
			if (i < N) loc[(size_t)tg * N + i] = make_double2(ar[r][j], ai[r][j]);
		}
	}
}

// C[MT x 64] = sum over the octant's offsets of T_dir[MT x MT] * B[MT x 64];
// 256 threads, thread (ty, tx) owns rows ty + 16 i and columns tx + 16 j.
// blockIdx.y = split s of S: slots [s*189/S, (s+1)*189/S); with S > 1 the
// partial sums go to part[s][cell][R] and a fixed-order reduction follows.
template <typename real, int TM, int TN, int DIM = 3>
__global__ void __launch_bounds__(256) m2l_gemm_kernel(const real* __restrict__ ops, const real* __restrict__ mult,
                                                       real* __restrict__ loc, const int32_t* __restrict__ vtab,
                                                       const int32_t* __restrict__ order,
                                                       const uint32_t* __restrict__ oct_count, int R,
                                                       real* __restrict__ part, size_t cells)
{
	const int S = gridDim.y, sidx = blockIdx.y;
	constexpr int SLOTS = GemmDim<DIM>::SLOTS;
	const int slot0 = sidx * SLOTS / S, slot1 = (sidx + 1) * SLOTS / S;
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
		for (int o = 0; o < GemmDim<DIM>::CLASSES; ++o) {
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
		if (tid < BN && tgt[tid] >= 0) mine = vtab[(size_t)tgt[tid] * SLOTS + slot];
		if (tid < BN) src[tid] = mine;
		if (!__syncthreads_or(mine >= 0)) continue;
		if constexpr (sizeof(real) == sizeof(float)) {
#pragma unroll
			for (int i = 0; i < TM; ++i)
#pragma unroll
				for (int j = 0; j < TN; ++j) part_[i][j] = real(0);
		}
		const real* A = ops + (size_t)GemmDim<DIM>::dir(oct, slot) * MT * MT;
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

template <typename real, int TM, int DIM>
void launch_gemm(dim3 grid, cudaStream_t s, const real* ops, const real* mult, real* loc, const M2LPlan& p, int R,
                 real* part)
{
	m2l_gemm_kernel<real, TM, 4, DIM><<<grid, 256, 0, s>>>(ops, mult, loc, p.vtab, p.order, p.oct_count, R, part,
	                                                         p.cells);
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

namespace {

std::mutex g_slots_mu;
bool g_slots_uploaded[64] = {};

// slot tables of both dimensions, once per device
int upload_slots(Context& ctx)
{
	std::lock_guard<std::mutex> lock(g_slots_mu);
	if (ctx.device < 0 || ctx.device >= 64) { ctx.last_error = "device index above 63"; return ERR_ARG; }
	if (g_slots_uploaded[ctx.device]) return OK;
	const M2LSlots& S = m2l_slots();
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_slot_dir, S.slot_dir, sizeof(S.slot_dir)));
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_dir_slot, S.dir_slot, sizeof(S.dir_slot)));
	int16_t sd[4][M2L_SLOTS2], ds[4][49];
	for (int o = 0; o < 4; ++o) {
		for (int d = 0; d < 49; ++d) ds[o][d] = -1;
		const int ox = (o >> 1) & 1, oy = o & 1;
		int s = 0;
		for (int dx = -2 - ox; dx <= 3 - ox; ++dx)
			for (int dy = -2 - oy; dy <= 3 - oy; ++dy) {
				if (std::max(std::abs(dx), std::abs(dy)) <= 1) continue;
				const int id = (dx + 3) * 7 + (dy + 3);
				sd[o][s] = (int16_t)id;
				ds[o][id] = (int16_t)s;
				++s;
			}
	}
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_slot_dir2, sd, sizeof(sd)));
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_dir_slot2, ds, sizeof(ds)));
	double fact[64];
	fact[0] = 1.0;
	for (int k = 1; k < 64; ++k) fact[k] = fact[k - 1] * k;
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_fact, fact, sizeof(fact)));
	g_slots_uploaded[ctx.device] = true;
	return OK;
}

} // namespace

int m2l_plan_build2d(Context& ctx, const DevTree& t, int L, M2LPlan& plan)
{
	if (int st = upload_slots(ctx)) return st;
	size_t m = t.lsize[L];
	plan.cells = m;
	plan.vtab = static_cast<int32_t*>(ctx.arena.take(sizeof(int32_t) * m * M2L_SLOTS2));
	plan.order = static_cast<int32_t*>(ctx.arena.take(sizeof(int32_t) * 2 * m));
	plan.oct_count = static_cast<uint32_t*>(ctx.arena.take(sizeof(uint32_t) * 16));
	if (!plan.vtab || !plan.order || !plan.oct_count) { ctx.last_error = "m2l plan: allocation failed"; return ERR_OOM; }
	cudaStream_t s = ctx.stream;
	LFMM_CUDA(ctx, cudaMemsetAsync(plan.vtab, 0xff, sizeof(int32_t) * m * M2L_SLOTS2, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(plan.oct_count, 0, sizeof(uint32_t) * 16, s));
	count_cls2_kernel<<<div_up(m, 256), 256, 0, s>>>(t, L, plan.oct_count);
	scatter_cls2_kernel<<<div_up(m, 256), 256, 0, s>>>(t, L, plan.oct_count, plan.order);
	vtab2_kernel<<<div_up(m, 128), 128, 0, s>>>(t, L, plan.vtab, ctx.dev_flags);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

double* m2l_ops2d(Context& ctx, int N, double h)
{
	for (auto& e : ctx.opcache)
		if (e.N == N && e.prec == 20 && e.h == h) { e.stamp = ++ctx.opcache_clock; return static_cast<double*>(e.ptr); }
	const int MT = (2 * N + 15) / 16 * 16;
	opcache_make_room(ctx);
	OpCacheEntry e;
	e.N = N; e.prec = 20; e.h = h; e.bytes = sizeof(double) * 49 * (size_t)MT * MT; e.stamp = ++ctx.opcache_clock;
	if (cudaMalloc(&e.ptr, e.bytes) != cudaSuccess) { cudaGetLastError(); ctx.last_error = "2D m2l operators: out of memory"; return nullptr; }
	cudaMemsetAsync(e.ptr, 0, e.bytes, ctx.stream);
	const size_t tasks = (size_t)49 * N * N;
	m2l_ops2d_kernel<<<div_up(tasks, 256), 256, 0, ctx.stream>>>(N, MT, h, static_cast<double*>(e.ptr));
	if (cudaGetLastError() != cudaSuccess) { cudaFree(e.ptr); ctx.last_error = "2D m2l operators: launch failed"; return nullptr; }
	ctx.opcache.push_back(e);
	return static_cast<double*>(e.ptr);
}

double2* m2l_tab2d(Context& ctx, int N, double h)
{
	for (auto& e : ctx.opcache)
		if (e.N == N && e.prec == 21 && e.h == h) { e.stamp = ++ctx.opcache_clock; return static_cast<double2*>(e.ptr); }
	if (upload_slots(ctx)) return nullptr;
	opcache_make_room(ctx);
	OpCacheEntry e;
	e.N = N; e.prec = 21; e.h = h; e.bytes = sizeof(double2) * 49 * (size_t)(2 * N + 1); e.stamp = ++ctx.opcache_clock;
	if (cudaMalloc(&e.ptr, e.bytes) != cudaSuccess) { cudaGetLastError(); ctx.last_error = "2D m2l tables: out of memory"; return nullptr; }
	const int cnt = 49 * (2 * N + 1);
	m2l2d_tab_kernel<<<div_up(cnt, 128), 128, 0, ctx.stream>>>(N, h, static_cast<double2*>(e.ptr));
	if (cudaGetLastError() != cudaSuccess) { cudaFree(e.ptr); ctx.last_error = "2D m2l tables: launch failed"; return nullptr; }
	ctx.opcache.push_back(e);
	return static_cast<double2*>(e.ptr);
}

int m2l_hankel2d(Context& ctx, const M2LPlan& plan, const double2* tab, const double2* mult, double2* loc, int N)
{
	if (N < 1 || N > 32) { ctx.last_error = "2D m2l: order too large"; return ERR_UNSUPPORTED; }
	const unsigned tiles = (unsigned)(plan.cells / 64 + 4);
	int S = 1;
	while (S < 8 && tiles * S < 4u * (unsigned)ctx.num_sms) S *= 2;
	double2* part = nullptr;
	if (S > 1) {
		part = static_cast<double2*>(ctx.arena.take(sizeof(double2) * (size_t)S * plan.cells * N));
		if (!part) S = 1;
	}
	const dim3 grid(tiles, S);
	cudaStream_t s = ctx.stream;
	const int TM = N <= 8 ? 2 : N <= 16 ? 4 : N <= 24 ? 6 : 8;
	switch (TM) {
	case 2: m2l2d_hankel_kernel<2><<<grid, 128, 0, s>>>(tab, mult, loc, plan.vtab, plan.order, plan.oct_count, N, part, plan.cells); break;
	case 4: m2l2d_hankel_kernel<4><<<grid, 128, 0, s>>>(tab, mult, loc, plan.vtab, plan.order, plan.oct_count, N, part, plan.cells); break;
	case 6: m2l2d_hankel_kernel<6><<<grid, 128, 0, s>>>(tab, mult, loc, plan.vtab, plan.order, plan.oct_count, N, part, plan.cells); break;
	default: m2l2d_hankel_kernel<8><<<grid, 128, 0, s>>>(tab, mult, loc, plan.vtab, plan.order, plan.oct_count, N, part, plan.cells); break;
	}
	if (S > 1) {
		const size_t nel = plan.cells * (size_t)N * 2;
		split_reduce_kernel<double><<<div_up(nel, 256), 256, 0, s>>>(reinterpret_cast<const double*>(part),
		                                                             reinterpret_cast<double*>(loc), nel, S);
	}
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

int m2l_plan_build(Context& ctx, const DevTree& t, int L, M2LPlan& plan)
{
	if (int st = upload_slots(ctx)) return st;
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

namespace {

template <typename real, int DIM>
int gemm_rt(Context& ctx, const M2LPlan& plan, const real* ops, const real* mult, real* loc, int R, int MT)
{
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
	if constexpr (DIM == 2) {
		switch (MT / 16) {
		case 1: launch_gemm<real, 1, 2>(grid, s, ops, mult, loc, plan, R, part); break;
		case 2: launch_gemm<real, 2, 2>(grid, s, ops, mult, loc, plan, R, part); break;
		case 3: launch_gemm<real, 3, 2>(grid, s, ops, mult, loc, plan, R, part); break;
		case 4: launch_gemm<real, 4, 2>(grid, s, ops, mult, loc, plan, R, part); break;
		default: ctx.last_error = "2D m2l gemm: order too large"; return ERR_UNSUPPORTED;
		}
	} else switch (MT / 16) {
	case 1: launch_gemm<real, 1, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 2: launch_gemm<real, 2, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 3: launch_gemm<real, 3, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 4: launch_gemm<real, 4, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 5: launch_gemm<real, 5, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 6: launch_gemm<real, 6, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 7: launch_gemm<real, 7, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 8: launch_gemm<real, 8, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 9: launch_gemm<real, 9, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 10: launch_gemm<real, 10, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 11: launch_gemm<real, 11, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 12: launch_gemm<real, 12, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 14: launch_gemm<real, 14, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	case 15: launch_gemm<real, 15, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
	default: ctx.last_error = "m2l gemm: order too large"; return ERR_UNSUPPORTED;
	}
	if (S > 1) {
		size_t nel = plan.cells * (size_t)R;
		split_reduce_kernel<real><<<div_up(nel, 256), 256, 0, s>>>(part, loc, nel, S);
	}
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

} // namespace

template <typename real>
int m2l_gemm(Context& ctx, const M2LPlan& plan, const real* ops, const real* mult, real* loc, int N)
{
	return gemm_rt<real, 3>(ctx, plan, ops, mult, loc, N * (N + 1), m2l_padded(N));
}

int m2l_gemm2d(Context& ctx, const M2LPlan& plan, const double* ops, const double* mult, double* loc, int N)
{
	return gemm_rt<double, 2>(ctx, plan, ops, mult, loc, 2 * N, (2 * N + 15) / 16 * 16);
}

template int m2l_gemm<double>(Context&, const M2LPlan&, const double*, const double*, double*, int);
template int m2l_gemm<float>(Context&, const M2LPlan&, const float*, const float*, float*, int);

} // namespace lfmm
