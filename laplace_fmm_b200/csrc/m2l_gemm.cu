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
__device__ int16_t g_dir_slot[8][343];    // global: vtab_kernel stages it in shared memory
// 2D: 4 child classes x 27 far offsets, direction id (dx + 3) * 7 + (dy + 3)
__constant__ int16_t c_slot_dir2[4][M2L_SLOTS2];
__device__ int16_t g_dir_slot2[4][49];    // global: vtab2_kernel stages it in shared memory

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
// and of the parent (reference cpu/morton_tree.cpp:147-208).  A warp per
// target cell: the row is first set to -1, then lane e places the far
// children of the parent's e-th close cell (the parent itself last), so
// every store of the warp lands in the same row.
__global__ void vtab_kernel(DevTree t, int L, int32_t* __restrict__ vtab, unsigned* flags)
{
	// the direction -> slot table in shared memory: the lanes look up
	// different entries, which constant memory would serialise
	__shared__ int16_t s_dir_slot[8 * 343];
	for (int i = threadIdx.x; i < 8 * 343; i += blockDim.x) s_dir_slot[i] = (&g_dir_slot[0][0])[i];
	__syncthreads();
	const int lane = threadIdx.x & 31;
	const size_t c = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const size_t m = t.lsize[L];
	if (c >= m) return;
	int32_t* row = vtab + c * M2L_SLOTS;
	for (int sl = lane; sl < M2L_SLOTS; sl += 32) row[sl] = -1;
	__syncwarp();
	const size_t off = t.loff[L], poff = t.loff[L - 1];
	int me[3];
	coords3(t.code[off + c], me);
	const int oct = ((me[0] & 1) << 2) | ((me[1] & 1) << 1) | (me[2] & 1);
	const int16_t* ds = s_dir_slot + oct * 343;
	const int32_t p = t.parent[off + c];
	const int npc = t.close_cnt[poff + p];
	const int32_t* pl = t.close_idx + (poff + p) * t.close_stride;
	for (int e = lane; e <= npc; e += 32) {
		const int32_t pn = e < npc ? pl[e] : p;
		// a child of pn sits at 2 coords(pn) + its octant bits (code = pn's code << 3 | octant)
		int q[3];
		coords3(t.code[poff + pn], q);
		const int bx = 2 * q[0] - me[0], by = 2 * q[1] - me[1], bz = 2 * q[2] - me[2];
		for (uint32_t k = t.beg[poff + pn]; k < t.end[poff + pn]; ++k) {
			if (k == c) continue;
			const int ko = (int)(t.code[off + k] & 7ull);
			const int dx = bx + ((ko >> 2) & 1), dy = by + ((ko >> 1) & 1), dz = bz + (ko & 1);
			if (max(max(abs(dx), abs(dy)), abs(dz)) <= 1) continue;
			const int slot = ds[(dx + 3) * 49 + (dy + 3) * 7 + (dz + 3)];
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
	// the direction -> slot table in shared memory: the threads look up
	// different entries, which constant memory would serialise
	__shared__ int16_t s_dir_slot2[4 * 49];
	for (int i = threadIdx.x; i < 4 * 49; i += blockDim.x) s_dir_slot2[i] = (&g_dir_slot2[0][0])[i];
	__syncthreads();
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	size_t m = t.lsize[L];
	if (c >= m) return;
	size_t off = t.loff[L], poff = t.loff[L - 1];
	int me[2];
	coords2g(t.code[off + c], me);
	const int cls = ((me[0] & 1) << 1) | (me[1] & 1);
	const int16_t* ds = s_dir_slot2 + cls * 49;
	int32_t* row = vtab + c * M2L_SLOTS2;
	int32_t p = t.parent[off + c];
	int npc = t.close_cnt[poff + p];
	const int32_t* pl = t.close_idx + (poff + p) * t.close_stride;
	for (int e = 0; e <= npc; ++e) {
		int32_t pn = e < npc ? pl[e] : p;
		// a child of pn sits at 2 coords(pn) + its quadrant bits (code = pn's code << 2 | quadrant)
		int q[2];
		coords2g(t.code[poff + pn], q);
		const int bx = 2 * q[0] - me[0], by = 2 * q[1] - me[1];
		for (uint32_t k = t.beg[poff + pn]; k < t.end[poff + pn]; ++k) {
			if (k == c) continue;
			const int ko = (int)(t.code[off + k] & 3ull);
			const int dx = bx + ((ko >> 1) & 1), dy = by + (ko & 1);
			if (max(abs(dx), abs(dy)) <= 1) continue;
			int slot = (abs(dx) <= 3 && abs(dy) <= 3) ? ds[(dx + 3) * 7 + (dy + 3)] : -1;
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

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int bytes)
{
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory"); }

// FP64 tensor-core MMA (mma.sync m8n8k4, the FP64 path of sm_100): D = A B + C
// with A 8x4 row-major (lane: A[lane/4][lane%4]), B 4x8 column-major
// (lane: B[lane%4][lane/4]) and C, D 8x8 (lane: C[lane/4][2 (lane%4) + 0, 1]).
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b)
{
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
	             : "+d"(d0), "+d"(d1)
	             : "d"(a), "d"(b));
}

constexpr int H2_LD = 136;             // row stride (doubles) of the staged W: conflict-free B fragments

// Dynamic shared memory of the Hankel kernel for order N (bytes).
inline size_t hankel_smem(int N)
{
	const int R4 = (N + 3) / 4 * 4, RS = N | 1;
	return sizeof(double2) * (64 * (size_t)RS + 2 * (size_t)N + 1) + sizeof(double) * (size_t)R4 * H2_LD +
	       sizeof(int32_t) * M2L_SLOTS2 * 65;
}

// Block of 128 threads per (quadrant class, tile of 64 targets) and slot
// range.  Per slot: W = pre (.) a (gathered sources, stored as columns
// 2c + re/im), S = H W on the FP64 tensor cores (warp w: columns
// [32w, 32w + 32), all rows in MTL tiles of 8), b += post (.) S on the
// accumulator fragments, which hold the re and im of one target side by side.
// The next non-empty slot's sources and tables are staged by cp.async
// (zero-filled where a target has no source) while the current one computes.
template <int MTL>
__global__ void __launch_bounds__(128, MTL < 4 ? 4 : 3) m2l2d_hankel_kernel(const double2* __restrict__ tab,
                                                           const double2* __restrict__ mult, double2* __restrict__ loc,
                                                           const int32_t* __restrict__ vtab,
                                                           const int32_t* __restrict__ order,
                                                           const uint32_t* __restrict__ cls_count, int N,
                                                           double2* __restrict__ part, size_t cells)
{
	const int S = gridDim.y, sidx = blockIdx.y;
	const int slot0 = sidx * M2L_SLOTS2 / S, slot1 = (sidx + 1) * M2L_SLOTS2 / S;
	if (S > 1) loc = part + (size_t)sidx * cells * N;
	const int R4 = (N + 3) / 4 * 4, W2 = 2 * N + 1;
	const int RS = N | 1;                  // odd row stride: conflict-free reads by source
	extern __shared__ __align__(16) unsigned char dsm[];
	double2* raw = reinterpret_cast<double2*>(dsm);                 // [64][RS] sources of a slot
	double2* sT = raw + 64 * RS;                                     // [2N+1] pre, post, log term
	double* Wc = reinterpret_cast<double*>(sT + W2);                 // [R4][H2_LD]
	int32_t* srcs = reinterpret_cast<int32_t*>(Wc + R4 * H2_LD);     // [27][65]
	__shared__ double sH[72];              // (k-1)!, read up to index 8 MTL + R4 - 2 <= 62
	__shared__ double2 spost[32];
	__shared__ double2 slg;
	__shared__ int32_t tgt[64];
	__shared__ int s_cls, s_n, s_cnt;
	__shared__ int s_list[M2L_SLOTS2];
	__shared__ uint32_t s_start, s_mask;
	const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
	if (tid == 0) {
		uint32_t b = blockIdx.x, start = 0;
		int cls = -1, nn = 0;
		for (int o = 0; o < 4; ++o) {
			const uint32_t cnt = cls_count[o], tiles = (cnt + 63) / 64;
			if (b < tiles) { cls = o; start += b * 64; nn = (int)min(64u, cnt - b * 64); break; }
			b -= tiles; start += cnt;
		}
		s_cls = cls; s_n = nn; s_start = start; s_mask = 0;
	}
	if (tid < 72) sH[tid] = tid == 0 || tid > 63 ? 0.0 : c_fact[tid - 1];
	__syncthreads();
	const int cls = s_cls;
	if (cls < 0) return;
	if (tid < 64) tgt[tid] = tid < s_n ? order[s_start + tid] : -1;
	for (int e = N * H2_LD + tid; e < R4 * H2_LD; e += 128) Wc[e] = 0.0;   // rows N..R4-1 stay 0
	__syncthreads();
	// every target's slot row (contiguous in vtab), and which slots are used
	for (int idx = tid; idx < 64 * M2L_SLOTS2; idx += 128) {
		const int c = idx / M2L_SLOTS2, sl = idx - c * M2L_SLOTS2;
		const int32_t v = tgt[c] >= 0 ? vtab[(size_t)tgt[c] * M2L_SLOTS2 + sl] : -1;
		srcs[sl * 65 + c] = v;
		if (v >= 0 && sl >= slot0 && sl < slot1) atomicOr(&s_mask, 1u << sl);
	}
	__syncthreads();
	if (tid == 0) {
		int n = 0;
		for (int sl = slot0; sl < slot1; ++sl)
			if (s_mask >> sl & 1u) s_list[n++] = sl;
		s_cnt = n;
	}
	__syncthreads();
	const int nl = s_cnt;
	auto issue = [&](int j) {
		const int sl = s_list[j];
		const int32_t* sr = srcs + sl * 65;
		if (lane < N)                          // warp w: sources w, w + 4, ...; lane: coefficient
			for (int c = w; c < 64; c += 4) {
				const int32_t s = sr[c];
				cp_async16(raw + c * RS + lane, s >= 0 ? mult + (size_t)s * N + lane : mult, s >= 0 ? 16 : 0);
			}
		if (tid < W2) cp_async16(sT + tid, tab + (size_t)c_slot_dir2[cls][sl] * W2 + tid, 16);
		cp_async_commit();
	};
	double ar[MTL][4][2];                  // b of rows 8 mt + g, target 16 w + 4 nt + t4 (re, im)
#pragma unroll
	for (int mt = 0; mt < MTL; ++mt)
#pragma unroll
		for (int nt = 0; nt < 4; ++nt) ar[mt][nt][0] = ar[mt][nt][1] = 0.0;
	if (nl > 0) issue(0);
	for (int j = 0; j < nl; ++j) {
		cp_async_wait<0>();
		__syncthreads();
		{
			const int c = tid & 63;            // source c, coefficients k = tid / 64 + 2 m
			for (int k = tid >> 6; k < N; k += 2) {
				const double2 a = raw[c * RS + k], p = sT[k];
				*reinterpret_cast<double2*>(Wc + k * H2_LD + 2 * c) =
				    make_double2(a.x * p.x - a.y * p.y, a.x * p.y + a.y * p.x);
			}
		}
		if (tid < N) spost[tid] = sT[N + tid];
		if (tid == N) slg = sT[2 * N];
		__syncthreads();
		if (j + 1 < nl) issue(j + 1);          // lands while the MMAs run
		double sacc[MTL][4][2];
#pragma unroll
		for (int mt = 0; mt < MTL; ++mt)
#pragma unroll
			for (int nt = 0; nt < 4; ++nt) sacc[mt][nt][0] = sacc[mt][nt][1] = 0.0;
		for (int k0 = 0; k0 < R4; k0 += 4) {
			double bf[4];
#pragma unroll
			for (int nt = 0; nt < 4; ++nt) bf[nt] = Wc[(k0 + t4) * H2_LD + 32 * w + 8 * nt + g];
#pragma unroll
			for (int mt = 0; mt < MTL; ++mt) {
				const double af = sH[8 * mt + g + k0 + t4];
#pragma unroll
				for (int nt = 0; nt < 4; ++nt) dmma_8x8x4(sacc[mt][nt][0], sacc[mt][nt][1], af, bf[nt]);
			}
		}
#pragma unroll
		for (int mt = 0; mt < MTL; ++mt) {
			const int i = 8 * mt + g;
			if (i < N) {
				const double2 p = spost[i];
#pragma unroll
				for (int nt = 0; nt < 4; ++nt) {
					const double sr_ = sacc[mt][nt][0], si_ = sacc[mt][nt][1];
					ar[mt][nt][0] += p.x * sr_ - p.y * si_;
					ar[mt][nt][1] += p.x * si_ + p.y * sr_;
				}
			}
		}
		if (g == 0) {                          // row 0: b_0 += a_0 lg, a_0 = -W[0]
			const double2 lg = slg;
#pragma unroll
			for (int nt = 0; nt < 4; ++nt) {
				const int c = 16 * w + 4 * nt + t4;
				const double a0r = -Wc[2 * c], a0i = -Wc[2 * c + 1];
				ar[0][nt][0] += a0r * lg.x - a0i * lg.y;
				ar[0][nt][1] += a0r * lg.y + a0i * lg.x;
			}
		}
	}
#pragma unroll
	for (int nt = 0; nt < 4; ++nt) {
		const int tg = tgt[16 * w + 4 * nt + t4];
		if (tg < 0) continue;
#pragma unroll
		for (int mt = 0; mt < MTL; ++mt) {
			const int i = 8 * mt + g;
			if (i < N) loc[(size_t)tg * N + i] = make_double2(ar[mt][nt][0], ar[mt][nt][1]);
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

// 3D FP64 M2L on the FP64 tensor cores: C[MT x 64] = sum over the octant
// class's non-empty slots of T_dir[MT x MT] B[MT x 64], B the gathered
// source multipoles.  256 threads: warp (wm, wn) = (w & 3, w >> 2) owns row
// tiles wm + 4 i (i < MTW) and target tiles 4 wn .. 4 wn + 3 (8 x 8 each),
// FP64 accumulators in registers across all slots.  The operator columns
// and source rows of the next 16-wide K chunk are staged by cp.async
// (double buffered, zero-filled past R and where a target has no source);
// both staged tiles are row-major with a row stride of 20 doubles, which
// keeps the fragment reads conflict-free.
constexpr int DG_LD = 20;

inline size_t dmma_gemm_smem(int MT) { return sizeof(double) * 2 * (size_t)(MT + 64) * DG_LD; }

template <int MTW>
__global__ void __launch_bounds__(256, 1) m2l_gemm_dmma_kernel(const double* __restrict__ ops,
                                                               const double* __restrict__ mult,
                                                               double* __restrict__ loc,
                                                               const int32_t* __restrict__ vtab,
                                                               const int32_t* __restrict__ order,
                                                               const uint32_t* __restrict__ oct_count, int R,
                                                               int MT, double* __restrict__ part, size_t cells)
{
	const int S = gridDim.y, sidx = blockIdx.y;
	const int slot0 = sidx * M2L_SLOTS / S, slot1 = (sidx + 1) * M2L_SLOTS / S;
	if (S > 1) loc = part + (size_t)sidx * cells * R;
	extern __shared__ __align__(16) double dsm_d[];
	double* As = dsm_d;                                  // [2][MT][DG_LD]
	double* Bs = dsm_d + 2 * MT * DG_LD;                 // [2][64][DG_LD]
	__shared__ int32_t tgt[64];
	__shared__ int16_t s_list[M2L_SLOTS];
	__shared__ uint32_t s_mask[6];
	__shared__ int s_oct, s_n, s_cnt;
	__shared__ uint32_t s_start;
	const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
	const int wm = w & 3, wn = w >> 2;
	if (tid == 0) {
		uint32_t b = blockIdx.x, start = 0;
		int oct = -1, nn = 0;
		for (int o = 0; o < 8; ++o) {
			const uint32_t cnt = oct_count[o], tiles = (cnt + 63) / 64;
			if (b < tiles) { oct = o; start += b * 64; nn = (int)min(64u, cnt - b * 64); break; }
			b -= tiles; start += cnt;
		}
		s_oct = oct; s_n = nn; s_start = start;
	}
	if (tid < 6) s_mask[tid] = 0;
	__syncthreads();
	const int oct = s_oct;
	if (oct < 0) return;
	if (tid < 64) tgt[tid] = tid < s_n ? order[s_start + tid] : -1;
	__syncthreads();
	for (int idx = tid; idx < 64 * M2L_SLOTS; idx += 256) {
		const int c = idx / M2L_SLOTS, sl = idx - c * M2L_SLOTS;
		if (sl < slot0 || sl >= slot1 || tgt[c] < 0) continue;
		if (vtab[(size_t)tgt[c] * M2L_SLOTS + sl] >= 0) atomicOr(&s_mask[sl >> 5], 1u << (sl & 31));
	}
	__syncthreads();
	if (tid == 0) {
		int n = 0;
		for (int sl = slot0; sl < slot1; ++sl)
			if (s_mask[sl >> 5] >> (sl & 31) & 1u) s_list[n++] = (int16_t)sl;
		s_cnt = n;
	}
	__syncthreads();
	const int KC = MT / 16;
	const int iters = s_cnt * KC;
	// B staging: thread (c, quarter) copies k = 16 kc + 4 quarter + {0..3} of target c's source
	const int bc = tid & 63, bq = tid >> 6;
	const int32_t my_tgt = tgt[bc];
	auto issue = [&](int it, int buf) {
		const int j = it / KC, kc = it - j * KC;
		const int sl = s_list[j];
		const double* A = ops + (size_t)c_slot_dir[oct][sl] * MT * MT + 16 * kc;
		double* ad = As + (size_t)buf * MT * DG_LD;
		for (int e = tid; e < MT * 8; e += 256) {
			const int r = e >> 3, q = e & 7;
			cp_async16(ad + r * DG_LD + 2 * q, A + (size_t)r * MT + 2 * q, 16);
		}
		const int32_t s = my_tgt >= 0 ? vtab[(size_t)my_tgt * M2L_SLOTS + sl] : -1;
		double* bd = Bs + (size_t)buf * 64 * DG_LD + bc * DG_LD + 4 * bq;
#pragma unroll
		for (int h = 0; h < 2; ++h) {
			const int k = 16 * kc + 4 * bq + 2 * h;
			const bool ok = s >= 0 && k < R;
			cp_async16(bd + 2 * h, ok ? mult + (size_t)s * R + k : mult, ok ? 16 : 0);
		}
		cp_async_commit();
	};
	double acc[MTW][4][2];
#pragma unroll
	for (int i = 0; i < MTW; ++i)
#pragma unroll
		for (int n = 0; n < 4; ++n) acc[i][n][0] = acc[i][n][1] = 0.0;
	const int MTT = MT / 8;                    // row tiles
	if (iters > 0) issue(0, 0);
	for (int it = 0; it < iters; ++it) {
		const int cur = it & 1;
		if (it + 1 < iters) { issue(it + 1, cur ^ 1); cp_async_wait<1>(); }
		else cp_async_wait<0>();
		__syncthreads();
		const double* a_ = As + (size_t)cur * MT * DG_LD;
		const double* b_ = Bs + (size_t)cur * 64 * DG_LD;
#pragma unroll
		for (int ks = 0; ks < 4; ++ks) {
			double bf[4];
#pragma unroll
			for (int n = 0; n < 4; ++n) bf[n] = b_[(8 * (4 * wn + n) + g) * DG_LD + 4 * ks + t4];
#pragma unroll
			for (int i = 0; i < MTW; ++i) {
				const int mt = wm + 4 * i;
				if (mt < MTT) {
					const double af = a_[(8 * mt + g) * DG_LD + 4 * ks + t4];
#pragma unroll
					for (int n = 0; n < 4; ++n) dmma_8x8x4(acc[i][n][0], acc[i][n][1], af, bf[n]);
				}
			}
		}
		__syncthreads();                       // the buffer is refilled two iterations on
	}
#pragma unroll
	for (int n = 0; n < 4; ++n)
#pragma unroll
		for (int h = 0; h < 2; ++h) {
			const int tg = tgt[8 * (4 * wn + n) + 2 * t4 + h];
			if (tg < 0) continue;
#pragma unroll
			for (int i = 0; i < MTW; ++i) {
				const int r = 8 * (wm + 4 * i) + g;
				if (r < R) loc[(size_t)tg * R + r] = acc[i][n][h];
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
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(g_dir_slot, S.dir_slot, sizeof(S.dir_slot)));
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
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(g_dir_slot2, ds, sizeof(ds)));
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
	const int MTL = (N + 7) / 8;           // row tiles of 8
	const size_t smem = hankel_smem(N);
	auto go = [&](auto kern) -> cudaError_t {
		cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		if (e != cudaSuccess) return e;
		kern<<<grid, 128, smem, s>>>(tab, mult, loc, plan.vtab, plan.order, plan.oct_count, N, part, plan.cells);
		return cudaGetLastError();
	};
	cudaError_t e;
	switch (MTL) {
	case 1: e = go(m2l2d_hankel_kernel<1>); break;
	case 2: e = go(m2l2d_hankel_kernel<2>); break;
	case 3: e = go(m2l2d_hankel_kernel<3>); break;
	default: e = go(m2l2d_hankel_kernel<4>); break;
	}
	if (e != cudaSuccess) return cuda_fail(ctx, e, "m2l2d_hankel_kernel");
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
	LFMM_CUDA(ctx, cudaMemsetAsync(plan.oct_count, 0, sizeof(uint32_t) * 16, s));
	if (m == 0) return OK;
	count_oct_kernel<<<div_up(m, 256), 256, 0, s>>>(t, L, plan.oct_count);
	scatter_oct_kernel<<<div_up(m, 256), 256, 0, s>>>(t, L, plan.oct_count, plan.order);
	vtab_kernel<<<div_up(m * 32, 256), 256, 0, s>>>(t, L, plan.vtab, ctx.dev_flags);   // warp per cell
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
	if constexpr (DIM == 3 && sizeof(real) == sizeof(double)) {
		const size_t smem = dmma_gemm_smem(MT);
		const int mtw = (MT / 8 + 3) / 4;
		auto go = [&](auto kern) -> cudaError_t {
			cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
			if (e != cudaSuccess) return e;
			kern<<<grid, 256, smem, s>>>(reinterpret_cast<const double*>(ops), reinterpret_cast<const double*>(mult),
			                             reinterpret_cast<double*>(loc), plan.vtab, plan.order, plan.oct_count, R, MT,
			                             reinterpret_cast<double*>(part), plan.cells);
			return cudaGetLastError();
		};
		cudaError_t e;
		switch (mtw) {
		case 1: e = go(m2l_gemm_dmma_kernel<1>); break;
		case 2: e = go(m2l_gemm_dmma_kernel<2>); break;
		case 3: e = go(m2l_gemm_dmma_kernel<3>); break;
		case 4: e = go(m2l_gemm_dmma_kernel<4>); break;
		case 5: e = go(m2l_gemm_dmma_kernel<5>); break;
		case 6: e = go(m2l_gemm_dmma_kernel<6>); break;
		case 7: e = go(m2l_gemm_dmma_kernel<7>); break;
		case 8: e = go(m2l_gemm_dmma_kernel<8>); break;
		case 9: e = go(m2l_gemm_dmma_kernel<9>); break;
		case 10: e = go(m2l_gemm_dmma_kernel<10>); break;
		case 11: e = go(m2l_gemm_dmma_kernel<11>); break;
		default: ctx.last_error = "m2l gemm: order too large"; return ERR_UNSUPPORTED;
		}
		if (e != cudaSuccess) return cuda_fail(ctx, e, "m2l_gemm_dmma_kernel");
	} else if constexpr (DIM == 2) {
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
	case 17: launch_gemm<real, 17, DIM>(grid, s, ops, mult, loc, plan, R, part); break;
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
