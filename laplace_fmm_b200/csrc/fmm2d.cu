// 2D Laplace FMM, FP64, following the reference's CPU solver
// (cpu/multipole.cpp): P2M 22-36, M2M 38-53, M2L 66-84, L2L 86-97, passes
// 99-231 (per level: L2L from the parent, then M2L from the far list),
// leaves 233-449 (P2P + L2P for potential and field).
// Warp per box with one expansion coefficient per lane (N <= 30), block per
// leaf for the near field.  The adaptive quadtree (fmm2d_solve_adaptive) adds
// the U / W / X lists of the adaptive octree's rules: P2P over U, M2P over W
// (a source cell's Laurent series evaluated at a leaf's targets), P2L over X
// (a leaf's sources placed straight into a cell's Taylor series).
#include "fmm2d.cuh"
#include "m2l_gemm.cuh"
#include "primitives.cuh"
#include <cmath>
#include <mutex>

namespace lfmm {

namespace {

constexpr int WPB2 = 4;
constexpr int BINOM_N = 2 * MAXN2;
// Pascal triangle in global memory (lanes read different entries, which
// constant memory would serialise): C(n,k) at n*60+k, and transposed,
// C(n,k) at k*60+n.
__device__ double c_binom[BINOM_N * BINOM_N];
__device__ double c_binomT[BINOM_N * BINOM_N];

// Natural logarithm of a normal, finite x > 0, table-driven after P. T. P.
// Tang, "Table-driven implementation of the logarithm function in IEEE
// floating-point arithmetic", ACM TOMS 16(4), 1990: x = 2^e m, m in [1, 2),
// c = 1 + i/256 the table point nearest m, t = m/c - 1 (|t| <= 2^-9) from the
// stored 1/c, log x = e ln2 + log c + log1p(t), log1p by its Taylor series to
// t^5 (truncation below 1e-17).  The table and the split ln2 = hi + lo (hi
// with 24 bits, so e hi is exact) are computed on the host in long double.
struct LogTable {
	double2 e[257];                    // (log c_i, 1 / c_i)
	double ln2_hi, ln2_lo;
};
__device__ LogTable c_logtab;

__device__ __forceinline__ double log_table(double x, const double2* __restrict__ tab, double ln2_hi, double ln2_lo)
{
	const int hi = __double2hiint(x);
	const int e = (hi >> 20) - 1023;
	const int mh = hi & 0xFFFFF;
	const int i = (mh + (1 << 11)) >> 12;
	const double m = __hiloint2double(mh | 0x3FF00000, __double2loint(x));
	const double2 c = tab[i];
	const double t = fma(m, c.y, -1.0);
	double q = fma(t, 0.2, -0.25);
	q = fma(t, q, 1.0 / 3.0);
	q = fma(t, q, -0.5);
	q = fma(t, q, 1.0);
	const double de = (double)e;
	return fma(de, ln2_hi, c.x + fma(de, ln2_lo, t * q));
}

struct Exp2 {
	int N;
	double2* outer;
	double2* inner;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{ return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 cdiv(double2 a, double2 b)
{
	double d = b.x * b.x + b.y * b.y;
	return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 cpow_u(double2 b, int e)
{
	double2 r = make_double2(1.0, 0.0);
	while (e) { if (e & 1) r = cmul(r, b); e >>= 1; b = cmul(b, b); }
	return r;
}
__device__ __forceinline__ void coords2(uint64_t code, int* c) { c[0] = (int)compact2(code >> 1); c[1] = (int)compact2(code); }

// a_k = -sum q (z - z0)^k / k, a_0 = sum q.  Lane k accumulates coefficient
// k over the leaf's particles, staged 32 at a time.  Uniform tree: the leaves
// of the last level; adaptive: every leaf, its sources [pbeg, send).
__global__ void __launch_bounds__(WPB2 * 32) p2m2d_kernel(DevTree t, Exp2 E)
{
	__shared__ double2 sz[WPB2][32];
	__shared__ double sq[WPB2][32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const size_t leaf = (size_t)blockIdx.x * WPB2 + w;
	size_t g;
	uint32_t pb, pe;
	if (t.adaptive) {
		if (leaf >= t.nleaves) return;
		g = t.leaves[leaf];
		pb = t.pbeg[g]; pe = t.send[g];
	} else {
		const int LL = t.depth - 1;
		if (leaf >= t.lsize[LL]) return;
		g = t.loff[LL] + leaf;
		pb = t.beg[g]; pe = t.end[g];
	}
	const int N = E.N;
	const double cx = t.cx[g], cy = t.cy[g];
	double2 acc = make_double2(0.0, 0.0);
	for (uint32_t base = pb; base < pe; base += 32) {
		const int cnt = (int)min(32u, pe - base);
		__syncwarp();
		if (lane < cnt) {
			const uint32_t i = base + lane;
			sq[w][lane] = t.q[i];
			sz[w][lane] = make_double2(t.x[i] - cx, t.y[i] - cy);
		}
		__syncwarp();
		if (lane < N)
			for (int j = 0; j < cnt; ++j) {
				const double2 p = cpow_u(sz[w][j], lane);
				acc.x = fma(sq[w][j], p.x, acc.x); acc.y = fma(sq[w][j], p.y, acc.y);
			}
	}
	if (lane < N) {
		if (lane > 0) acc = make_double2(-acc.x / lane, -acc.y / lane);
		E.outer[g * N + lane] = acc;
	}
}

// b_j += sum_{i=1..j} a_i z0^(j-i) C(j-1, i-1) - a_0 z0^j / j, b_0 += a_0 ; z0 = child - parent
__global__ void __launch_bounds__(WPB2 * 32) m2m2d_kernel(DevTree t, Exp2 E, int L)
{
	__shared__ double2 sa[WPB2][32];
	__shared__ double2 sp[WPB2][32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t c = (size_t)blockIdx.x * WPB2 + w;
	if (c >= t.lsize[L]) return;
	const int N = E.N;
	size_t g = t.loff[L] + c, cb = t.loff[L + 1];
	if (t.is_leaf && t.is_leaf[g]) return;          // adaptive: a leaf keeps its P2M
	double2 acc = make_double2(0.0, 0.0);
	for (uint32_t k = t.beg[g]; k < t.end[g]; ++k) {
		size_t gk = cb + k;
		double2 z0 = make_double2(t.cx[gk] - t.cx[g], t.cy[gk] - t.cy[g]);
		__syncwarp();
		if (lane < N) { sa[w][lane] = E.outer[gk * N + lane]; sp[w][lane] = cpow_u(z0, lane); }
		__syncwarp();
		int j = lane;
		if (j < N) {
			if (j == 0) { acc.x += sa[w][0].x; acc.y += sa[w][0].y; }
			else {
				double2 s = make_double2(0.0, 0.0);
				for (int i = 1; i <= j; ++i) {
					double2 v = cmul(sa[w][i], sp[w][j - i]);
					double bc = c_binomT[(i - 1) * BINOM_N + (j - 1)];
					s.x += v.x * bc; s.y += v.y * bc;
				}
				double2 a0z = cmul(sa[w][0], sp[w][j]);
				acc.x += s.x - a0z.x / j; acc.y += s.y - a0z.y / j;
			}
		}
	}
	if (lane < N) E.outer[g * N + lane] = acc;
}

// Per level L >= 2: b = L2L(parent inner) (overwrite), then += M2L over the
// far list.  L2L as b_k = sum_{n>=k} a_n C(n,k) (-z0)^(n-k), z0 = parent - child
// (the reference's in-place Horner shift, cpu/multipole.cpp:86-97).
// M2L: z0 = source - target; b_0 += a_0 conj(log(-z0)) + sum_j w_j,
// b_i += (-a_0 / i + sum_j w_j C(i+j-1, j-1)) / z0^i, w_j = (-1)^j a_j / z0^j.
__global__ void __launch_bounds__(WPB2 * 32) down2d_kernel(DevTree t, Exp2 E, int L)
{
	__shared__ double2 sa[WPB2][32];
	__shared__ double2 sw[WPB2][32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t c = (size_t)blockIdx.x * WPB2 + w;
	if (c >= t.lsize[L]) return;
	const int N = E.N;
	size_t off = t.loff[L], poff = t.loff[L - 1], g = off + c;
	int32_t p = t.parent[g];
	size_t gp = poff + p;
	double2 acc = make_double2(0.0, 0.0);
	if (L >= 3) {
		double2 mz = make_double2(-(t.cx[gp] - t.cx[g]), -(t.cy[gp] - t.cy[g]));
		if (lane < N) sa[w][lane] = E.inner[gp * N + lane];
		__syncwarp();
		if (lane < N) {
			double2 pw = make_double2(1.0, 0.0);
			for (int n = lane; n < N; ++n) {
				double2 v = cmul(sa[w][n], pw);
				double bc = c_binom[n * BINOM_N + lane];
				acc.x += v.x * bc; acc.y += v.y * bc;
				pw = cmul(pw, mz);
			}
		}
	}
	int me[2];
	coords2(t.code[g], me);
	int npc = t.close_cnt[gp];
	const int32_t* pl = t.close_idx + gp * t.close_stride;
	const double cx = t.cx[g], cy = t.cy[g];
	for (int e = 0; e <= npc; ++e) {
		int32_t pn = e < npc ? pl[e] : p;
		for (uint32_t k = t.beg[poff + pn]; k < t.end[poff + pn]; ++k) {
			if (k == c) continue;
			size_t gk = off + k;
			int o[2];
			coords2(t.code[gk], o);
			if (max(abs(o[0] - me[0]), abs(o[1] - me[1])) <= 1) continue;
			double2 z0 = make_double2(t.cx[gk] - cx, t.cy[gk] - cy);
			__syncwarp();
			double2 zl = make_double2(1.0, 0.0);
			if (lane < N) {
				double2 a = E.outer[gk * N + lane];
				sa[w][lane] = a;
				zl = cpow_u(z0, lane);
				sw[w][lane] = lane == 0 ? a : cdiv(make_double2(dsgn(lane) * a.x, dsgn(lane) * a.y), zl);
			}
			__syncwarp();
			if (lane < N) {
				double2 a0 = sa[w][0];
				if (lane == 0) {
					double2 mz = make_double2(-z0.x, -z0.y);
					double2 lg = make_double2(log(sqrt(mz.x * mz.x + mz.y * mz.y)), -atan2(mz.y, mz.x));
					double2 v = cmul(a0, lg);
					double sr = v.x, si = v.y;
					for (int j = 1; j < N; ++j) { sr += sw[w][j].x; si += sw[w][j].y; }
					acc.x += sr; acc.y += si;
				} else {
					int i = lane;
					double sr = 0.0, si = 0.0;
					for (int j = 1; j < N; ++j) {
						double bc = c_binom[(i + j - 1) * BINOM_N + (j - 1)];
						sr += sw[w][j].x * bc; si += sw[w][j].y * bc;
					}
					double2 num = make_double2(-a0.x / i + sr, -a0.y / i + si);
					double2 v = cdiv(num, zl);
					acc.x += v.x; acc.y += v.y;
				}
			}
		}
	}
	if (lane < N) E.inner[g * N + lane] = acc;
}

// L2L for L >= 3 added onto the M2L result of the level's GEMM:
// b_k += sum_{n>=k} a_n C(n,k) (-z0)^(n-k), z0 = parent - child.
__global__ void __launch_bounds__(WPB2 * 32) l2l2d_add_kernel(DevTree t, Exp2 E, int L)
{
	__shared__ double2 sa[WPB2][32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t c = (size_t)blockIdx.x * WPB2 + w;
	if (c >= t.lsize[L]) return;
	const int N = E.N;
	const size_t g = t.loff[L] + c, gp = t.loff[L - 1] + t.parent[g];
	const double2 mz = make_double2(-(t.cx[gp] - t.cx[g]), -(t.cy[gp] - t.cy[g]));
	if (lane < N) sa[w][lane] = E.inner[gp * N + lane];
	__syncwarp();
	if (lane >= N) return;
	double2 acc = E.inner[g * N + lane];
	double2 pw = make_double2(1.0, 0.0);
	for (int n = lane; n < N; ++n) {
		const double2 v = cmul(sa[w][n], pw);
		const double bc = c_binom[n * BINOM_N + lane];
		acc.x += v.x * bc; acc.y += v.y * bc;
		pw = cmul(pw, mz);
	}
	E.inner[g * N + lane] = acc;
}

// Leaves: P2P over the close list (the leaf itself first) and L2P
// (reference cpu/multipole.cpp:233-449).  One warp per work unit, a leaf's
// targets in chunks of 32 (so a crowded leaf of a clustered set spreads over
// many warps); a leaf of nt <= 16 targets is one unit whose warp runs TP = nt
// rounded up to a power of two targets at once and splits the sources into
// 32 / TP phases, summed by shuffles at the end.
constexpr int LW2 = 4;

__device__ __forceinline__ void leaf_targets(const DevTree& t, size_t g, uint32_t& tb, uint32_t& te)
{
	const bool tmode = t.targets_num > 0;
	tb = tmode ? t.tbeg[g] : t.beg[g];
	te = tmode ? t.tend[g] : t.end[g];
}

__global__ void leaf_units_kernel(DevTree t, uint32_t* __restrict__ units)
{
	const int LL = t.depth - 1;
	const size_t leaf = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (leaf >= t.lsize[LL]) return;
	uint32_t tb, te;
	leaf_targets(t, t.loff[LL] + leaf, tb, te);
	const uint32_t nt = te > tb ? te - tb : 0;
	units[leaf] = nt == 0 ? 0 : (nt <= 16 ? 1 : (nt + 31) / 32);
}

__global__ void __launch_bounds__(LW2 * 32) leaves2d_kernel(DevTree t, Exp2 E, const uint32_t* __restrict__ ubeg,
                                                            const uint32_t* __restrict__ total,
                                                            double* __restrict__ pot_out, double* __restrict__ fld_out)
{
	__shared__ double sx[LW2][32], sy[LW2][32], sq[LW2][32];
	__shared__ double2 sL[LW2][32];
	__shared__ double2 slog[257];
	for (int k = threadIdx.x; k < 257; k += LW2 * 32) slog[k] = c_logtab.e[k];
	const double ln2_hi = c_logtab.ln2_hi, ln2_lo = c_logtab.ln2_lo;
	__syncthreads();
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int LL = t.depth - 1;
	const uint32_t u = blockIdx.x * LW2 + w;
	if (u >= *total) return;
	// the leaf of unit u: the last leaf whose first unit is <= u
	uint32_t lo = 0, hi = (uint32_t)t.lsize[LL] - 1;
	while (lo < hi) {
		const uint32_t mid = (lo + hi + 1) >> 1;
		if (ubeg[mid] <= u) lo = mid; else hi = mid - 1;
	}
	const size_t off = t.loff[LL], g = off + lo;
	uint32_t tb, te;
	leaf_targets(t, g, tb, te);
	const int N = E.N;
	if (lane < N) sL[w][lane] = E.inner[g * N + lane];
	__syncwarp();
	const int nt = (int)(te - tb);
	int lt = 5;                                        // log2 of the targets per pass
	if (nt <= 16) { lt = 0; while ((1 << lt) < nt) ++lt; }
	const int TP = 1 << lt, G = 32 >> lt, ti = lane & (TP - 1), ph = lane >> lt;
	const int ncl = t.close_cnt[g];
	const int32_t* cl = t.close_idx + g * t.close_stride;
	const double cx = t.cx[g], cy = t.cy[g];
	{
		const uint32_t t0 = tb + 32u * (u - ubeg[lo]);
		const uint32_t i = t0 + ti;
		const bool valid = i < te;
		double xi = 0.0, yi = 0.0;
		if (valid) { xi = t.x[i]; yi = t.y[i]; }
		double pot = 0.0, fr = 0.0, fi = 0.0;
		// the close cells' particles as one stream (the leaf first): lane e
		// holds cell e's first particle and its inclusive end in the stream
		uint32_t cbeg = 0, cinc = 0;
		if (lane <= ncl) {
			const size_t sc = lane == 0 ? g : off + cl[lane - 1];
			cbeg = t.beg[sc];
			cinc = t.end[sc] - cbeg;
		}
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t v = __shfl_up_sync(0xffffffffu, cinc, o);
			if (lane >= o) cinc += v;
		}
		const uint32_t total = __shfl_sync(0xffffffffu, cinc, ncl);
		for (uint32_t s0 = 0; s0 < total; s0 += 32) {
			const int cnt = (int)min(32u, total - s0);
			const uint32_t pos = s0 + lane;
			uint32_t j = 0;
			for (int e = 0; e <= ncl; ++e) {        // the cell holding stream position pos
				const uint32_t inc = __shfl_sync(0xffffffffu, cinc, e);
				const uint32_t bg = __shfl_sync(0xffffffffu, cbeg, e);
				const uint32_t ex = e ? __shfl_sync(0xffffffffu, cinc, e - 1) : 0u;
				if (pos >= ex && pos < inc) j = bg + (pos - ex);
			}
			__syncwarp();
			if (lane < cnt) { sx[w][lane] = t.x[j]; sy[w][lane] = t.y[j]; sq[w][lane] = t.q[j]; }
			__syncwarp();
			if (valid) {
				for (int k = ph; k < cnt; k += G) {
					const double dx = xi - sx[w][k], dy = yi - sy[w][k];
					const double r2 = fmax(dx * dx + dy * dy, FORCE_EPS2);
					pot = fma(sq[w][k], log_table(r2, slog, ln2_hi, ln2_lo), pot);     // halved below
					const double qr = sq[w][k] / r2;
					fr = fma(dx, qr, fr); fi = fma(-dy, qr, fi);
				}
			}
		}
		for (int o = TP; o < 32; o <<= 1) {
			pot += __shfl_xor_sync(0xffffffffu, pot, o);
			fr += __shfl_xor_sync(0xffffffffu, fr, o);
			fi += __shfl_xor_sync(0xffffffffu, fi, o);
		}
		pot *= 0.5;                                    // sum q log r2 -> sum q log r
		if (valid && ph == 0) {
			double2 dz = make_double2(xi - cx, yi - cy), pw = make_double2(1.0, 0.0);
			for (int k = 0; k < N; ++k) {
				const double2 Lk = sL[w][k];
				pot += Lk.x * pw.x - Lk.y * pw.y;
				if (k + 1 < N) {
					const double2 v = cmul(sL[w][k + 1], pw);
					fr += (k + 1) * v.x; fi += (k + 1) * v.y;
				}
				pw = cmul(pw, dz);
			}
			const uint32_t o = t.orig[i];
			pot_out[o] = pot;
			fld_out[2 * (size_t)o] = fr; fld_out[2 * (size_t)o + 1] = fi;
		}
	}
}

// P2L over the X list: cell B's Taylor series gains the log of every source
// of a leaf C in X(B) (a monopole, so the series is exact in its terms):
// b_0 += q conj(log(-d)), b_i += -q / (i d^i), d = z_j - c_B (the M2L rule of
// down2d_kernel with a_0 = q and no other terms).  Warp per cell; sources
// taken 16 at a time: lane j < 16 stages source j's log term and the powers
// d^-1 .. d^-(N-1) (N - 1 products, once per source), then lane i sums
// coefficient i over the 16 sources.
constexpr int P2L_CHUNK = 16;

__global__ void __launch_bounds__(WPB2 * 32) p2l2d_kernel(DevTree t, Exp2 E)
{
	__shared__ double2 spw[WPB2][P2L_CHUNK][MAXN2];   // [source][i]: q d^-i (i >= 1); [0]: q conj(log(-d))
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const size_t g = (size_t)blockIdx.x * WPB2 + w;
	if (g >= t.ncells) return;
	const uint32_t xb = t.x_off[g], xe = t.x_off[g + 1];
	if (xb == xe) return;
	const int N = E.N;
	const double cx = t.cx[g], cy = t.cy[g];
	double2 acc = make_double2(0.0, 0.0);
	const double inv_i = lane > 0 ? -1.0 / (double)lane : 0.0;
	for (uint32_t e = xb; e < xe; ++e) {
		const int32_t C = t.x_idx[e];
		const uint32_t pb = t.pbeg[C], pe = t.send[C];
		for (uint32_t base = pb; base < pe; base += P2L_CHUNK) {
			const int cnt = (int)min((uint32_t)P2L_CHUNK, pe - base);
			__syncwarp();
			if (lane < cnt) {
				const uint32_t i = base + lane;
				const double qj = t.q[i];
				const double dx = t.x[i] - cx, dy = t.y[i] - cy;
				const double r2 = dx * dx + dy * dy;
				spw[w][lane][0] = make_double2(qj * 0.5 * log(r2), -qj * atan2(-dy, -dx));
				const double2 inv = make_double2(dx / r2, -dy / r2);
				double2 p = make_double2(qj * inv.x, qj * inv.y);
				for (int k = 1; k < N; ++k) {
					spw[w][lane][k] = p;
					p = cmul(p, inv);
				}
			}
			__syncwarp();
			if (lane < N) {
				if (lane == 0)
					for (int j = 0; j < cnt; ++j) { acc.x += spw[w][j][0].x; acc.y += spw[w][j][0].y; }
				else
					for (int j = 0; j < cnt; ++j) {
						const double2 v = spw[w][j][lane];
						acc.x = fma(inv_i, v.x, acc.x); acc.y = fma(inv_i, v.y, acc.y);
					}
			}
		}
	}
	if (lane < N) {
		double2 b = E.inner[g * N + lane];
		b.x += acc.x; b.y += acc.y;
		E.inner[g * N + lane] = b;
	}
}

__global__ void leaf_units_adaptive_kernel(DevTree t, uint32_t* __restrict__ units)
{
	const size_t li = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (li >= t.nleaves) return;
	const size_t g = t.leaves[li];
	const uint32_t nt = t.tend[g] > t.tbeg[g] ? t.tend[g] - t.tbeg[g] : 0;
	units[li] = nt == 0 ? 0 : (nt <= 16 ? 1 : (nt + 31) / 32);
}

// Leaves of the adaptive quadtree: P2P over the leaf itself and its U list
// (any length: the cells are taken 32 at a time, their sources streamed as
// one list), M2P over the W list (phases of the warp split the W cells),
// then L2P.  Work units as leaves2d_kernel's: a leaf's targets in chunks of
// 32, a leaf of <= 16 targets one unit of TP = nt rounded up to a power of
// two targets and 32 / TP source phases.
__global__ void __launch_bounds__(LW2 * 32) leaves2d_adaptive_kernel(DevTree t, Exp2 E,
                                                                     const uint32_t* __restrict__ ubeg,
                                                                     const uint32_t* __restrict__ total,
                                                                     double* __restrict__ pot_out,
                                                                     double* __restrict__ fld_out)
{
	__shared__ double sx[LW2][32], sy[LW2][32], sq[LW2][32];
	__shared__ double2 sL[LW2][32];
	__shared__ double2 slog[257];
	for (int k = threadIdx.x; k < 257; k += LW2 * 32) slog[k] = c_logtab.e[k];
	const double ln2_hi = c_logtab.ln2_hi, ln2_lo = c_logtab.ln2_lo;
	__syncthreads();
	const unsigned FULL = 0xffffffffu;
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const uint32_t u = blockIdx.x * LW2 + w;
	if (u >= *total) return;
	uint32_t lo = 0, hi = (uint32_t)t.nleaves - 1;     // the leaf whose units hold u
	while (lo < hi) {
		const uint32_t mid = (lo + hi + 1) >> 1;
		if (ubeg[mid] <= u) lo = mid; else hi = mid - 1;
	}
	const size_t li = lo, g = t.leaves[li];
	const uint32_t tb = t.tbeg[g], te = t.tend[g];
	const int N = E.N;
	if (lane < N) sL[w][lane] = E.inner[g * N + lane];
	__syncwarp();
	const int nt = (int)(te - tb);
	int lt = 5;
	if (nt <= 16) { lt = 0; while ((1 << lt) < nt) ++lt; }
	const int TP = 1 << lt, G = 32 >> lt, ti = lane & (TP - 1), ph = lane >> lt;
	const uint32_t i = tb + 32u * (u - ubeg[li]) + ti;
	const bool valid = i < te;
	double xi = 0.0, yi = 0.0;
	if (valid) { xi = t.x[i]; yi = t.y[i]; }
	double pot = 0.0, fpot = 0.0, fr = 0.0, fi = 0.0;
	// near field: the leaf, then U
	const uint32_t ub = t.u_off[li];
	const uint32_t ncell = t.u_off[li + 1] - ub + 1;
	for (uint32_t c0 = 0; c0 < ncell; c0 += 32) {
		const int gc = (int)min(32u, ncell - c0);
		uint32_t cbeg = 0, cinc = 0;
		if (lane < gc) {
			const uint32_t e = c0 + lane;
			const size_t sc = e == 0 ? g : (size_t)t.u_idx[ub + e - 1];
			cbeg = t.pbeg[sc];
			cinc = t.send[sc] - cbeg;
		}
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t v = __shfl_up_sync(FULL, cinc, o);
			if (lane >= o) cinc += v;
		}
		const uint32_t tot = __shfl_sync(FULL, cinc, gc - 1);
		for (uint32_t s0 = 0; s0 < tot; s0 += 32) {
			const int cnt = (int)min(32u, tot - s0);
			const uint32_t pos = s0 + lane;
			// the group's cell holding stream position pos: the first e with pos < inc[e]
			int clo = 0, chi = gc - 1;
#pragma unroll
			for (int it = 0; it < 5; ++it) {
				const int mid = (clo + chi) >> 1;
				const uint32_t v = __shfl_sync(FULL, cinc, mid);
				if (clo < chi) { if (pos < v) chi = mid; else clo = mid + 1; }
			}
			const uint32_t ex = __shfl_sync(FULL, cinc, clo > 0 ? clo - 1 : 0);
			const uint32_t bg = __shfl_sync(FULL, cbeg, clo);
			const uint32_t j = bg + (pos - (clo > 0 ? ex : 0u));
			__syncwarp();
			if (lane < cnt) { sx[w][lane] = t.x[j]; sy[w][lane] = t.y[j]; sq[w][lane] = t.q[j]; }
			__syncwarp();
			if (valid) {
				for (int k = ph; k < cnt; k += G) {
					const double dx = xi - sx[w][k], dy = yi - sy[w][k];
					const double r2 = fmax(dx * dx + dy * dy, FORCE_EPS2);
					pot = fma(sq[w][k], log_table(r2, slog, ln2_hi, ln2_lo), pot);     // halved below
					const double qr = sq[w][k] / r2;
					fr = fma(dx, qr, fr); fi = fma(-dy, qr, fi);
				}
			}
		}
	}
	// M2P over W: phi = a_0 log w + sum_k a_k w^-k, phi' = a_0 / w - sum_k k a_k w^-(k+1), w = z - c_D
	if (valid) {
		const uint32_t wb = t.w_off[li], we = t.w_off[li + 1];
		for (uint32_t e = wb + ph; e < we; e += G) {
			const size_t D = (size_t)t.w_idx[e];
			const double2* a = E.outer + D * N;
			const double wx = xi - t.cx[D], wy = yi - t.cy[D];
			const double r2 = wx * wx + wy * wy;
			const double2 iw = make_double2(wx / r2, -wy / r2);
			const double2 a0 = a[0];
			double2 phi = make_double2(0.0, 0.0), dphi = cmul(a0, iw), p = iw;
			for (int k = 1; k < N; ++k) {
				const double2 tk = cmul(a[k], p);
				phi.x += tk.x; phi.y += tk.y;
				const double2 tk1 = cmul(tk, iw);
				dphi.x = fma(-(double)k, tk1.x, dphi.x); dphi.y = fma(-(double)k, tk1.y, dphi.y);
				p = cmul(p, iw);
			}
			double re_log = 0.5 * a0.x * log_table(r2, slog, ln2_hi, ln2_lo);
			if (a0.y != 0.0) re_log -= a0.y * atan2(wy, wx);
			fpot += re_log + phi.x;
			fr += dphi.x; fi += dphi.y;
		}
	}
	for (int o = TP; o < 32; o <<= 1) {
		pot += __shfl_xor_sync(FULL, pot, o);
		fpot += __shfl_xor_sync(FULL, fpot, o);
		fr += __shfl_xor_sync(FULL, fr, o);
		fi += __shfl_xor_sync(FULL, fi, o);
	}
	pot = 0.5 * pot + fpot;                            // sum q log r2 -> sum q log r
	if (valid && ph == 0) {
		const double cx = t.cx[g], cy = t.cy[g];
		double2 dz = make_double2(xi - cx, yi - cy), pw = make_double2(1.0, 0.0);
		for (int k = 0; k < N; ++k) {
			const double2 Lk = sL[w][k];
			pot += Lk.x * pw.x - Lk.y * pw.y;
			if (k + 1 < N) {
				const double2 v = cmul(sL[w][k + 1], pw);
				fr += (k + 1) * v.x; fi += (k + 1) * v.y;
			}
			pw = cmul(pw, dz);
		}
		const uint32_t o = t.orig[i];
		pot_out[o] = pot;
		fld_out[2 * (size_t)o] = fr; fld_out[2 * (size_t)o + 1] = fi;
	}
}

std::mutex g_binom_mu;
bool g_binom_ready[64] = {};

// Pascal triangle and logarithm table, once per device.
int upload_2d_constants(Context& ctx)
{
	if (ctx.device < 0 || ctx.device >= 64) { ctx.last_error = "device index above 63"; return ERR_ARG; }
	std::unique_lock<std::mutex> lock(g_binom_mu);
	if (g_binom_ready[ctx.device]) return OK;
	static double b[BINOM_N * BINOM_N], bt[BINOM_N * BINOM_N];
	for (int i = 0; i < BINOM_N * BINOM_N; ++i) b[i] = 0.0;
	b[0] = 1.0;
	for (int i = 1; i < BINOM_N; ++i) {
		b[i * BINOM_N] = 1.0; b[i * BINOM_N + i] = 1.0;
		for (int j = 1; j < i; ++j) b[i * BINOM_N + j] = b[(i - 1) * BINOM_N + j] + b[(i - 1) * BINOM_N + j - 1];
	}
	for (int n = 0; n < BINOM_N; ++n)
		for (int k = 0; k < BINOM_N; ++k) bt[k * BINOM_N + n] = b[n * BINOM_N + k];
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_binom, b, sizeof(b)));
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_binomT, bt, sizeof(bt)));
	LogTable lt;
	for (int i = 0; i <= 256; ++i) {
		const long double c = 1.0L + (long double)i / 256.0L;
		lt.e[i] = make_double2((double)logl(c), (double)(1.0L / c));
	}
	const long double ln2 = logl(2.0L);
	lt.ln2_hi = (double)(float)ln2;
	lt.ln2_lo = (double)(ln2 - (long double)lt.ln2_hi);
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_logtab, &lt, sizeof(lt)));
	g_binom_ready[ctx.device] = true;
	return OK;
}

// M2L of levels 2 .. depth-1 grouped by (quadrant class, offset): the Hankel
// factorisation (default) or dense operators (LFMM_M2L=simt); each level's
// kernel writes (not adds) the level's local expansions.
int m2l2d_levels(Context& ctx, const DevTree& t, Exp2& E, int N, bool timing)
{
	cudaStream_t s = ctx.stream;
	int st;
	const size_t mark = ctx.arena.mark();
	for (int L = 2; L < t.depth; ++L) {
		if (t.lsize[L] == 0) continue;
		M2LPlan plan;
		if ((st = m2l_plan_build2d(ctx, t, L, plan))) return st;
		const double h = t.geo_host[3] / (double)(1ull << L);
		const double* ops = nullptr;
		const double2* tab = nullptr;
		if (ctx.m2l_engine == 0) ops = m2l_ops2d(ctx, N, h);
		else tab = m2l_tab2d(ctx, N, h);
		if (!ops && !tab) return ERR_OOM;
		const bool timed = timing && ctx.kev_used + 2 <= 32;
		if (timed) LFMM_CUDA(ctx, cudaEventRecord(ctx.kev[ctx.kev_used], s));
		if (ops) st = m2l_gemm2d(ctx, plan, ops, reinterpret_cast<double*>(E.outer + t.loff[L] * N),
		                         reinterpret_cast<double*>(E.inner + t.loff[L] * N), N);
		else st = m2l_hankel2d(ctx, plan, tab, E.outer + t.loff[L] * N, E.inner + t.loff[L] * N, N);
		if (st) return st;
		if (timed) { LFMM_CUDA(ctx, cudaEventRecord(ctx.kev[ctx.kev_used + 1], s)); ctx.kev_used += 2; }
		ctx.arena.rewind(mark);
	}
	return OK;
}

void fill_m2l_kernel_times(Context& ctx, SolveStats* stats)
{
	stats->ms_m2l_kernel = 0.f;
	for (int k = 0; k + 1 < ctx.kev_used; k += 2) {
		float ms = 0.f;
		cudaEventElapsedTime(&ms, ctx.kev[k], ctx.kev[k + 1]);
		stats->ms_m2l_kernel += ms;
	}
	stats->n_m2l_kernel = ctx.kev_used / 2;
}

} // namespace

int fmm2d_solve_device(Context& ctx, const ParticleInput& in, int N, int depth, double* pot, double* field,
                       SolveStats* stats)
{
	if (N < 1 || N > MAXN2) { ctx.last_error = "order out of range (1 <= N <= 30)"; return ERR_ARG; }
	int st = upload_2d_constants(ctx);
	if (st) return st;
	cudaStream_t s = ctx.stream;
	const bool timing = ctx.timing != 0;
	ctx.kev_used = 0;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[0], s));
	DevTree t;
	st = tree_build(ctx, in, depth, t);
	if (st) return st;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[1], s));
	Exp2 E;
	E.N = N;
	E.outer = static_cast<double2*>(ctx.arena.take(sizeof(double2) * t.ncells * N));
	E.inner = static_cast<double2*>(ctx.arena.take(sizeof(double2) * t.ncells * N));
	if (!E.outer || !E.inner) { ctx.last_error = "fmm2d: device allocation failed"; return ERR_OOM; }
	const int LL = depth - 1;
	const size_t n_out = in.nt ? in.nt : in.ns;
	LFMM_CUDA(ctx, cudaMemsetAsync(pot, 0, sizeof(double) * n_out, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(field, 0, sizeof(double) * 2 * n_out, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(E.inner, 0, sizeof(double2) * t.ncells * N, s));
	p2m2d_kernel<<<div_up(t.lsize[LL], WPB2), WPB2 * 32, 0, s>>>(t, E);
	for (int L = depth - 2; L >= 0; --L) m2m2d_kernel<<<div_up(t.lsize[L], WPB2), WPB2 * 32, 0, s>>>(t, E, L);
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[2], s));
	if (ctx.m2l_engine == 1) {
		// one warp per target cell over its far list
		for (int L = 2; L < depth; ++L) down2d_kernel<<<div_up(t.lsize[L], WPB2), WPB2 * 32, 0, s>>>(t, E, L);
	} else {
		// M2L grouped by (quadrant class, offset), all levels, then the L2L
		// passes top-down
		if ((st = m2l2d_levels(ctx, t, E, N, timing))) return st;
		for (int L = 3; L < depth; ++L)
			if (t.lsize[L]) l2l2d_add_kernel<<<div_up(t.lsize[L], WPB2), WPB2 * 32, 0, s>>>(t, E, L);
	}
	if (timing) { LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[3], s)); LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[4], s)); }
	if (t.lsize[LL]) {
		const size_t nl = t.lsize[LL];
		uint32_t* units = static_cast<uint32_t*>(ctx.arena.take(sizeof(uint32_t) * (2 * nl + 1)));
		uint32_t* scr = static_cast<uint32_t*>(ctx.arena.take(sizeof(uint32_t) * scan_scratch_words(nl)));
		if (!units || !scr) { ctx.last_error = "fmm2d: device allocation failed"; return ERR_OOM; }
		leaf_units_kernel<<<div_up(nl, 256), 256, 0, s>>>(t, units);
		scan_exclusive_u32(units, units + nl, nl, units + 2 * nl, scr, s);
		// at most one unit per leaf plus one per 32 targets
		const size_t max_units = nl + (n_out + 31) / 32;
		leaves2d_kernel<<<div_up(max_units, LW2), LW2 * 32, 0, s>>>(t, E, units + nl, units + 2 * nl, pot, field);
	}
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[5], s));
	LFMM_CUDA(ctx, cudaGetLastError());
	if (stats) {
		unsigned long long h[3];
		unsigned long long* counters = static_cast<unsigned long long*>(ctx.arena.take(32));
		if (!counters) { ctx.last_error = "fmm2d: device allocation failed"; return ERR_OOM; }
		if ((st = tree_count_pairs(ctx, t, counters, h))) return st;
		stats->n_far_pairs = h[0]; stats->n_close_pairs = h[1]; stats->n_p2p_pairs = h[2];
		stats->N = N; stats->depth = depth;
		stats->n_particles = t.n; stats->n_cells = t.ncells; stats->n_leaves = t.lsize[LL];
		stats->targets_num = t.targets_num;
		if (timing) {
			cudaEventElapsedTime(&stats->ms_tree, ctx.ev[0], ctx.ev[1]);
			cudaEventElapsedTime(&stats->ms_upward, ctx.ev[1], ctx.ev[2]);
			cudaEventElapsedTime(&stats->ms_m2l, ctx.ev[2], ctx.ev[3]);
			cudaEventElapsedTime(&stats->ms_leaves, ctx.ev[4], ctx.ev[5]);
			cudaEventElapsedTime(&stats->ms_total, ctx.ev[0], ctx.ev[5]);
			fill_m2l_kernel_times(ctx, stats);
		}
	}
	return OK;
}

int fmm2d_solve_adaptive(Context& ctx, const ParticleInput& in, int N, int depth, int max_leaf, double* pot,
                         double* field, SolveStats* stats)
{
	if (N < 1 || N > MAXN2) { ctx.last_error = "order out of range (1 <= N <= 30)"; return ERR_ARG; }
	int st = upload_2d_constants(ctx);
	if (st) return st;
	cudaStream_t s = ctx.stream;
	const bool timing = ctx.timing != 0;
	ctx.kev_used = 0;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[0], s));
	DevTree t;
	if ((st = tree_build_adaptive(ctx, in, depth, max_leaf, t))) return st;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[1], s));
	Exp2 E;
	E.N = N;
	E.outer = static_cast<double2*>(ctx.arena.take(sizeof(double2) * t.ncells * N));
	E.inner = static_cast<double2*>(ctx.arena.take(sizeof(double2) * t.ncells * N));
	if (!E.outer || !E.inner) { ctx.last_error = "fmm2d: device allocation failed"; return ERR_OOM; }
	const size_t n_out = in.nt ? in.nt : in.ns;
	LFMM_CUDA(ctx, cudaMemsetAsync(pot, 0, sizeof(double) * n_out, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(field, 0, sizeof(double) * 2 * n_out, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(E.inner, 0, sizeof(double2) * t.ncells * N, s));
	const size_t nl = t.nleaves;
	if (nl) p2m2d_kernel<<<div_up(nl, WPB2), WPB2 * 32, 0, s>>>(t, E);
	for (int L = t.depth - 2; L >= 0; --L)
		if (t.lsize[L]) m2m2d_kernel<<<div_up(t.lsize[L], WPB2), WPB2 * 32, 0, s>>>(t, E, L);
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[2], s));
	if ((st = m2l2d_levels(ctx, t, E, N, timing))) return st;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[3], s));
	if (t.n_x) p2l2d_kernel<<<div_up(t.ncells, WPB2), WPB2 * 32, 0, s>>>(t, E);
	for (int L = 3; L < t.depth; ++L)
		if (t.lsize[L]) l2l2d_add_kernel<<<div_up(t.lsize[L], WPB2), WPB2 * 32, 0, s>>>(t, E, L);
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[4], s));
	if (nl) {
		uint32_t* units = static_cast<uint32_t*>(ctx.arena.take(sizeof(uint32_t) * (2 * nl + 1)));
		uint32_t* scr = static_cast<uint32_t*>(ctx.arena.take(sizeof(uint32_t) * scan_scratch_words(nl)));
		if (!units || !scr) { ctx.last_error = "fmm2d: device allocation failed"; return ERR_OOM; }
		leaf_units_adaptive_kernel<<<div_up(nl, 256), 256, 0, s>>>(t, units);
		scan_exclusive_u32(units, units + nl, nl, units + 2 * nl, scr, s);
		const size_t max_units = nl + (n_out + 31) / 32;
		leaves2d_adaptive_kernel<<<div_up(max_units, LW2), LW2 * 32, 0, s>>>(t, E, units + nl, units + 2 * nl, pot,
		                                                                        field);
	}
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[5], s));
	LFMM_CUDA(ctx, cudaGetLastError());
	if (stats) {
		unsigned long long h[4];
		if ((st = tree_adaptive_counts(ctx, t, h))) return st;
		stats->N = N; stats->depth = t.depth;
		stats->n_particles = t.n; stats->n_cells = t.ncells; stats->n_leaves = t.nleaves;
		stats->targets_num = t.targets_num;
		stats->n_far_pairs = h[0]; stats->n_close_pairs = h[1]; stats->n_p2p_pairs = h[2];
		stats->n_m2p = h[3]; stats->n_w = t.n_w; stats->n_x = t.n_x;
		if (timing) {
			cudaEventElapsedTime(&stats->ms_tree, ctx.ev[0], ctx.ev[1]);
			cudaEventElapsedTime(&stats->ms_upward, ctx.ev[1], ctx.ev[2]);
			cudaEventElapsedTime(&stats->ms_m2l, ctx.ev[2], ctx.ev[3]);
			cudaEventElapsedTime(&stats->ms_l2l, ctx.ev[3], ctx.ev[4]);
			cudaEventElapsedTime(&stats->ms_leaves, ctx.ev[4], ctx.ev[5]);
			cudaEventElapsedTime(&stats->ms_total, ctx.ev[0], ctx.ev[5]);
			fill_m2l_kernel_times(ctx, stats);
		}
	}
	return OK;
}

} // namespace lfmm
