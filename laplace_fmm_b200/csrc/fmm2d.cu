// 2D Laplace FMM, FP64, following the reference's CPU solver
// (cpu/multipole.cpp): P2M 22-36, M2M 38-53, M2L 66-84, L2L 86-97, passes
// 99-231 (per level: L2L from the parent, then M2L from the far list),
// leaves 233-449 (P2P + L2P for potential and field).
// Warp per box with one expansion coefficient per lane (N <= 30), block per
// leaf for the near field.
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
// k over the leaf's particles, staged 32 at a time.
__global__ void __launch_bounds__(WPB2 * 32) p2m2d_kernel(DevTree t, Exp2 E)
{
	__shared__ double2 sz[WPB2][32];
	__shared__ double sq[WPB2][32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int LL = t.depth - 1;
	size_t leaf = (size_t)blockIdx.x * WPB2 + w;
	if (leaf >= t.lsize[LL]) return;
	size_t g = t.loff[LL] + leaf;
	const int N = E.N;
	const double cx = t.cx[g], cy = t.cy[g];
	const uint32_t pb = t.beg[g], pe = t.end[g];
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

std::mutex g_binom_mu;
bool g_binom_ready[64] = {};

} // namespace

int fmm2d_solve_device(Context& ctx, const ParticleInput& in, int N, int depth, double* pot, double* field,
                       SolveStats* stats)
{
	if (N < 1 || N > MAXN2) { ctx.last_error = "order out of range (1 <= N <= 30)"; return ERR_ARG; }
	if (ctx.device < 0 || ctx.device >= 64) { ctx.last_error = "device index above 63"; return ERR_ARG; }
	std::unique_lock<std::mutex> lock(g_binom_mu);
	if (!g_binom_ready[ctx.device]) {
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
	}
	lock.unlock();
	cudaStream_t s = ctx.stream;
	const bool timing = ctx.timing != 0;
	ctx.kev_used = 0;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[0], s));
	DevTree t;
	int st = tree_build(ctx, in, depth, t);
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
		// M2L grouped by (quadrant class, offset), all levels: the Hankel
		// factorisation (default) or dense operators (simt); then the L2L
		// passes top-down
		const size_t mark = ctx.arena.mark();
		for (int L = 2; L < depth; ++L) {
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
			stats->ms_m2l_kernel = 0.f;
			for (int k = 0; k + 1 < ctx.kev_used; k += 2) {
				float ms = 0.f;
				cudaEventElapsedTime(&ms, ctx.kev[k], ctx.kev[k + 1]);
				stats->ms_m2l_kernel += ms;
			}
			stats->n_m2l_kernel = ctx.kev_used / 2;
		}
	}
	return OK;
}

} // namespace lfmm
