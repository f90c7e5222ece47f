// 3D rotation-based Laplace FMM, plain FP64 form.
//
// Operators follow the reference's CPU solver (cpu/multipole3d.cpp): P2M
// 20-49, rotate-z / rotate-y 51-113, M2M / M2L / L2L as rotate, z-translate,
// rotate back 115-226, passes 228-412, P2P + L2P 855-1294.  Every kernel is
// warp-per-box (P2M, M2M, M2L, L2L) or block-per-leaf (P2P + L2P); lanes own
// expansion coefficients, per-box data is staged in shared memory, there are
// no atomics and no per-thread local arrays.
#include "fmm3d.cuh"
#include "m2l_gemm.cuh"
#include <algorithm>

namespace lfmm {

namespace {

constexpr int CMAX = (MAXN3 * (MAXN3 + 1) / 2 + 31) / 32;   // coefficients per lane (6)
constexpr int NX2MAX = MAXN3 * (MAXN3 + 1) / 2;             // 171
constexpr int WPB = 4;                                      // warps per block, box kernels


enum { OP_M2M = 0, OP_M2L = 1, OP_L2L = 2 };

struct Exp {
	int N, Nx2;
	double2* outer;
	double2* inner;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{ return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

__device__ __forceinline__ int dir_id(int dx, int dy, int dz) { return (dx + 3) * 49 + (dy + 3) * 7 + (dz + 3); }

__device__ __forceinline__ void coords3(uint64_t code, int* c)
{ c[0] = (int)compact3(code >> 2); c[1] = (int)compact3(code >> 1); c[2] = (int)compact3(code); }

// res[n,m] = d(n,m,0) a[n,0] + sum_k (Re a[n,k](d_{m,k}+d_{m,-k}), Im a[n,k](d_{m,k}-d_{m,-k}))
__device__ __forceinline__ void rotate_y_warp(const double2* __restrict__ in, double2* __restrict__ out,
                                              const double* __restrict__ D, int Nx2)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int t = 0; t < CMAX; ++t) {
		int c = lane + 32 * t;
		if (c < Nx2) {
			const int n = tri_row(c), m = c - tix(n, 0);
			const double* Dr = D + dix(n, m, 0);
			double vr = 0.0, vi = 0.0;
			const double2* row = in + tix(n, 0);
			for (int k = 1; k <= n; ++k) {
				double z1 = Dr[k], z2 = Dr[-k];
				double2 w = row[k];
				vr = fma(w.x, z1 + z2, vr);
				vi = fma(w.y, z1 - z2, vi);
			}
			double d0 = Dr[0];
			vr = fma(d0, row[0].x, vr);
			vi = fma(d0, row[0].y, vi);
			out[c] = make_double2(vr, vi);
		}
	}
}

struct Smem {
	double2 a[NX2MAX];
	double2 b[NX2MAX];
	double rn[2 * MAXN3 + 2];
};

// acc += R_z(-phi) R_y(-theta) T_z(rho) R_y(theta) R_z(phi) src, warp-cooperative.
template <int OP>
__device__ void translate_warp(const double2* __restrict__ src, double px, double py, double pz, int dirid,
                               double2 (&acc)[CMAX], int N, int Nx2, Smem& sm, const DevTables& T, unsigned* flags)
{
	const int lane = threadIdx.x & 31;
	int4 di = T.dirinfo[dirid];
	if (di.x < 0 || di.y < 0 || di.z < 0 || di.w < 0) {
		if (lane == 0) atomicOr(flags, DEV_ERR_DIRECTION);
		return;
	}
	const double* D1 = T.dmat + (size_t)di.x * dsize(MAXN3);
	const double* D2 = T.dmat + (size_t)di.y * dsize(MAXN3);
	const double2* E1 = T.emat + di.z * MAXN3;
	const double2* E2 = T.emat + di.w * MAXN3;
	double rho = sqrt(px * px + py * py + pz * pz) + 1e-12;
	if (OP == OP_M2L) {
		double inv = 1.0 / rho;
		for (int i = lane; i < 2 * N + 1; i += 32) {
			double p = 1.0;
			for (int j = 0; j < i; ++j) p *= inv;
			sm.rn[i] = p;
		}
	} else {
		for (int i = lane; i < N; i += 32) {
			double p = 1.0;
			for (int j = 0; j < i; ++j) p *= rho;
			sm.rn[i] = p;
		}
	}
#pragma unroll
	for (int t = 0; t < CMAX; ++t) {
		int c = lane + 32 * t;
		if (c < Nx2) sm.a[c] = cmul(src[c], E1[c - tix(tri_row(c), 0)]);
	}
	__syncwarp();
	rotate_y_warp(sm.a, sm.b, D1, Nx2);
	__syncwarp();
	const double* cube = OP == OP_M2L ? T.m2l : (OP == OP_M2M ? T.m2m : T.l2l);
#pragma unroll
	for (int t = 0; t < CMAX; ++t) {
		int c = lane + 32 * t;
		if (c < Nx2) {
			const int j = tri_row(c), k = c - tix(j, 0);
			const double* cf = cube + (j * MAXN3 + k) * MAXN3;
			double sr = 0.0, si = 0.0;
			if (OP == OP_M2L) {
				for (int n = k; n < N; ++n) {
					double f = cf[n] * sm.rn[j + n + 1];
					double2 w = sm.b[tix(n, k)];
					sr = fma(f, w.x, sr); si = fma(f, w.y, si);
				}
			} else if (OP == OP_M2M) {
				for (int n = 0; j - n >= k; ++n) {
					double f = cf[n] * sm.rn[n];
					double2 w = sm.b[tix(j - n, k)];
					sr = fma(f, w.x, sr); si = fma(f, w.y, si);
				}
			} else {
				for (int n = j; n < N; ++n) {
					double f = cf[n] * sm.rn[n - j];
					double2 w = sm.b[tix(n, k)];
					sr = fma(f, w.x, sr); si = fma(f, w.y, si);
				}
			}
			sm.a[c] = make_double2(sr, si);
		}
	}
	__syncwarp();
	rotate_y_warp(sm.a, sm.b, D2, Nx2);
	__syncwarp();
#pragma unroll
	for (int t = 0; t < CMAX; ++t) {
		int c = lane + 32 * t;
		if (c < Nx2) {
			double2 v = cmul(sm.b[c], E2[c - tix(tri_row(c), 0)]);
			acc[t].x += v.x; acc[t].y += v.y;
		}
	}
	__syncwarp();
}

// ---------------------------------------------------------------- P2M
__global__ void __launch_bounds__(WPB * 32) p2m_kernel(DevTree t, Exp E, const double* __restrict__ knm)
{
	__shared__ double2 sacc[WPB][NX2MAX];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int LL = t.depth - 1;
	size_t leaf = (size_t)blockIdx.x * WPB + w;
	if (leaf >= t.lsize[LL]) return;
	size_t g = t.loff[LL] + leaf;
	const int N = E.N, Nx2 = E.Nx2;
	for (int c = lane; c < Nx2; c += 32) sacc[w][c] = make_double2(0.0, 0.0);
	__syncwarp();
	const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
	const uint32_t b = t.beg[g], e = t.end[g];
	for (uint32_t base = b; base < e; base += 32) {
		uint32_t i = base + lane;
		double q = 0.0, r = 1.0, th = 1.0, ph = 0.0;
		if (i < e) {
			q = t.q[i];
			dec_to_sph(t.x[i] - cx, t.y[i] - cy, t.z[i] - cz, r, th, ph);
		}
		double y, x;
		sincos(th, &y, &x);
		double Pmm = 1.0, rpow = 1.0;
		for (int m = 0; m < N; ++m) {
			if (m > 0) { Pmm = Pmm * y * (1 - 2 * m); rpow *= r; }
			double sm_, cm_;
			sincos(m * ph, &sm_, &cm_);
			// r^n: r^m at n = m (r^0 = 1), then one factor of r per degree
			double Pn = Pmm, Pn1 = 0.0, rn = rpow;
			for (int n = m; n < N; ++n) {
				if (n > m) {
					double Pnew = (n == m + 1) ? Pmm * x * (2 * n - 1)
					                           : ((2 * n - 1) * x * Pn - (n + m - 1) * Pn1) / (n - m);
					Pn1 = Pn; Pn = Pnew; rn *= r;
				}
				double vr, vi;
				if (n == 0) { vr = q; vi = 0.0; }
				else {
					double f = q * rn * knm[tix(n, m)] * Pn;
					vr = f * cm_; vi = -f * sm_;
				}
				vr = warp_sum(vr); vi = warp_sum(vi);
				if (lane == 0) {
					double2 a = sacc[w][tix(n, m)];
					sacc[w][tix(n, m)] = make_double2(a.x + vr, a.y + vi);
				}
			}
		}
	}
	__syncwarp();
	double2* out = E.outer + g * Nx2;
	for (int c = lane; c < Nx2; c += 32) out[c] = sacc[w][c];
}

// ---------------------------------------------------------------- M2M
__global__ void __launch_bounds__(WPB * 32) m2m_kernel(DevTree t, Exp E, int L, DevTables T, unsigned* flags)
{
	__shared__ Smem sm[WPB];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t c = (size_t)blockIdx.x * WPB + w;
	if (c >= t.lsize[L]) return;
	size_t g = t.loff[L] + c, cb = t.loff[L + 1];
	double2 acc[CMAX];
#pragma unroll
	for (int k = 0; k < CMAX; ++k) acc[k] = make_double2(0.0, 0.0);
	for (uint32_t k = t.beg[g]; k < t.end[g]; ++k) {
		size_t gk = cb + k;
		uint64_t oct = t.code[gk] & 7ull;
		int d = dir_id(2 * (int)((oct >> 2) & 1) - 1, 2 * (int)((oct >> 1) & 1) - 1, 2 * (int)(oct & 1) - 1);
		translate_warp<OP_M2M>(E.outer + gk * E.Nx2, t.cx[gk] - t.cx[g], t.cy[gk] - t.cy[g], t.cz[gk] - t.cz[g], d,
		                       acc, E.N, E.Nx2, sm[w], T, flags);
	}
	double2* out = E.outer + g * E.Nx2;
#pragma unroll
	for (int k = 0; k < CMAX; ++k) {
		int cc = lane + 32 * k;
		if (cc < E.Nx2) out[cc] = acc[k];
	}
}

// ---------------------------------------------------------------- M2L
// Far list of c: children of the parent's close cells and of the parent that
// are not adjacent to c (reference cpu/morton_tree.cpp:147-208), in that order.
__global__ void __launch_bounds__(WPB * 32) m2l_kernel(DevTree t, Exp E, int L, DevTables T, unsigned* flags)
{
	__shared__ Smem sm[WPB];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t c = (size_t)blockIdx.x * WPB + w;
	if (c >= t.lsize[L]) return;
	size_t off = t.loff[L], poff = t.loff[L - 1];
	size_t g = off + c;
	int me[3];
	coords3(t.code[g], me);
	double2 acc[CMAX];
#pragma unroll
	for (int k = 0; k < CMAX; ++k) acc[k] = make_double2(0.0, 0.0);
	int32_t p = t.parent[g];
	int npc = t.close_cnt[poff + p];
	const int32_t* pl = t.close_idx + (poff + p) * t.close_stride;
	const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
	for (int e = 0; e <= npc; ++e) {
		int32_t pn = e < npc ? pl[e] : p;
		for (uint32_t k = t.beg[poff + pn]; k < t.end[poff + pn]; ++k) {
			if (k == c) continue;
			size_t gk = off + k;
			int o[3];
			coords3(t.code[gk], o);
			int dx = o[0] - me[0], dy = o[1] - me[1], dz = o[2] - me[2];
			if (max(max(abs(dx), abs(dy)), abs(dz)) <= 1) continue;
			translate_warp<OP_M2L>(E.outer + gk * E.Nx2, t.cx[gk] - cx, t.cy[gk] - cy, t.cz[gk] - cz,
			                       dir_id(dx, dy, dz), acc, E.N, E.Nx2, sm[w], T, flags);
		}
	}
	double2* out = E.inner + g * E.Nx2;
#pragma unroll
	for (int k = 0; k < CMAX; ++k) {
		int cc = lane + 32 * k;
		if (cc < E.Nx2) out[cc] = acc[k];
	}
}

// ---------------------------------------------------------------- L2L
__global__ void __launch_bounds__(WPB * 32) l2l_kernel(DevTree t, Exp E, int L, DevTables T, unsigned* flags)
{
	__shared__ Smem sm[WPB];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t c = (size_t)blockIdx.x * WPB + w;
	if (c >= t.lsize[L]) return;
	size_t g = t.loff[L] + c;
	size_t gp = t.loff[L - 1] + t.parent[g];
	double2* out = E.inner + g * E.Nx2;
	double2 acc[CMAX];
#pragma unroll
	for (int k = 0; k < CMAX; ++k) {
		int cc = lane + 32 * k;
		acc[k] = cc < E.Nx2 ? out[cc] : make_double2(0.0, 0.0);
	}
	uint64_t oct = t.code[g] & 7ull;
	int d = dir_id(1 - 2 * (int)((oct >> 2) & 1), 1 - 2 * (int)((oct >> 1) & 1), 1 - 2 * (int)(oct & 1));
	translate_warp<OP_L2L>(E.inner + gp * E.Nx2, t.cx[gp] - t.cx[g], t.cy[gp] - t.cy[g], t.cz[gp] - t.cz[g], d, acc,
	                       E.N, E.Nx2, sm[w], T, flags);
#pragma unroll
	for (int k = 0; k < CMAX; ++k) {
		int cc = lane + 32 * k;
		if (cc < E.Nx2) out[cc] = acc[k];
	}
}

// ---------------------------------------------------------------- P2P + L2P
constexpr int LEAF_THREADS = 128;

// Local expansion evaluated at one target (reference cpu/multipole3d.cpp:
// 1152-1208): Legendre recurrence streamed degree by degree per order m,
// potential and the spherical-gradient field, then the Cartesian transform.
__device__ void l2p_eval(const double2* __restrict__ Lc, double dx, double dy, double dz, int N,
                         const double* __restrict__ knm, double& pot, double& fx, double& fy, double& fz)
{
	double r, th, ph;
	dec_to_sph(dx, dy, dz, r, th, ph);
	double y, x;
	sincos(th, &y, &x);
	double phi = 0.0, mt0 = 0.0, mt1 = 0.0, mt2 = 0.0;
	double Pmm = 1.0, rpow = 1.0 / r;
	for (int m = 0; m < N; ++m) {
		if (m > 0) { Pmm = Pmm * y * (1 - 2 * m); rpow *= r; }
		double sm_, cm_;
		sincos(m * ph, &sm_, &cm_);
		const double mult = m ? 2.0 : 1.0;
		double Pn = Pmm, Pn1 = 0.0, rn = rpow;
		for (int n = m; n < N; ++n) {
			double Pnext = (n == m) ? Pmm * x * (2 * n + 1)
			                        : ((2 * n + 1) * x * Pn - (n + m) * Pn1) / (n + 1 - m);
			double K = knm[tix(n, m)];
			double Yr = Pn * cm_ * K, Yi = Pn * sm_ * K;
			double2 Lnm = Lc[tix(n, m)];
			double cr = Lnm.x * rn, ci = Lnm.y * rn;
			double ycr = Yr * cr - Yi * ci;                       // Re(Y coef)
			phi += mult * (r * ycr);
			double g = K * ((1 - m + n) * Pnext - (n + 1) * x * Pn) / y;
			double dthr = cm_ * g, dthi = sm_ * g;
			mt0 -= mult * (n * ycr);
			mt1 -= mult * (cr * dthr - ci * dthi);
			mt2 -= mult * (cr * (-m * Yi) - ci * (m * Yr));
			Pn1 = Pn; Pn = Pnext; rn *= r;
		}
	}
	pot += phi;
	double s2, c2;
	sincos(ph, &s2, &c2);
	const double s1 = y, c1 = x;
	fx += mt0 * s1 * c2 + mt1 * c1 * c2 - mt2 * s2 / s1;
	fy += mt0 * s1 * s2 + mt1 * c1 * s2 + mt2 * c2 / s1;
	fz += mt0 * c1 - mt1 * s1;
}

// One block per leaf: targets of the leaf against the leaf's sources and
// every close leaf's sources, staged through shared memory in tiles, then
// L2P; results scattered to input order.  q / max(r, 1e-4) and
// q (r_i - r_j) / max(r, 1e-4)^3 as reference common/avx.h:128-146.
__global__ void __launch_bounds__(LEAF_THREADS) leaves_kernel(DevTree t, Exp E, const double* __restrict__ knm,
                                                              double* __restrict__ pot_out,
                                                              double* __restrict__ fld_out)
{
	__shared__ double sx[LEAF_THREADS], sy[LEAF_THREADS], sz[LEAF_THREADS], sq[LEAF_THREADS];
	__shared__ double2 sL[NX2MAX];
	const int LL = t.depth - 1;
	size_t leaf = blockIdx.x;
	if (leaf >= t.lsize[LL]) return;
	size_t off = t.loff[LL], g = off + leaf;
	const bool tmode = t.targets_num > 0;
	const uint32_t tb = tmode ? t.tbeg[g] : t.beg[g];
	const uint32_t te = tmode ? t.tend[g] : t.end[g];
	if (tb >= te) return;
	for (int c = threadIdx.x; c < E.Nx2; c += LEAF_THREADS) sL[c] = E.inner[g * E.Nx2 + c];
	const int ncl = t.close_cnt[g];
	const int32_t* cl = t.close_idx + g * t.close_stride;
	const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
	for (uint32_t t0 = tb; t0 < te; t0 += LEAF_THREADS) {
		uint32_t i = t0 + threadIdx.x;
		const bool valid = i < te;
		double xi = 0.0, yi = 0.0, zi = 0.0;
		if (valid) { xi = t.x[i]; yi = t.y[i]; zi = t.z[i]; }
		double pot = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
		for (int e = -1; e < ncl; ++e) {
			size_t sc = e < 0 ? g : off + cl[e];
			const uint32_t sb = t.beg[sc], se = t.end[sc];
			for (uint32_t s0 = sb; s0 < se; s0 += LEAF_THREADS) {
				const int cnt = min((uint32_t)LEAF_THREADS, se - s0);
				__syncthreads();
				if (threadIdx.x < cnt) {
					uint32_t j = s0 + threadIdx.x;
					sx[threadIdx.x] = t.x[j]; sy[threadIdx.x] = t.y[j]; sz[threadIdx.x] = t.z[j]; sq[threadIdx.x] = t.q[j];
				}
				__syncthreads();
				if (valid) {
					for (int j = 0; j < cnt; ++j) {
						double dx = xi - sx[j], dy = yi - sy[j], dz = zi - sz[j];
						double r2 = fmax(dx * dx + dy * dy + dz * dz, FORCE_EPS2);
						double inv = rsqrt(r2);
						double qi = sq[j] * inv;
						double qi3 = qi * inv * inv;
						pot += qi;
						fx = fma(dx, qi3, fx); fy = fma(dy, qi3, fy); fz = fma(dz, qi3, fz);
					}
				}
			}
		}
		__syncthreads();
		if (valid) {
			l2p_eval(sL, xi - cx, yi - cy, zi - cz, E.N, knm, pot, fx, fy, fz);
			uint32_t o = t.orig[i];
			pot_out[o] = pot;
			fld_out[3 * (size_t)o] = fx; fld_out[3 * (size_t)o + 1] = fy; fld_out[3 * (size_t)o + 2] = fz;
		}
	}
}

// Dense M2L operators of one level: column r of T_d is the rotation-based
// M2L (the same translate_warp as the per-pair path) applied to the r-th
// unit vector, for the far offset d * h.  out: [343][MT][MT], pre-zeroed.
__global__ void __launch_bounds__(WPB * 32) m2l_ops_kernel(int N, int MT, double h, DevTables T, double* out,
                                                           unsigned* flags)
{
	__shared__ Smem sm[WPB];
	__shared__ double2 unit[WPB][NX2MAX];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int Nx2 = N * (N + 1) / 2, R = 2 * Nx2;
	size_t task = (size_t)blockIdx.x * WPB + w;
	int dirid = (int)(task / R), r = (int)(task % R);
	if (dirid >= 343) return;
	int dx = dirid / 49 - 3, dy = (dirid / 7) % 7 - 3, dz = dirid % 7 - 3;
	if (max(max(abs(dx), abs(dy)), abs(dz)) <= 1) return;
	for (int c = lane; c < Nx2; c += 32)
		unit[w][c] = make_double2(c == r / 2 && !(r & 1) ? 1.0 : 0.0, c == r / 2 && (r & 1) ? 1.0 : 0.0);
	__syncwarp();
	double2 acc[CMAX];
#pragma unroll
	for (int k = 0; k < CMAX; ++k) acc[k] = make_double2(0.0, 0.0);
	translate_warp<OP_M2L>(unit[w], dx * h, dy * h, dz * h, dirid, acc, N, Nx2, sm[w], T, flags);
	double* op = out + (size_t)dirid * MT * MT;
#pragma unroll
	for (int k = 0; k < CMAX; ++k) {
		int c = lane + 32 * k;
		if (c < Nx2) {
			op[(size_t)(2 * c) * MT + r] = acc[k].x;
			op[(size_t)(2 * c + 1) * MT + r] = acc[k].y;
		}
	}
}


// The plain form's kernels need no constant tables (the (n, m) of a
// triangular index is computed: tri_row); kept as the solvers' setup hook.
int upload_constants(Context& ctx)
{
	(void)ctx;
	return OK;
}

} // namespace

// Dense FP64 M2L operators for cell size h, cached in the context.
double* m2l_ops_fp64(Context& ctx, int N, double h)
{
	for (auto& e : ctx.opcache)
		if (e.N == N && e.prec == 0 && e.h == h) { e.stamp = ++ctx.opcache_clock; return static_cast<double*>(e.ptr); }
	if (upload_constants(ctx)) return nullptr;
	const int MT = m2l_padded(N), R = N * (N + 1);
	size_t bytes = sizeof(double) * 343 * (size_t)MT * MT;
	opcache_make_room(ctx);
	OpCacheEntry e;
	e.N = N; e.prec = 0; e.h = h; e.bytes = bytes; e.stamp = ++ctx.opcache_clock;
	if (cudaMalloc(&e.ptr, bytes) != cudaSuccess) { cudaGetLastError(); ctx.last_error = "m2l operators: out of memory"; return nullptr; }
	cudaMemsetAsync(e.ptr, 0, bytes, ctx.stream);
	size_t tasks = (size_t)343 * R;
	m2l_ops_kernel<<<div_up(tasks, WPB), WPB * 32, 0, ctx.stream>>>(N, MT, h, ctx.tables.d, static_cast<double*>(e.ptr),
	                                                                 ctx.dev_flags);
	if (cudaGetLastError() != cudaSuccess) { cudaFree(e.ptr); ctx.last_error = "m2l operators: launch failed"; return nullptr; }
	ctx.opcache.push_back(e);
	return static_cast<double*>(e.ptr);
}

int fmm3d_solve_device(Context& ctx, const ParticleInput& in, int N, int depth, double* pot, double* field,
                       SolveStats* stats, DevTree* tree_out, double2** inner_out, double2** outer_out)
{
	if (N < 1 || N > MAXN3) { ctx.last_error = "order out of range (1 <= N <= 18)"; return ERR_ARG; }
	int st = upload_constants(ctx);
	if (st) return st;
	cudaStream_t s = ctx.stream;
	const bool timing = ctx.timing != 0;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[0], s));
	DevTree t;
	st = tree_build(ctx, in, depth, t);
	if (st) return st;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[1], s));
	Exp E;
	E.N = N; E.Nx2 = N * (N + 1) / 2;
	E.outer = static_cast<double2*>(ctx.arena.take(sizeof(double2) * t.ncells * E.Nx2));
	E.inner = static_cast<double2*>(ctx.arena.take(sizeof(double2) * t.ncells * E.Nx2));
	unsigned long long* counters = static_cast<unsigned long long*>(ctx.arena.take(32));
	if (!E.outer || !E.inner || !counters) { ctx.last_error = "fmm3d: device allocation failed"; return ERR_OOM; }
	const int LL = depth - 1;
	const size_t n_out = in.nt ? in.nt : in.ns;
	LFMM_CUDA(ctx, cudaMemsetAsync(pot, 0, sizeof(double) * n_out, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(field, 0, sizeof(double) * 3 * n_out, s));
	size_t lo = depth > 2 ? t.loff[2] : t.ncells;
	LFMM_CUDA(ctx, cudaMemsetAsync(E.inner, 0, sizeof(double2) * lo * E.Nx2, s));
	// upward
	p2m_kernel<<<div_up(t.lsize[LL], WPB), WPB * 32, 0, s>>>(t, E, ctx.tables.d.knm);
	for (int L = depth - 2; L >= 0; --L)
		m2m_kernel<<<div_up(t.lsize[L], WPB), WPB * 32, 0, s>>>(t, E, L, ctx.tables.d, ctx.dev_flags);
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[2], s));
	// downward
	const bool gemm = ctx.m2l_engine != 1 && m2l_gemm_supported(N);     // FP64: SIMT GEMMs unless rotations asked
	for (int L = 2; L < depth; ++L) {
		if (gemm) {
			double h = t.geo_host[3] / (double)(1ull << L);
			double* ops = m2l_ops_fp64(ctx, N, h);
			if (!ops) return ERR_OOM;
			M2LPlan plan;
			if ((st = m2l_plan_build(ctx, t, L, plan))) return st;
			const size_t off = t.loff[L] * E.Nx2;
			if ((st = m2l_gemm<double>(ctx, plan, ops, reinterpret_cast<const double*>(E.outer + off),
			                           reinterpret_cast<double*>(E.inner + off), N)))
				return st;
		} else {
			m2l_kernel<<<div_up(t.lsize[L], WPB), WPB * 32, 0, s>>>(t, E, L, ctx.tables.d, ctx.dev_flags);
		}
	}
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[3], s));
	for (int L = 3; L < depth; ++L)
		l2l_kernel<<<div_up(t.lsize[L], WPB), WPB * 32, 0, s>>>(t, E, L, ctx.tables.d, ctx.dev_flags);
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[4], s));
	leaves_kernel<<<(unsigned)t.lsize[LL], LEAF_THREADS, 0, s>>>(t, E, ctx.tables.d.knm, pot, field);
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[5], s));
	LFMM_CUDA(ctx, cudaGetLastError());
	if (stats) {
		unsigned long long h[3];
		if ((st = tree_count_pairs(ctx, t, counters, h))) return st;
		stats->N = N; stats->depth = depth;
		stats->n_particles = t.n; stats->n_cells = t.ncells; stats->n_leaves = t.lsize[LL];
		stats->targets_num = t.targets_num;
		stats->n_far_pairs = h[0]; stats->n_close_pairs = h[1]; stats->n_p2p_pairs = h[2];
		if (timing) {
			cudaEventElapsedTime(&stats->ms_tree, ctx.ev[0], ctx.ev[1]);
			cudaEventElapsedTime(&stats->ms_upward, ctx.ev[1], ctx.ev[2]);
			cudaEventElapsedTime(&stats->ms_m2l, ctx.ev[2], ctx.ev[3]);
			cudaEventElapsedTime(&stats->ms_l2l, ctx.ev[3], ctx.ev[4]);
			cudaEventElapsedTime(&stats->ms_leaves, ctx.ev[4], ctx.ev[5]);
			cudaEventElapsedTime(&stats->ms_total, ctx.ev[0], ctx.ev[5]);
		}
	}
	if (tree_out) *tree_out = t;
	if (inner_out) *inner_out = E.inner;
	if (outer_out) *outer_out = E.outer;
	return OK;
}

} // namespace lfmm
