// 3D FMM, mixed-precision form.
//
// Same tree (FP64, bit-exact) and operators as the plain form, in scaled
// expansions: multipole a_nm / h^n and local L_nm h^(n+1) for a level of cell
// size h.  Scaled, every operator is level-independent and every coefficient
// is O(total charge), so FP32 holds them without underflow at depth:
//   M2L   rho / h = |d|                      (one operator per far offset d)
//   M2M   (rho / h_child)^n, row j times 2^-j
//   L2L   (rho / h_parent)^(n-j), row j times 2^-(j+1)
//   P2M / L2P with r / h; potential times 1/h, field times 1/h^2.
// Levels 0-3 stay FP64 (their expansions carry the coarse far field); levels
// 4 and below run in FP32.  The near field runs in FP32 on leaf-relative
// coordinates (pair offsets accurate to ~1e-7 of the leaf size), with per-tile
// partial sums carried in FP64 (compensated summation per target) and the
// self term q_i / 1e-4 added in FP64.
#include "fmm3d.cuh"
#include "m2l_gemm.cuh"

namespace lfmm {

double* m2l_ops_fp64(Context& ctx, int N, double h);

namespace {

constexpr int CMAX = (MAXN3 * (MAXN3 + 1) / 2 + 31) / 32;
constexpr int NX2MAX = MAXN3 * (MAXN3 + 1) / 2;
constexpr int WPB = 4;
constexpr int FP64_LEVELS = 4;   // levels < 4 run in FP64

__constant__ unsigned char c_n_of[NX2MAX];
__constant__ unsigned char c_m_of[NX2MAX];

template <typename real> struct V2;
template <> struct V2<double> { using t = double2; static __device__ __forceinline__ double2 make(double a, double b) { return make_double2(a, b); } };
template <> struct V2<float> { using t = float2; static __device__ __forceinline__ float2 make(float a, float b) { return make_float2(a, b); } };

template <typename real>
struct Tab {
	const real* dmat;
	const typename V2<real>::t* emat;
	const real* m2m;
	const real* l2l;
	const real* knm;
	const int4* dirinfo;
};

template <typename real>
__device__ __forceinline__ typename V2<real>::t cmulv(typename V2<real>::t a, typename V2<real>::t b)
{ return V2<real>::make(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

__device__ __forceinline__ void coords3(uint64_t code, int* c)
{ c[0] = (int)compact3(code >> 2); c[1] = (int)compact3(code >> 1); c[2] = (int)compact3(code); }
__device__ __forceinline__ int dir_id(int dx, int dy, int dz) { return (dx + 3) * 49 + (dy + 3) * 7 + (dz + 3); }

template <typename real>
struct SmemT {
	typename V2<real>::t a[NX2MAX];
	typename V2<real>::t b[NX2MAX];
	real rn[2 * MAXN3 + 2];
};

template <typename real>
__device__ __forceinline__ void rotate_y_t(const typename V2<real>::t* __restrict__ in, typename V2<real>::t* __restrict__ out,
                                           const real* __restrict__ D, int Nx2)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int t = 0; t < CMAX; ++t) {
		int c = lane + 32 * t;
		if (c < Nx2) {
			int n = c_n_of[c], m = c_m_of[c];
			const real* Dr = D + dix(n, m, 0);
			real vr = 0, vi = 0;
			const typename V2<real>::t* row = in + tix(n, 0);
			for (int k = 1; k <= n; ++k) {
				real z1 = Dr[k], z2 = Dr[-k];
				typename V2<real>::t w = row[k];
				vr = fma(w.x, z1 + z2, vr);
				vi = fma(w.y, z1 - z2, vi);
			}
			real d0 = Dr[0];
			vr = fma(d0, row[0].x, vr);
			vi = fma(d0, row[0].y, vi);
			out[c] = V2<real>::make(vr, vi);
		}
	}
}

enum { SOP_M2M = 0, SOP_L2L = 1 };

// Scaled M2M / L2L along one of the 8 diagonal offsets (warp-cooperative).
template <int OP, typename real>
__device__ void translate_scaled(const typename V2<real>::t* __restrict__ src, int dirid,
                                 typename V2<real>::t (&acc)[CMAX], int N, int Nx2, SmemT<real>& sm,
                                 const Tab<real>& T, unsigned* flags)
{
	const int lane = threadIdx.x & 31;
	int4 di = T.dirinfo[dirid];
	if (di.x < 0 || di.y < 0 || di.z < 0 || di.w < 0) {
		if (lane == 0) atomicOr(flags, DEV_ERR_DIRECTION);
		return;
	}
	const real* D1 = T.dmat + (size_t)di.x * dsize(MAXN3);
	const real* D2 = T.dmat + (size_t)di.y * dsize(MAXN3);
	const typename V2<real>::t* E1 = T.emat + di.z * MAXN3;
	const typename V2<real>::t* E2 = T.emat + di.w * MAXN3;
	// M2M: rho / h_child = sqrt(3)/2 ; L2L: rho / h_parent = sqrt(3)/4
	const double rho = OP == SOP_M2M ? 0.86602540378443864676 : 0.43301270189221932338;
	for (int i = lane; i < N; i += 32) {
		double p = 1.0;
		for (int j = 0; j < i; ++j) p *= rho;
		sm.rn[i] = (real)p;
	}
#pragma unroll
	for (int t = 0; t < CMAX; ++t) {
		int c = lane + 32 * t;
		if (c < Nx2) sm.a[c] = cmulv<real>(src[c], E1[c_m_of[c]]);
	}
	__syncwarp();
	rotate_y_t<real>(sm.a, sm.b, D1, Nx2);
	__syncwarp();
	const real* cube = OP == SOP_M2M ? T.m2m : T.l2l;
#pragma unroll
	for (int t = 0; t < CMAX; ++t) {
		int c = lane + 32 * t;
		if (c < Nx2) {
			int j = c_n_of[c], k = c_m_of[c];
			const real* cf = cube + (j * MAXN3 + k) * MAXN3;
			real sr = 0, si = 0;
			if (OP == SOP_M2M) {
				for (int n = 0; j - n >= k; ++n) {
					real f = cf[n] * sm.rn[n];
					typename V2<real>::t w = sm.b[tix(j - n, k)];
					sr = fma(f, w.x, sr); si = fma(f, w.y, si);
				}
				real s = (real)ldexp(1.0, -j);
				sr *= s; si *= s;
			} else {
				for (int n = j; n < N; ++n) {
					real f = cf[n] * sm.rn[n - j];
					typename V2<real>::t w = sm.b[tix(n, k)];
					sr = fma(f, w.x, sr); si = fma(f, w.y, si);
				}
				real s = (real)ldexp(1.0, -(j + 1));
				sr *= s; si *= s;
			}
			sm.a[c] = V2<real>::make(sr, si);
		}
	}
	__syncwarp();
	rotate_y_t<real>(sm.a, sm.b, D2, Nx2);
	__syncwarp();
#pragma unroll
	for (int t = 0; t < CMAX; ++t) {
		int c = lane + 32 * t;
		if (c < Nx2) {
			typename V2<real>::t v = cmulv<real>(sm.b[c], E2[c_m_of[c]]);
			acc[t].x += v.x; acc[t].y += v.y;
		}
	}
	__syncwarp();
}

// parent (level L, array par) = sum of scaled M2M from its children (level L+1, array chi)
template <typename real>
__global__ void __launch_bounds__(WPB * 32) m2m_scaled_kernel(DevTree t, int L, const typename V2<real>::t* __restrict__ chi,
                                                              typename V2<real>::t* __restrict__ par, int N,
                                                              Tab<real> T, unsigned* flags)
{
	__shared__ SmemT<real> sm[WPB];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t c = (size_t)blockIdx.x * WPB + w;
	if (c >= t.lsize[L]) return;
	const int Nx2 = N * (N + 1) / 2;
	size_t g = t.loff[L] + c, cb = t.loff[L + 1];
	typename V2<real>::t acc[CMAX];
#pragma unroll
	for (int k = 0; k < CMAX; ++k) acc[k] = V2<real>::make(0, 0);
	for (uint32_t k = t.beg[g]; k < t.end[g]; ++k) {
		uint64_t oct = t.code[cb + k] & 7ull;
		int d = dir_id(2 * (int)((oct >> 2) & 1) - 1, 2 * (int)((oct >> 1) & 1) - 1, 2 * (int)(oct & 1) - 1);
		translate_scaled<SOP_M2M, real>(chi + (size_t)k * Nx2, d, acc, N, Nx2, sm[w], T, flags);
	}
	typename V2<real>::t* out = par + c * Nx2;
#pragma unroll
	for (int k = 0; k < CMAX; ++k) {
		int cc = lane + 32 * k;
		if (cc < Nx2) out[cc] = acc[k];
	}
}

// Float leaf-relative coordinates and charges, block per leaf.
__global__ void relcoords_kernel(DevTree t, float* __restrict__ xr, float* __restrict__ yr, float* __restrict__ zr,
                                 float* __restrict__ qf)
{
	const int LL = t.depth - 1;
	size_t leaf = blockIdx.x;
	if (leaf >= t.lsize[LL]) return;
	size_t g = t.loff[LL] + leaf;
	const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
	uint32_t b = t.beg[g], e = t.tend[g] > t.end[g] ? t.tend[g] : t.end[g];
	for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x) {
		xr[i] = (float)(t.x[i] - cx); yr[i] = (float)(t.y[i] - cy); zr[i] = (float)(t.z[i] - cz);
		qf[i] = (float)t.q[i];
	}
}

// P2M in scaled form: a~_nm = sum q (r/h)^n K_nm P_nm(cos t) e^{-i m phi} (FP32)
__global__ void __launch_bounds__(WPB * 32) p2m_scaled_kernel(DevTree t, const float* __restrict__ xr,
                                                              const float* __restrict__ yr, const float* __restrict__ zr,
                                                              const float* __restrict__ qf, float inv_h, int N,
                                                              const float* __restrict__ knm, float2* __restrict__ outer)
{
	__shared__ float2 sacc[WPB][NX2MAX];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int LL = t.depth - 1;
	size_t leaf = (size_t)blockIdx.x * WPB + w;
	if (leaf >= t.lsize[LL]) return;
	size_t g = t.loff[LL] + leaf;
	const int Nx2 = N * (N + 1) / 2;
	for (int c = lane; c < Nx2; c += 32) sacc[w][c] = make_float2(0.f, 0.f);
	__syncwarp();
	const uint32_t b = t.beg[g], e = t.end[g];
	for (uint32_t base = b; base < e; base += 32) {
		uint32_t i = base + lane;
		float q = 0.f, r = 1.f, th = 1.f, ph = 0.f;
		if (i < e) { q = qf[i]; dec_to_sph<float>(xr[i] * inv_h, yr[i] * inv_h, zr[i] * inv_h, r, th, ph); }
		float y, x;
		sincosf(th, &y, &x);
		float Pmm = 1.f, rpow = 1.f;
		for (int m = 0; m < N; ++m) {
			if (m > 0) { Pmm = Pmm * y * (float)(1 - 2 * m); rpow *= r; }
			float sm_, cm_;
			sincosf(m * ph, &sm_, &cm_);
			float Pn = Pmm, Pn1 = 0.f, rn = rpow;
			for (int n = m; n < N; ++n) {
				if (n > m) {
					float Pnew = (n == m + 1) ? Pmm * x * (float)(2 * n - 1)
					                          : ((float)(2 * n - 1) * x * Pn - (float)(n + m - 1) * Pn1) / (float)(n - m);
					Pn1 = Pn; Pn = Pnew; rn *= r;
				}
				float vr, vi;
				if (n == 0) { vr = q; vi = 0.f; }
				else { float f = q * rn * knm[tix(n, m)] * Pn; vr = f * cm_; vi = -f * sm_; }
				vr = warp_sum(vr); vi = warp_sum(vi);
				if (lane == 0) { float2 a = sacc[w][tix(n, m)]; sacc[w][tix(n, m)] = make_float2(a.x + vr, a.y + vi); }
			}
		}
	}
	__syncwarp();
	float2* out = outer + leaf * Nx2;
	for (int c = lane; c < Nx2; c += 32) out[c] = sacc[w][c];
}

__global__ void d2f_kernel(const double* __restrict__ in, float* __restrict__ out, size_t n)
{
	size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (float)in[i];
}
__global__ void f2d_kernel(const float* __restrict__ in, double* __restrict__ out, size_t n)
{
	size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (double)in[i];
}

// Scaled local expansion at one target (FP32): the plain L2P formula at r/h;
// the caller multiplies the potential by 1/h and the field by 1/h^2.
__device__ void l2p_scaled(const float2* __restrict__ Lc, float dx, float dy, float dz, int N,
                           const float* __restrict__ knm, float& pot, float& fx, float& fy, float& fz)
{
	float r, th, ph;
	dec_to_sph<float>(dx, dy, dz, r, th, ph);
	float y, x;
	sincosf(th, &y, &x);
	float phi = 0.f, mt0 = 0.f, mt1 = 0.f, mt2 = 0.f;
	float Pmm = 1.f, rpow = 1.f / r;
	for (int m = 0; m < N; ++m) {
		if (m > 0) { Pmm = Pmm * y * (float)(1 - 2 * m); rpow *= r; }
		float sm_, cm_;
		sincosf(m * ph, &sm_, &cm_);
		const float mult = m ? 2.f : 1.f;
		float Pn = Pmm, Pn1 = 0.f, rn = rpow;
		for (int n = m; n < N; ++n) {
			float Pnext = (n == m) ? Pmm * x * (float)(2 * n + 1)
			                       : ((float)(2 * n + 1) * x * Pn - (float)(n + m) * Pn1) / (float)(n + 1 - m);
			float K = knm[tix(n, m)];
			float Yr = Pn * cm_ * K, Yi = Pn * sm_ * K;
			float2 Lnm = Lc[tix(n, m)];
			float cr = Lnm.x * rn, ci = Lnm.y * rn;
			float ycr = Yr * cr - Yi * ci;
			phi += mult * (r * ycr);
			float gq = K * ((float)(1 - m + n) * Pnext - (float)(n + 1) * x * Pn) / y;
			mt0 -= mult * ((float)n * ycr);
			mt1 -= mult * (cr * cm_ * gq - ci * sm_ * gq);
			mt2 -= mult * (cr * (-(float)m * Yi) - ci * ((float)m * Yr));
			Pn1 = Pn; Pn = Pnext; rn *= r;
		}
	}
	pot = phi;
	float s2, c2;
	sincosf(ph, &s2, &c2);
	fx = mt0 * y * c2 + mt1 * x * c2 - mt2 * s2 / y;
	fy = mt0 * y * s2 + mt1 * x * s2 + mt2 * c2 / y;
	fz = mt0 * x - mt1 * y;
}

constexpr int LTM = 128;

// Near field (FP32, leaf-relative) + far field (scaled FP32 L2P), block per
// leaf.  Source tiles are shifted into the target leaf's frame by the FP64
// centre difference rounded once; each tile's partial sums go into FP64
// accumulators; the self pair is skipped and q_i / 1e-4 added in FP64.
__global__ void __launch_bounds__(LTM) leaves_mixed_kernel(DevTree t, const float* __restrict__ xr,
                                                           const float* __restrict__ yr, const float* __restrict__ zr,
                                                           const float* __restrict__ qf, const float2* __restrict__ inner,
                                                           int N, float inv_h, const float* __restrict__ knm,
                                                           double* __restrict__ pot_out, double* __restrict__ fld_out)
{
	__shared__ float sx[LTM], sy[LTM], sz[LTM], sq[LTM];
	__shared__ float2 sL[NX2MAX];
	const int LL = t.depth - 1;
	size_t leaf = blockIdx.x;
	if (leaf >= t.lsize[LL]) return;
	size_t off = t.loff[LL], g = off + leaf;
	const bool tmode = t.targets_num > 0;
	const uint32_t tb = tmode ? t.tbeg[g] : t.beg[g];
	const uint32_t te = tmode ? t.tend[g] : t.end[g];
	if (tb >= te) return;
	const int Nx2 = N * (N + 1) / 2;
	for (int c = threadIdx.x; c < Nx2; c += LTM) sL[c] = inner[leaf * Nx2 + c];
	const int ncl = t.close_cnt[g];
	const int32_t* cl = t.close_idx + g * t.close_stride;
	const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
	for (uint32_t t0 = tb; t0 < te; t0 += LTM) {
		uint32_t i = t0 + threadIdx.x;
		const bool valid = i < te;
		float xi = 0.f, yi = 0.f, zi = 0.f;
		if (valid) { xi = xr[i]; yi = yr[i]; zi = zr[i]; }
		double pot = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
		for (int e = -1; e < ncl; ++e) {
			size_t sc = e < 0 ? g : off + cl[e];
			const float shx = (float)(t.cx[sc] - cx), shy = (float)(t.cy[sc] - cy), shz = (float)(t.cz[sc] - cz);
			const uint32_t sb = t.beg[sc], se = t.end[sc];
			for (uint32_t s0 = sb; s0 < se; s0 += LTM) {
				const int cnt = min((uint32_t)LTM, se - s0);
				__syncthreads();
				if (threadIdx.x < cnt) {
					uint32_t j = s0 + threadIdx.x;
					sx[threadIdx.x] = xr[j] + shx; sy[threadIdx.x] = yr[j] + shy; sz[threadIdx.x] = zr[j] + shz;
					sq[threadIdx.x] = qf[j];
				}
				__syncthreads();
				if (valid) {
					const int self = (e < 0) ? (int)i - (int)s0 : -1;   // skip the self pair
					float p = 0.f, ax = 0.f, ay = 0.f, az = 0.f;
					for (int j = 0; j < cnt; ++j) {
						float dx = xi - sx[j], dy = yi - sy[j], dz = zi - sz[j];
						float r2 = fmaxf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), (float)FORCE_EPS2);
						float inv = rsqrtf(r2);
						float qi = (j == self) ? 0.f : sq[j] * inv;
						float qi3 = qi * inv * inv;
						p += qi;
						ax = fmaf(dx, qi3, ax); ay = fmaf(dy, qi3, ay); az = fmaf(dz, qi3, az);
					}
					pot += p; fx += ax; fy += ay; fz += az;
				}
			}
		}
		__syncthreads();
		if (valid) {
			float lp, lx, ly, lz;
			l2p_scaled(sL, xi * inv_h, yi * inv_h, zi * inv_h, N, knm, lp, lx, ly, lz);
			const double ih = (double)inv_h;
			pot += (double)lp * ih;
			fx += (double)lx * ih * ih; fy += (double)ly * ih * ih; fz += (double)lz * ih * ih;
			if (!tmode) pot += t.q[i] * (1.0 / FORCE_EPS);
			uint32_t o = t.orig[i];
			pot_out[o] = pot;
			fld_out[3 * (size_t)o] = fx; fld_out[3 * (size_t)o + 1] = fy; fld_out[3 * (size_t)o + 2] = fz;
		}
	}
}

// child (level L, array chi) += scaled L2L from its parent (level L-1, array par)
template <typename real>
__global__ void __launch_bounds__(WPB * 32) l2l_scaled_kernel(DevTree t, int L, const typename V2<real>::t* __restrict__ par,
                                                              typename V2<real>::t* __restrict__ chi, int N,
                                                              Tab<real> T, unsigned* flags)
{
	__shared__ SmemT<real> sm[WPB];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t c = (size_t)blockIdx.x * WPB + w;
	if (c >= t.lsize[L]) return;
	const int Nx2 = N * (N + 1) / 2;
	size_t g = t.loff[L] + c;
	int32_t p = t.parent[g];
	typename V2<real>::t* out = chi + c * Nx2;
	typename V2<real>::t acc[CMAX];
#pragma unroll
	for (int k = 0; k < CMAX; ++k) {
		int cc = lane + 32 * k;
		acc[k] = cc < Nx2 ? out[cc] : V2<real>::make(0, 0);
	}
	uint64_t oct = t.code[g] & 7ull;
	int d = dir_id(1 - 2 * (int)((oct >> 2) & 1), 1 - 2 * (int)((oct >> 1) & 1), 1 - 2 * (int)(oct & 1));
	translate_scaled<SOP_L2L, real>(par + (size_t)p * Nx2, d, acc, N, Nx2, sm[w], T, flags);
#pragma unroll
	for (int k = 0; k < CMAX; ++k) {
		int cc = lane + 32 * k;
		if (cc < Nx2) out[cc] = acc[k];
	}
}

bool g_mixed_const_ready = false;

} // namespace

// FP32 copy of the level-independent (scaled) M2L operators, cached.
float* m2l_ops_fp32(Context& ctx, int N)
{
	for (auto& e : ctx.opcache)
		if (e.N == N && e.prec == 1) { e.stamp = ++ctx.opcache_clock; return static_cast<float*>(e.ptr); }
	double* d = m2l_ops_fp64(ctx, N, 1.0);
	if (!d) return nullptr;
	const int MT = m2l_padded(N);
	size_t n = (size_t)343 * MT * MT;
	OpCacheEntry e;
	e.N = N; e.prec = 1; e.h = 1.0; e.bytes = n * sizeof(float); e.stamp = ++ctx.opcache_clock;
	if (cudaMalloc(&e.ptr, e.bytes) != cudaSuccess) { cudaGetLastError(); ctx.last_error = "m2l operators: out of memory"; return nullptr; }
	d2f_kernel<<<div_up(n, 256), 256, 0, ctx.stream>>>(d, static_cast<float*>(e.ptr), n);
	ctx.opcache.push_back(e);
	return static_cast<float*>(e.ptr);
}

int fmm3d_solve_mixed(Context& ctx, const ParticleInput& in, int N, int depth, double* pot, double* field,
                      SolveStats* stats)
{
	if (N < 1 || N > MAXN3) { ctx.last_error = "order out of range (1 <= N <= 18)"; return ERR_ARG; }
	if (!m2l_gemm_supported(N)) { ctx.last_error = "mixed form supports N <= 13"; return ERR_UNSUPPORTED; }
	if (!g_mixed_const_ready) {
		unsigned char n_of[NX2MAX], m_of[NX2MAX];
		for (int n = 0; n < MAXN3; ++n)
			for (int m = 0; m <= n; ++m) { n_of[tix(n, m)] = (unsigned char)n; m_of[tix(n, m)] = (unsigned char)m; }
		LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_n_of, n_of, sizeof(n_of)));
		LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_m_of, m_of, sizeof(m_of)));
		g_mixed_const_ready = true;
	}
	cudaStream_t s = ctx.stream;
	const bool timing = ctx.timing != 0;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[0], s));
	DevTree t;
	int st = tree_build(ctx, in, depth, t);
	if (st) return st;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[1], s));
	const int LL = depth - 1;
	const int B = LL < FP64_LEVELS ? LL : FP64_LEVELS;     // levels < B in FP64, >= B in FP32 (leaves FP32)
	const int Nx2 = N * (N + 1) / 2;
	const double scale = t.geo_host[3];
	const DevTables& TD = ctx.tables.d;
	Tab<double> Td{TD.dmat, TD.emat, TD.m2m, TD.l2l, TD.knm, TD.dirinfo};
	Tab<float> Tf{TD.dmat_f, TD.emat_f, TD.m2m_f, TD.l2l_f, TD.knm_f, TD.dirinfo};
	// expansion storage: FP64 for levels < B, FP32 for levels >= B (level-local pointers)
	size_t cd = B > 0 ? t.loff[B] : 0, cf = t.ncells - cd;
	double2* od = static_cast<double2*>(ctx.arena.take(sizeof(double2) * (cd + 1) * Nx2));
	double2* id = static_cast<double2*>(ctx.arena.take(sizeof(double2) * (cd + 1) * Nx2));
	float2* of = static_cast<float2*>(ctx.arena.take(sizeof(float2) * cf * Nx2));
	float2* if_ = static_cast<float2*>(ctx.arena.take(sizeof(float2) * cf * Nx2));
	const size_t n = t.n;
	float* xr = static_cast<float*>(ctx.arena.take(sizeof(float) * n));
	float* yr = static_cast<float*>(ctx.arena.take(sizeof(float) * n));
	float* zr = static_cast<float*>(ctx.arena.take(sizeof(float) * n));
	float* qf = static_cast<float*>(ctx.arena.take(sizeof(float) * n));
	size_t bmax = 0;
	for (int L = 0; L < depth; ++L) bmax = std::max(bmax, t.lsize[L]);
	void* conv = ctx.arena.take(sizeof(double2) * bmax * Nx2);
	unsigned long long* counters = static_cast<unsigned long long*>(ctx.arena.take(32));
	if (!od || !id || !of || !if_ || !xr || !qf || !conv || !counters) { ctx.last_error = "mixed: allocation failed"; return ERR_OOM; }
	auto OD = [&](int L) { return od + t.loff[L] * Nx2; };
	auto ID = [&](int L) { return id + t.loff[L] * Nx2; };
	auto OF = [&](int L) { return of + (t.loff[L] - cd) * Nx2; };
	auto IF = [&](int L) { return if_ + (t.loff[L] - cd) * Nx2; };
	auto h_of = [&](int L) { return scale / (double)(1ull << L); };
	const size_t n_out = in.nt ? in.nt : in.ns;
	LFMM_CUDA(ctx, cudaMemsetAsync(pot, 0, sizeof(double) * n_out, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(field, 0, sizeof(double) * 3 * n_out, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(id, 0, sizeof(double2) * (cd + 1) * Nx2, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(if_, 0, sizeof(float2) * cf * Nx2, s));
	relcoords_kernel<<<(unsigned)t.lsize[LL], 128, 0, s>>>(t, xr, yr, zr, qf);
	// upward
	p2m_scaled_kernel<<<div_up(t.lsize[LL], WPB), WPB * 32, 0, s>>>(t, xr, yr, zr, qf, (float)(1.0 / h_of(LL)), N,
	                                                                TD.knm_f, OF(LL));
	for (int L = LL - 1; L >= 0; --L) {
		unsigned grid = div_up(t.lsize[L], WPB);
		if (L >= B) {
			m2m_scaled_kernel<float><<<grid, WPB * 32, 0, s>>>(t, L, OF(L + 1), OF(L), N, Tf, ctx.dev_flags);
		} else if (L + 1 >= B) {
			size_t m = t.lsize[L + 1] * Nx2 * 2;
			f2d_kernel<<<div_up(m, 256), 256, 0, s>>>(reinterpret_cast<const float*>(OF(L + 1)), static_cast<double*>(conv), m);
			m2m_scaled_kernel<double><<<grid, WPB * 32, 0, s>>>(t, L, static_cast<double2*>(conv), OD(L), N, Td, ctx.dev_flags);
		} else {
			m2m_scaled_kernel<double><<<grid, WPB * 32, 0, s>>>(t, L, OD(L + 1), OD(L), N, Td, ctx.dev_flags);
		}
	}
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[2], s));
	// M2L: level-independent operators (FP64 on levels < B, FP32 below)
	if (depth > 2) {
		double* opd = m2l_ops_fp64(ctx, N, 1.0);
		float* opf = m2l_ops_fp32(ctx, N);
		if (!opd || !opf) return ERR_OOM;
		for (int L = 2; L <= LL; ++L) {
			M2LPlan plan;
			if ((st = m2l_plan_build(ctx, t, L, plan))) return st;
			if (L < B) st = m2l_gemm<double>(ctx, plan, opd, reinterpret_cast<const double*>(OD(L)), reinterpret_cast<double*>(ID(L)), N);
			else st = m2l_gemm<float>(ctx, plan, opf, reinterpret_cast<const float*>(OF(L)), reinterpret_cast<float*>(IF(L)), N);
			if (st) return st;
		}
	}
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[3], s));
	for (int L = 3; L <= LL; ++L) {
		unsigned grid = div_up(t.lsize[L], WPB);
		if (L < B) {
			l2l_scaled_kernel<double><<<grid, WPB * 32, 0, s>>>(t, L, ID(L - 1), ID(L), N, Td, ctx.dev_flags);
		} else if (L - 1 < B) {
			size_t m = t.lsize[L - 1] * Nx2 * 2;
			d2f_kernel<<<div_up(m, 256), 256, 0, s>>>(reinterpret_cast<const double*>(ID(L - 1)), static_cast<float*>(conv), m);
			l2l_scaled_kernel<float><<<grid, WPB * 32, 0, s>>>(t, L, static_cast<float2*>(conv), IF(L), N, Tf, ctx.dev_flags);
		} else {
			l2l_scaled_kernel<float><<<grid, WPB * 32, 0, s>>>(t, L, IF(L - 1), IF(L), N, Tf, ctx.dev_flags);
		}
	}
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[4], s));
	leaves_mixed_kernel<<<(unsigned)t.lsize[LL], LTM, 0, s>>>(t, xr, yr, zr, qf, IF(LL), N, (float)(1.0 / h_of(LL)),
	                                                          TD.knm_f, pot, field);
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
	return OK;
}

} // namespace lfmm
