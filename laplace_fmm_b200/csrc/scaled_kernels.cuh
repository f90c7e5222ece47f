// Device kernels of the scaled-expansion 3D solver (plain FP64 or mixed
// FP32), included only by fmm3d_scaled.cu.  Scaled expansions: multipole
// a_nm / h^n and local L_nm h^(n+1) for a cell of size h; every operator is
// then level-independent and every coefficient O(total charge):
//   M2L   rho / h = |d|                      (one operator per far offset d)
//   M2M   (rho / h_child)^n, row j times 2^-j
//   L2L   (rho / h_parent)^(n-j), row j times 2^-(j+1)
//   P2M / L2P / P2L / M2P with r / h; potential times 1/h, field times 1/h^2.
#pragma once
#include "fmm3d.cuh"
#include "m2l_gemm.cuh"

namespace lfmm {
namespace scaled {

constexpr int CMAX = (MAXN3 * (MAXN3 + 1) / 2 + 31) / 32;
constexpr int NX2MAX = MAXN3 * (MAXN3 + 1) / 2;
constexpr int WPB = 4;

template <typename real> struct V2;
template <> struct V2<double> { using t = double2; static __device__ __forceinline__ double2 make(double a, double b) { return make_double2(a, b); } };
template <> struct V2<float> { using t = float2; static __device__ __forceinline__ float2 make(float a, float b) { return make_float2(a, b); } };

constexpr int NXD = (MAXN3 + 1) * (MAXN3 + 2) / 2;   // coefficients of degree <= MAXN3
// Solid harmonics in Cartesian form, orthonormal basis B_nm = r^n Y_nm
// (regular) and r^-(n+1) Y_nm (irregular), Y_nm = sqrt((n-m)!/(n+m)!)
// P_n^m(cos t) e^{i m phi} with the Condon-Shortley phase:
//   B_00 = 1 (or 1/r), B_mm = s_m w B_{m-1,m-1}, w = x + iy (or w / r^2),
//   s_m = -sqrt((2m - 1) / (2m)),
//   B_{n+1,m} = a_nm z B_nm - b_nm r^2 B_{n-1,m}   (or (a z B_nm - b B_{n-1,m}) / r^2)
// with (a_nm, b_nm) = ((2n + 1) / sqrt((n+1)^2 - m^2), sqrt((n^2 - m^2) / ((n+1)^2 - m^2)))
// stored at tix(n, m).
__constant__ float2 c_rec_f[NXD];
__constant__ double2 c_rec_d[NXD];
__constant__ float c_sig_f[MAXN3 + 2];
__constant__ double c_sig_d[MAXN3 + 2];
template <typename real> __device__ __forceinline__ typename V2<real>::t rec_c(int i);
template <> __device__ __forceinline__ float2 rec_c<float>(int i) { return c_rec_f[i]; }
template <> __device__ __forceinline__ double2 rec_c<double>(int i) { return c_rec_d[i]; }
template <typename real> __device__ __forceinline__ real sig_c(int m);
template <> __device__ __forceinline__ float sig_c<float>(int m) { return c_sig_f[m]; }
template <> __device__ __forceinline__ double sig_c<double>(int m) { return c_sig_d[m]; }
constexpr int NINV = 64;
__constant__ float c_inv_f[NINV];      // 1 / k (k >= 1), rounded to FP32
__constant__ double c_inv_d[NINV];     // 1 / k, FP64
template <typename real> __device__ __forceinline__ real inv_of(int k);
template <> __device__ __forceinline__ float inv_of<float>(int k) { return c_inv_f[k]; }
template <> __device__ __forceinline__ double inv_of<double>(int k) { return c_inv_d[k]; }


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
			const int n = tri_row(c), m = c - tix(n, 0);
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
		if (c < Nx2) sm.a[c] = cmulv<real>(src[c], E1[c - tix(tri_row(c), 0)]);
	}
	__syncwarp();
	rotate_y_t<real>(sm.a, sm.b, D1, Nx2);
	__syncwarp();
	const real* cube = OP == SOP_M2M ? T.m2m : T.l2l;
#pragma unroll
	for (int t = 0; t < CMAX; ++t) {
		int c = lane + 32 * t;
		if (c < Nx2) {
			const int j = tri_row(c), k = c - tix(j, 0);
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
			typename V2<real>::t v = cmulv<real>(sm.b[c], E2[c - tix(tri_row(c), 0)]);
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
	if (t.beg[g] >= t.end[g]) return;     // a leaf keeps its P2M expansion
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

template <typename real> __device__ __forceinline__ real rsq(real x);
template <> __device__ __forceinline__ float rsq<float>(float x) { return rsqrtf(x); }
template <> __device__ __forceinline__ double rsq<double>(double x) { return rsqrt(x); }
template <typename real> __device__ __forceinline__ void sc(real a, real* s, real* c);
template <> __device__ __forceinline__ void sc<float>(float a, float* s, float* c) { sincosf(a, s, c); }
template <> __device__ __forceinline__ void sc<double>(double a, double* s, double* c) { sincos(a, s, c); }

// Leaf-relative coordinates (real) and charges, block per leaf.
template <typename real>
__global__ void relcoords_kernel(DevTree t, real* __restrict__ xr, real* __restrict__ yr, real* __restrict__ zr,
                                 real* __restrict__ qr)
{
	if (blockIdx.x >= t.nleaves) return;
	size_t g = t.leaves[blockIdx.x];
	const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
	for (uint32_t i = t.pbeg[g] + threadIdx.x; i < t.pend[g]; i += blockDim.x) {
		xr[i] = (real)(t.x[i] - cx); yr[i] = (real)(t.y[i] - cy); zr[i] = (real)(t.z[i] - cz);
		qr[i] = (real)t.q[i];
	}
}

// Regular (P2M) or singular (P2L) harmonics of the warp's particles summed
// into sacc: regular  q (r/h)^n K P_nm e^{-i m phi}
//            singular q (r/h)^-(n+1) K P_nm e^{-i m phi}
template <bool SINGULAR, typename real>
__device__ __forceinline__ void accumulate_harmonics(real q, real r, real th, real ph, int N, const real* __restrict__ knm,
                                                     typename V2<real>::t* sacc)
{
	const int lane = threadIdx.x & 31;
	real y, x;
	sc<real>(th, &y, &x);
	const real ir = real(1) / r;
	real Pmm = 1, rpow = SINGULAR ? ir : real(1);
	for (int m = 0; m < N; ++m) {
		if (m > 0) { Pmm = Pmm * y * (real)(1 - 2 * m); rpow *= SINGULAR ? ir : r; }
		real sm_, cm_;
		sc<real>(m * ph, &sm_, &cm_);
		real Pn = Pmm, Pn1 = 0, rn = rpow;
		for (int n = m; n < N; ++n) {
			if (n > m) {
				real Pnew = (n == m + 1) ? Pmm * x * (real)(2 * n - 1)
				                         : ((real)(2 * n - 1) * x * Pn - (real)(n + m - 1) * Pn1) / (real)(n - m);
				Pn1 = Pn; Pn = Pnew; rn *= SINGULAR ? ir : r;
			}
			real f = q * rn * knm[tix(n, m)] * Pn;
			real vr = warp_sum(f * cm_), vi = warp_sum(-f * sm_);
			if (lane == 0) { typename V2<real>::t a = sacc[tix(n, m)]; sacc[tix(n, m)] = V2<real>::make(a.x + vr, a.y + vi); }
		}
	}
}

// One warp's particles (lane = particle, q = 0 for none) summed into the
// coefficients q conj(B_nm) (regular: P2M; irregular: P2L) through the
// Cartesian recurrences of eval_cart: for each order m the lanes write their
// N - m values to a row of buf (stride 2 MAXN3 + 1, odd: conflict-free
// columns), then lane c adds up column c (in FP64 for orders 0 and 1, else
// in a tree of FP32 partial sums).
constexpr int ACC_LD = 2 * MAXN3 + 1;

template <bool IRR, typename real>
__device__ __forceinline__ void accumulate_cart(real q, real x, real y, real z, int N, typename V2<real>::t* sacc,
                                                real* buf, int lane)
{
	using v2 = typename V2<real>::t;
	const real r2 = x * x + y * y + z * z;
	const real ir2 = IRR ? real(1) / r2 : real(0);
	const real wx = IRR ? x * ir2 : x, wy = IRR ? y * ir2 : y;
	real bx = IRR ? rsq<real>(r2) : real(1), by = 0;
	real* row = buf + lane * ACC_LD;
	for (int m = 0; m < N; ++m) {
		if (m > 0) {
			const real sgm = sig_c<real>(m);
			const real nx = sgm * (wx * bx - wy * by), ny = sgm * (wx * by + wy * bx);
			bx = nx; by = ny;
		}
		real px = 0, py = 0, cx = bx, cy = by;
		int i = tix(m, m);
		for (int n = m; n < N; ++n) {
			row[2 * (n - m)] = q * cx;
			row[2 * (n - m) + 1] = -q * cy;
			const v2 ab = rec_c<real>(i);
			const real az = ab.x * z, bb = IRR ? ab.y : ab.y * r2;
			real nx = fma(az, cx, -bb * px), ny = fma(az, cy, -bb * py);
			if (IRR) { nx *= ir2; ny *= ir2; }
			px = cx; py = cy; cx = nx; cy = ny;
			i += n + 1;
		}
		__syncwarp();
		if (lane < 2 * (N - m)) {
			real* a = reinterpret_cast<real*>(sacc + tix(m + (lane >> 1), m)) + (lane & 1);
			if (m < 2) {
				// orders 0 and 1 in FP64: the leaves' monopole and dipole rounding
				// errors add up over the whole far field
				double sum = 0.0;
#pragma unroll 8
				for (int r = 0; r < 32; ++r) sum += (double)buf[r * ACC_LD + lane];
				*a += (real)sum;
			} else {
				// eight interleaved partial sums, then a tree
				real p[8];
#pragma unroll
				for (int k = 0; k < 8; ++k) p[k] = buf[k * ACC_LD + lane];
#pragma unroll
				for (int r = 8; r < 32; r += 8)
#pragma unroll
					for (int k = 0; k < 8; ++k) p[k] += buf[(r + k) * ACC_LD + lane];
				*a += ((p[0] + p[1]) + (p[2] + p[3])) + ((p[4] + p[5]) + (p[6] + p[7]));
			}
		}
		__syncwarp();
	}
}

// P2M, warp per leaf, in the leaf's scaled frame
template <typename real>
__global__ void __launch_bounds__(WPB * 32) p2m_scaled_kernel(DevTree t, const real* __restrict__ xr, const real* __restrict__ yr,
                                                              const real* __restrict__ zr, const real* __restrict__ qr,
                                                              int N, const real* __restrict__ knm,
                                                              typename V2<real>::t* __restrict__ outer)
{
	__shared__ typename V2<real>::t sacc[WPB][NX2MAX];
	__shared__ real sbuf[WPB][32 * ACC_LD];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t li = (size_t)blockIdx.x * WPB + w;
	if (li >= t.nleaves) return;
	const size_t g = t.leaves[li];
	const int Nx2 = N * (N + 1) / 2;
	for (int c = lane; c < Nx2; c += 32) sacc[w][c] = V2<real>::make(0, 0);
	__syncwarp();
	const real ih = (real)(1.0 / cell_size(t, g));
	const uint32_t b = t.pbeg[g], e = t.send[g];
	for (uint32_t base = b; base < e; base += 32) {
		uint32_t i = base + lane;
		real q = 0, x = 0, y = 0, z = 0;
		if (i < e) { q = qr[i]; x = xr[i] * ih; y = yr[i] * ih; z = zr[i] * ih; }
		accumulate_cart<false, real>(q, x, y, z, N, sacc[w], sbuf[w], lane);
	}
	__syncwarp();
	typename V2<real>::t* out = outer + g * Nx2;
	for (int c = lane; c < Nx2; c += 32) out[c] = sacc[w][c];
}

// P2L over the X list, warp per cell: inner[g] += singular harmonics of every
// X leaf's sources about g's centre (scaled by g's size).
template <typename real>
__global__ void __launch_bounds__(WPB * 32) p2l_kernel(DevTree t, int N, const real* __restrict__ knm,
                                                       typename V2<real>::t* __restrict__ inner)
{
	__shared__ typename V2<real>::t sacc[WPB][NX2MAX];
	__shared__ real sbuf[WPB][32 * ACC_LD];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	size_t g = (size_t)blockIdx.x * WPB + w;
	if (g >= t.ncells) return;
	const uint32_t xb = t.x_off[g], xe = t.x_off[g + 1];
	if (xb == xe) return;
	const int Nx2 = N * (N + 1) / 2;
	for (int c = lane; c < Nx2; c += 32) sacc[w][c] = V2<real>::make(0, 0);
	__syncwarp();
	const double ih = 1.0 / cell_size(t, g);
	const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
	for (uint32_t e = xb; e < xe; ++e) {
		const int32_t C = t.x_idx[e];
		const uint32_t b = t.pbeg[C], en = t.send[C];
		for (uint32_t base = b; base < en; base += 32) {
			uint32_t i = base + lane;
			real q = 0, x = 0, y = 0, z = 1;              // an empty lane: q = 0 at a finite point
			if (i < en) {
				q = (real)t.q[i];
				x = (real)((t.x[i] - cx) * ih); y = (real)((t.y[i] - cy) * ih); z = (real)((t.z[i] - cz) * ih);
			}
			accumulate_cart<true, real>(q, x, y, z, N, sacc[w], sbuf[w], lane);
		}
	}
	__syncwarp();
	typename V2<real>::t* out = inner + g * Nx2;
	for (int c = lane; c < Nx2; c += 32) {
		typename V2<real>::t a = out[c], b = sacc[w][c];
		out[c] = V2<real>::make(a.x + b.x, a.y + b.y);
	}
}

// Expansion evaluated at one target, in the expansion's scaled frame:
// LOCAL  phi = sum (2 - d_m0) Re(r^n Y_nm L_nm)      (reference L2P form,
//        cpu/multipole3d.cpp:1152-1208)
// MULTI  phi = sum (2 - d_m0) Re(r^-(n+1) Y_nm a_nm)  (M2P)
// with Y_nm = K_nm P_nm e^{i m phi}; returns phi and -grad phi.
template <bool LOCAL, typename real>
__device__ void eval_expansion(const typename V2<real>::t* __restrict__ Lc, real dx, real dy, real dz, int N,
                               const real* __restrict__ knm, real& pot, real& fx, real& fy, real& fz)
{
	real r, th, ph;
	dec_to_sph<real>(dx, dy, dz, r, th, ph);
	real y, x;
	sc<real>(th, &y, &x);
	const real ir = real(1) / r, iy = real(1) / y;
	real phi = 0, mt0 = 0, mt1 = 0, mt2 = 0;
	real s1, c1;
	sc<real>(ph, &s1, &c1);
	real cm_ = 1, sm_ = 0;           // cos(m phi), sin(m phi) by the angle-addition recurrence
	// LOCAL: rn = r^(n-1) ; MULTI: rn = r^-(n+2)
	real Pmm = 1, rpow = LOCAL ? ir : ir * ir;
	for (int m = 0; m < N; ++m) {
		if (m > 0) {
			Pmm = Pmm * y * (real)(1 - 2 * m);
			rpow *= LOCAL ? r : ir;
			const real cn = cm_ * c1 - sm_ * s1;
			sm_ = sm_ * c1 + cm_ * s1;
			cm_ = cn;
		}
		const real mult = m ? real(2) : real(1);
		real Pn = Pmm, Pn1 = 0, rn = rpow;
		for (int n = m; n < N; ++n) {
			real Pnext = (n == m) ? Pmm * x * (real)(2 * n + 1)
			                      : ((real)(2 * n + 1) * x * Pn - (real)(n + m) * Pn1) * inv_of<real>(n + 1 - m);
			real K = knm[tix(n, m)];
			real Yr = Pn * cm_ * K, Yi = Pn * sm_ * K;
			typename V2<real>::t A = Lc[tix(n, m)];
			real cr = A.x * rn, ci = A.y * rn;
			real ycr = Yr * cr - Yi * ci;                 // Re(Y A) r^(n-1) or r^-(n+2)
			real gq = K * ((real)(1 - m + n) * Pnext - (real)(n + 1) * x * Pn) * iy;
			if (LOCAL) {
				phi += mult * (r * ycr);
				mt0 -= mult * ((real)n * ycr);
			} else {
				phi += mult * (r * ycr);
				mt0 += mult * ((real)(n + 1) * ycr);
			}
			mt1 -= mult * (cr * cm_ * gq - ci * sm_ * gq);
			mt2 -= mult * (cr * (-(real)m * Yi) - ci * ((real)m * Yr));
			Pn1 = Pn; Pn = Pnext; rn *= LOCAL ? r : ir;
		}
	}
	pot = phi;
	const real s2 = s1, c2 = c1;
	fx = mt0 * y * c2 + mt1 * x * c2 - mt2 * s2 * iy;
	fy = mt0 * y * s2 + mt1 * x * s2 + mt2 * c2 * iy;
	fz = mt0 * x - mt1 * y;
}

template <typename real>
__global__ void convert_kernel(const real* __restrict__ in, double* __restrict__ out, size_t n)
{
	size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (double)in[i];
}
template <typename real>
__global__ void convert_back_kernel(const double* __restrict__ in, real* __restrict__ out, size_t n)
{
	size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (real)in[i];
}

// warps (leaves) per block of the leaf kernel (static shared memory <= 48 KB)
template <typename real> constexpr int leaf_warps() { return sizeof(real) == sizeof(float) ? 8 : 4; }

// Near and local field of every target particle: one warp per leaf, lane =
// target (chunks of 32).  P2P over the leaf itself and its U list, sources
// staged 32 at a time in the warp's shared memory as offsets in the target
// leaf's frame split hi + lo (FP32 pairs keep ~1e-7 relative accuracy
// however close the pair; lo unused in FP64), partial sums over 8 sources
// carried in FP64; M2P over the W list; L2P of the leaf's local expansion;
// self term in FP64; outputs written in input order.
template <typename real, int LW = leaf_warps<real>()>
__global__ void __launch_bounds__(LW * 32) leaves_scaled_kernel(DevTree t, const real* __restrict__ qr,
                                                               const typename V2<real>::t* __restrict__ outer,
                                                               const typename V2<real>::t* __restrict__ inner, int N,
                                                               const real* __restrict__ knm, double* __restrict__ pot_out,
                                                               double* __restrict__ fld_out)
{
	using v2 = typename V2<real>::t;
	constexpr bool SPLIT = sizeof(real) == sizeof(float);
	__shared__ real sx[LW][32], sy[LW][32], sz[LW][32], sq[LW][32];
	__shared__ real lx[LW][32], ly[LW][32], lz[LW][32];
	__shared__ v2 sL[LW][NX2MAX], sM[LW][NX2MAX];
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const size_t li = (size_t)blockIdx.x * LW + w;
	if (li >= t.nleaves) return;
	const size_t g = t.leaves[li];
	const uint32_t tb = t.tbeg[g], te = t.tend[g];
	if (tb >= te) return;
	const bool tmode = t.targets_num > 0;
	const int Nx2 = N * (N + 1) / 2;
	const double ihg = 1.0 / cell_size(t, g);
	for (int c = lane; c < Nx2; c += 32) sL[w][c] = inner[g * Nx2 + c];
	const uint32_t ub = t.u_off[li], ue = t.u_off[li + 1];
	const uint32_t wb = t.w_off[li], we = t.w_off[li + 1];
	const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
	__syncwarp();
	for (uint32_t t0 = tb; t0 < te; t0 += 32) {
		const uint32_t i = t0 + lane;
		const bool valid = i < te;
		real xi = 0, yi = 0, zi = 0, xl = 0, yl = 0, zl = 0;
		if (valid) {
			const double ax_ = t.x[i] - cx, ay_ = t.y[i] - cy, az_ = t.z[i] - cz;
			xi = (real)ax_; yi = (real)ay_; zi = (real)az_;
			if (SPLIT) { xl = (real)(ax_ - (double)xi); yl = (real)(ay_ - (double)yi); zl = (real)(az_ - (double)zi); }
		}
		double pot = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
		for (int64_t e = (int64_t)ub - 1; e < (int64_t)ue; ++e) {
			const size_t sc_ = e < (int64_t)ub ? g : (size_t)t.u_idx[e];
			const uint32_t sb = t.pbeg[sc_], se = t.send[sc_];
			for (uint32_t s0 = sb; s0 < se; s0 += 32) {
				const int cnt = min(32u, se - s0);
				__syncwarp();
				if (lane < cnt) {
					const uint32_t j = s0 + lane;
					const double dx_ = t.x[j] - cx, dy_ = t.y[j] - cy, dz_ = t.z[j] - cz;
					const real hx = (real)dx_, hy = (real)dy_, hz = (real)dz_;
					sx[w][lane] = hx; sy[w][lane] = hy; sz[w][lane] = hz;
					if (SPLIT) {
						lx[w][lane] = (real)(dx_ - (double)hx); ly[w][lane] = (real)(dy_ - (double)hy);
						lz[w][lane] = (real)(dz_ - (double)hz);
					}
					sq[w][lane] = qr[j];
				}
				__syncwarp();
				if (valid) {
					const int self = (sc_ == g) ? (int)i - (int)s0 : -1;
					for (int j0 = 0; j0 < cnt; j0 += 8) {
						const int j1 = min(cnt, j0 + 8);
						real p = 0, ax = 0, ay = 0, az = 0;
						for (int j = j0; j < j1; ++j) {
							real dx = xi - sx[w][j], dy = yi - sy[w][j], dz = zi - sz[w][j];
							if (SPLIT) { dx += xl - lx[w][j]; dy += yl - ly[w][j]; dz += zl - lz[w][j]; }
							const real r2 = fmax(fma(dx, dx, fma(dy, dy, dz * dz)), (real)FORCE_EPS2);
							const real inv = rsq<real>(r2);
							const real qi = (j == self) ? real(0) : sq[w][j] * inv;
							const real qi3 = qi * inv * inv;
							p += qi;
							ax = fma(dx, qi3, ax); ay = fma(dy, qi3, ay); az = fma(dz, qi3, az);
						}
						pot += p; fx += ax; fy += ay; fz += az;
					}
				}
			}
		}
		// M2P over the W list
		for (uint32_t e = wb; e < we; ++e) {
			const size_t D = t.w_idx[e];
			__syncwarp();
			for (int c = lane; c < Nx2; c += 32) sM[w][c] = outer[D * Nx2 + c];
			__syncwarp();
			if (valid) {
				const double ihd = 1.0 / cell_size(t, D);
				real mp, mx_, my_, mz_;
				eval_expansion<false, real>(sM[w], (real)((t.x[i] - t.cx[D]) * ihd), (real)((t.y[i] - t.cy[D]) * ihd),
				                            (real)((t.z[i] - t.cz[D]) * ihd), N, knm, mp, mx_, my_, mz_);
				pot += (double)mp * ihd;
				fx += (double)mx_ * ihd * ihd; fy += (double)my_ * ihd * ihd; fz += (double)mz_ * ihd * ihd;
			}
		}
		if (valid) {
			real lp, lx_, ly_, lz_;
			eval_expansion<true, real>(sL[w], (real)(xi * ihg), (real)(yi * ihg), (real)(zi * ihg), N, knm, lp, lx_, ly_,
			                           lz_);
			pot += (double)lp * ihg;
			fx += (double)lx_ * ihg * ihg; fy += (double)ly_ * ihg * ihg; fz += (double)lz_ * ihg * ihg;
			if (!tmode) pot += t.q[i] * (1.0 / FORCE_EPS);
			const uint32_t o = t.orig[i];
			pot_out[o] = pot;
			fld_out[3 * (size_t)o] = fx; fld_out[3 * (size_t)o + 1] = fy; fld_out[3 * (size_t)o + 2] = fz;
		}
	}
}

// Expansion evaluation through Cartesian solid harmonics.  A real field
// phi = sum_{n, m >= 0} (2 - d_m0) Re(E_nm B_nm) (E stored for m >= 0; the
// m < 0 coefficients are (-1)^m conj(E_n|m|)) has, with the derivative rules
//   regular:   d_z B_nm = sqrt((n-m)(n+m)) B_{n-1,m},
//              (d_x + i d_y) B_nm = sqrt((n-m)(n-m-1)) B_{n-1,m+1},
//              (d_x - i d_y) B_nm = -sqrt((n+m)(n+m-1)) B_{n-1,m-1},
//   irregular: d_z B_nm = -sqrt((n+1-m)(n+1+m)) B_{n+1,m},
//              (d_x + i d_y) B_nm = sqrt((n+m+1)(n+m+2)) B_{n+1,m+1},
//              (d_x - i d_y) B_nm = -sqrt((n-m+1)(n-m+2)) B_{n+1,m-1},
// a gradient that is again a real field in the same basis, of degree one
// less (local) or one more (multipole).  derive_coefs turns E into the
// potential's and the three gradient components' coefficients, the weight
// (2 - d_m0) folded in; eval_cart streams one target's harmonics through the
// recurrences and takes the four dot products.
template <typename real>
__device__ __forceinline__ typename V2<real>::t coef_full(const typename V2<real>::t* __restrict__ E, int N, int n, int m)
{
	using v2 = typename V2<real>::t;
	if (n < 0 || n >= N || m > n || -m > n) return V2<real>::make(0, 0);
	if (m == 0) return V2<real>::make(E[tix(n, 0)].x, 0);
	if (m > 0) return E[tix(n, m)];
	const v2 e = E[tix(n, -m)];
	return (m & 1) ? V2<real>::make(-e.x, e.y) : V2<real>::make(e.x, -e.y);
}

// The four coefficient sets of one (n, m): potential, d/dx, d/dy, d/dz.
template <typename real> struct Coef4 {
	typename V2<real>::t f, gx, gy, gz;
};
// FP32 form as stored for eval_cart: the real parts of the four sets, then
// their negated imaginary parts, so one float4 load feeds two packed FMAs.
struct CoefP {
	float4 re, im;
};
template <typename real> struct CoefStore { using t = Coef4<real>; };
template <> struct CoefStore<float> { using t = CoefP; };
__device__ __forceinline__ void put_coef(Coef4<double>* C, int e, const Coef4<double>& o) { C[e] = o; }
__device__ __forceinline__ void put_coef(CoefP* C, int e, const Coef4<float>& o)
{
	C[e].re = make_float4(o.f.x, o.gx.x, o.gy.x, o.gz.x);
	C[e].im = make_float4(-o.f.y, -o.gx.y, -o.gy.y, -o.gz.y);
}

template <bool IRR, typename real>
__device__ void derive_coefs(const typename V2<real>::t* __restrict__ E, int N, typename CoefStore<real>::t* C,
                             int lane)
{
	using v2 = typename V2<real>::t;
	const int NB = IRR ? N + 1 : N, NG = IRR ? N + 1 : N - 1;
	for (int e = lane; e < NB * (NB + 1) / 2; e += 32) {
		const int n = tri_row(e), k = e - tix(n, 0);
		Coef4<real> o;
		if (n < N) {
			const v2 c = E[e];
			o.f = k ? V2<real>::make(2 * c.x, 2 * c.y) : V2<real>::make(c.x, 0);
		} else {
			o.f = V2<real>::make(0, 0);
		}
		if (n < NG) {
			v2 Z, P, M;
			if (!IRR) {
				const v2 c0 = coef_full<real>(E, N, n + 1, k), cm = coef_full<real>(E, N, n + 1, k - 1);
				const v2 cp = coef_full<real>(E, N, n + 1, k + 1);
				const real fz = sqrt((real)((n + 1 - k) * (n + 1 + k))), fp = sqrt((real)((n + 2 - k) * (n + 1 - k)));
				const real fm = sqrt((real)((n + 2 + k) * (n + 1 + k)));
				Z = V2<real>::make(c0.x * fz, c0.y * fz);
				P = V2<real>::make(cm.x * fp, cm.y * fp);
				M = V2<real>::make(-cp.x * fm, -cp.y * fm);
			} else {
				const v2 c0 = coef_full<real>(E, N, n - 1, k), cm = coef_full<real>(E, N, n - 1, k - 1);
				const v2 cp = coef_full<real>(E, N, n - 1, k + 1);
				const real fz = sqrt((real)max((n - k) * (n + k), 0)), fp = sqrt((real)max((n + k - 1) * (n + k), 0));
				const real fm = sqrt((real)max((n - k - 1) * (n - k), 0));
				Z = V2<real>::make(-c0.x * fz, -c0.y * fz);
				P = V2<real>::make(cm.x * fp, cm.y * fp);
				M = V2<real>::make(-cp.x * fm, -cp.y * fm);
			}
			// d_x = (P + M) / 2, d_y = (P - M) / 2i; weight 2 for k > 0
			const real w = k ? real(1) : real(0.5);
			o.gx = V2<real>::make(w * (P.x + M.x), w * (P.y + M.y));
			o.gy = V2<real>::make(w * (P.y - M.y), -w * (P.x - M.x));
			o.gz = V2<real>::make(2 * w * Z.x, 2 * w * Z.y);
		} else {
			o.gx = o.gy = o.gz = V2<real>::make(0, 0);
		}
		put_coef(C, e, o);
	}
}

// phi and grad phi at (x, y, z) (the expansion's scaled frame) from the
// coefficients of derive_coefs (zero where a set has no such degree).
template <bool IRR, typename real>
__device__ void eval_cart(const Coef4<real>* C, real x, real y, real z, int N, real& pot, real& gx, real& gy,
                          real& gz)
{
	using v2 = typename V2<real>::t;
	const int NB = IRR ? N + 1 : N;
	const real r2 = x * x + y * y + z * z;
	const real ir2 = IRR ? real(1) / r2 : real(0);
	const real wx = IRR ? x * ir2 : x, wy = IRR ? y * ir2 : y;
	real bx = IRR ? rsq<real>(r2) : real(1), by = 0;
	real p = 0, ex = 0, ey = 0, ez = 0;
	for (int m = 0; m < NB; ++m) {
		if (m > 0) {
			const real sgm = sig_c<real>(m);
			const real nx = sgm * (wx * bx - wy * by), ny = sgm * (wx * by + wy * bx);
			bx = nx; by = ny;
		}
		real px = 0, py = 0, cx = bx, cy = by;
		int i = tix(m, m);
		for (int n = m; n < NB; ++n) {
			const Coef4<real> c = C[i];
			p = fma(c.f.x, cx, fma(-c.f.y, cy, p));
			ex = fma(c.gx.x, cx, fma(-c.gx.y, cy, ex));
			ey = fma(c.gy.x, cx, fma(-c.gy.y, cy, ey));
			ez = fma(c.gz.x, cx, fma(-c.gz.y, cy, ez));
			const v2 ab = rec_c<real>(i);
			const real az = ab.x * z, bb = IRR ? ab.y : ab.y * r2;
			real nx = fma(az, cx, -bb * px), ny = fma(az, cy, -bb * py);
			if (IRR) { nx *= ir2; ny *= ir2; }
			px = cx; py = cy; cx = nx; cy = ny;
			i += n + 1;                        // tix(n + 1, m)
		}
	}
	pot = p; gx = ex; gy = ey; gz = ez;
}

// The FP32 evaluation on packed f32x2 arithmetic (sm_100): the potential and
// d/dx sums in one float2, d/dy and d/dz in another, the harmonic's real and
// imaginary parts in a third; the same operations in the same order as the
// scalar form.
template <bool IRR>
__device__ void eval_cart(const CoefP* C, float x, float y, float z, int N, float& pot, float& gx, float& gy,
                          float& gz)
{
	const int NB = IRR ? N + 1 : N;
	const float r2 = x * x + y * y + z * z;
	const float ir2 = IRR ? 1.f / r2 : 0.f;
	const float wx = IRR ? x * ir2 : x, wy = IRR ? y * ir2 : y;
	float bx = IRR ? rsq<float>(r2) : 1.f, by = 0.f;
	float2 pe = make_float2(0.f, 0.f), yz = pe;
	const float2 ir22 = make_float2(ir2, ir2);
	for (int m = 0; m < NB; ++m) {
		if (m > 0) {
			const float sgm = sig_c<float>(m);
			const float nx = sgm * (wx * bx - wy * by), ny = sgm * (wx * by + wy * bx);
			bx = nx; by = ny;
		}
		float2 pv = make_float2(0.f, 0.f), cv = make_float2(bx, by);
		int i = tix(m, m);
		for (int n = m; n < NB; ++n) {
			const float4 re = C[i].re, im = C[i].im;
			const float2 cxx = make_float2(cv.x, cv.x), cyy = make_float2(cv.y, cv.y);
			pe = __ffma2_rn(make_float2(re.x, re.y), cxx, __ffma2_rn(make_float2(im.x, im.y), cyy, pe));
			yz = __ffma2_rn(make_float2(re.z, re.w), cxx, __ffma2_rn(make_float2(im.z, im.w), cyy, yz));
			const float2 ab = c_rec_f[i];
			const float az = ab.x * z, bb = IRR ? ab.y : ab.y * r2;
			float2 nv = __ffma2_rn(make_float2(az, az), cv, __fmul2_rn(make_float2(-bb, -bb), pv));
			if (IRR) nv = __fmul2_rn(nv, ir22);
			pv = cv; cv = nv;
			i += n + 1;                        // tix(n + 1, m)
		}
	}
	pot = pe.x; gx = pe.y; gy = yz.x; gz = yz.y;
}

// FP32 near field on its own (few registers, high occupancy): one warp per
// leaf, targets in passes of up to 32; a pass of np <= 16 targets runs
// TP = np rounded up to a power of two targets at once and splits the
// sources into 32 / TP phases (groups of 4), summed by shuffles.  Sources of
// the leaf and its U list are staged 32 at a time as negated hi + lo offsets in the
// target leaf's frame, padded with zero charges to a multiple of 4 and read
// as float4; the self pair is only tested for in the leaf's own chunks.
// Partial sums over 16 sources in FP32, carried in FP64; 1/r from the
// hardware approximation (relative error below 2^-22.9; r^2 >= 1e-8 is never
// subnormal).  Writes pot (with the reference's self term) and field in
// input order; the expansions are added by eval_scaled_kernel.
__device__ __forceinline__ float rsqrt_approx(float x)
{
	float y;
	asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
	return y;
}

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// Sources are staged NEGATED (leaf centre minus source, hi and lo), so each
// offset is a packed add: dx = (xi + sx) + (xl + lx), the same value as the
// difference.  Two sources per packed FP32 instruction (add / mul / fma
// .f32x2, sm_100); the clamp and 1/r stay scalar.
template <bool SELF>
__device__ __forceinline__ void p2p_f32_chunk(const float* __restrict__ sx, const float* __restrict__ sy,
                                              const float* __restrict__ sz, const float* __restrict__ lx,
                                              const float* __restrict__ ly, const float* __restrict__ lz,
                                              const float* __restrict__ sq, int cnt4, int jb, int js, int self,
                                              float xi, float yi, float zi, float xl, float yl, float zl,
                                              double& pot, double& fx, double& fy, double& fz)
{
	const float2 xi2 = f2(xi, xi), yi2 = f2(yi, yi), zi2 = f2(zi, zi);
	const float2 xl2 = f2(xl, xl), yl2 = f2(yl, yl), zl2 = f2(zl, zl);
	const float eps2 = (float)FORCE_EPS2;
	for (int j0 = jb; j0 < cnt4; j0 += 4 * js) {
		float2 p = f2(0.f, 0.f), ax = p, ay = p, az = p;
#pragma unroll
		for (int h = 0; h < 4; ++h) {
			const int j = j0 + js * h;
			if (j < cnt4) {
				const float4 X = *reinterpret_cast<const float4*>(sx + j), Y = *reinterpret_cast<const float4*>(sy + j);
				const float4 Z = *reinterpret_cast<const float4*>(sz + j), XL = *reinterpret_cast<const float4*>(lx + j);
				const float4 YL = *reinterpret_cast<const float4*>(ly + j), ZL = *reinterpret_cast<const float4*>(lz + j);
				const float4 Q = *reinterpret_cast<const float4*>(sq + j);
				const float2 xs[2] = {f2(X.x, X.y), f2(X.z, X.w)}, ys[2] = {f2(Y.x, Y.y), f2(Y.z, Y.w)};
				const float2 zs[2] = {f2(Z.x, Z.y), f2(Z.z, Z.w)}, xls[2] = {f2(XL.x, XL.y), f2(XL.z, XL.w)};
				const float2 yls[2] = {f2(YL.x, YL.y), f2(YL.z, YL.w)}, zls[2] = {f2(ZL.x, ZL.y), f2(ZL.z, ZL.w)};
				const float2 qs[2] = {f2(Q.x, Q.y), f2(Q.z, Q.w)};
#pragma unroll
				for (int k = 0; k < 2; ++k) {
					const float2 dx = __fadd2_rn(__fadd2_rn(xi2, xs[k]), __fadd2_rn(xl2, xls[k]));
					const float2 dy = __fadd2_rn(__fadd2_rn(yi2, ys[k]), __fadd2_rn(yl2, yls[k]));
					const float2 dz = __fadd2_rn(__fadd2_rn(zi2, zs[k]), __fadd2_rn(zl2, zls[k]));
					const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
					const float2 inv = f2(rsqrt_approx(fmaxf(r2.x, eps2)), rsqrt_approx(fmaxf(r2.y, eps2)));
					float2 qi = __fmul2_rn(qs[k], inv);
					if (SELF) {
						if (j + 2 * k == self) qi.x = 0.f;
						if (j + 2 * k + 1 == self) qi.y = 0.f;
					}
					const float2 qi3 = __fmul2_rn(qi, __fmul2_rn(inv, inv));
					p = __fadd2_rn(p, qi);
					ax = __ffma2_rn(dx, qi3, ax); ay = __ffma2_rn(dy, qi3, ay); az = __ffma2_rn(dz, qi3, az);
				}
			}
		}
		pot += (double)p.x + (double)p.y; fx += (double)ax.x + (double)ax.y;
		fy += (double)ay.x + (double)ay.y; fz += (double)az.x + (double)az.y;
	}
}

template <int LW>
__global__ void __launch_bounds__(LW * 32, 768 / (LW * 32)) p2p_f32_kernel(DevTree t, const float* __restrict__ qr,
                                                         double* __restrict__ pot_out, double* __restrict__ fld_out,
                                                         unsigned* __restrict__ next_leaf)
{
	__shared__ __align__(16) float sx[LW][32], sy[LW][32], sz[LW][32], sq[LW][32];
	__shared__ __align__(16) float lx[LW][32], ly[LW][32], lz[LW][32];
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const bool tmode = t.targets_num > 0;
	// a resident grid: each warp takes the next leaf from a counter
	for (;;) {
		unsigned lid = 0;
		if (lane == 0) lid = atomicAdd(next_leaf, 1u);
		const size_t li = __shfl_sync(0xffffffffu, lid, 0);
		if (li >= t.nleaves) return;
		const size_t g = t.leaves[li];
		const uint32_t tb = t.tbeg[g], te = t.tend[g];
		if (tb >= te) continue;
		const uint32_t ub = t.u_off[li], ue = t.u_off[li + 1];
		const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
		for (uint32_t t0 = tb; t0 < te; t0 += 32) {
			const int np = (int)min(32u, te - t0);
			int lt = 0;                            // log2 of the targets run at once
			while ((1 << lt) < np) ++lt;
			const int ti = lane & ((1 << lt) - 1), ph = lane >> lt, G = 32 >> lt;
			const uint32_t i = t0 + ti;
			const bool valid = ti < np;
			float xi = 0.f, yi = 0.f, zi = 0.f, xl = 0.f, yl = 0.f, zl = 0.f;
			if (valid) {
				const double ax_ = t.x[i] - cx, ay_ = t.y[i] - cy, az_ = t.z[i] - cz;
				xi = (float)ax_; yi = (float)ay_; zi = (float)az_;
				xl = (float)(ax_ - (double)xi); yl = (float)(ay_ - (double)yi); zl = (float)(az_ - (double)zi);
			}
			double pot = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
			for (int64_t e = (int64_t)ub - 1; e < (int64_t)ue; ++e) {
				const bool own = e < (int64_t)ub;
				const size_t sc_ = own ? g : (size_t)t.u_idx[e];
				const uint32_t sb = t.pbeg[sc_], se = t.send[sc_];
				for (uint32_t s0 = sb; s0 < se; s0 += 32) {
					const int cnt = min(32u, se - s0), cnt4 = (cnt + 3) & ~3;
					__syncwarp();
					if (lane < cnt) {
						const uint32_t j = s0 + lane;
						const double dx_ = cx - t.x[j], dy_ = cy - t.y[j], dz_ = cz - t.z[j];   // negated
						const float hx = (float)dx_, hy = (float)dy_, hz = (float)dz_;
						sx[w][lane] = hx; sy[w][lane] = hy; sz[w][lane] = hz;
						lx[w][lane] = (float)(dx_ - (double)hx); ly[w][lane] = (float)(dy_ - (double)hy);
						lz[w][lane] = (float)(dz_ - (double)hz);
						sq[w][lane] = qr[j];
					} else if (lane < cnt4) {
						sx[w][lane] = sy[w][lane] = sz[w][lane] = 0.f;
						lx[w][lane] = ly[w][lane] = lz[w][lane] = 0.f;
						sq[w][lane] = 0.f;
					}
					__syncwarp();
					if (valid) {
						if (own)
							p2p_f32_chunk<true>(sx[w], sy[w], sz[w], lx[w], ly[w], lz[w], sq[w], cnt4, 4 * ph, 4 * G,
							                    (int)(i - s0), xi, yi, zi, xl, yl, zl, pot, fx, fy, fz);
						else
							p2p_f32_chunk<false>(sx[w], sy[w], sz[w], lx[w], ly[w], lz[w], sq[w], cnt4, 4 * ph, 4 * G, -1, xi,
							                     yi, zi, xl, yl, zl, pot, fx, fy, fz);
					}
				}
			}
			for (int o = 1 << lt; o < 32; o <<= 1) {
				pot += __shfl_xor_sync(0xffffffffu, pot, o);
				fx += __shfl_xor_sync(0xffffffffu, fx, o);
				fy += __shfl_xor_sync(0xffffffffu, fy, o);
				fz += __shfl_xor_sync(0xffffffffu, fz, o);
			}
			if (valid && ph == 0) {
				if (!tmode) pot += t.q[i] * (1.0 / FORCE_EPS);
				const uint32_t o = t.orig[i];
				pot_out[o] = pot;
				fld_out[3 * (size_t)o] = fx; fld_out[3 * (size_t)o + 1] = fy; fld_out[3 * (size_t)o + 2] = fz;
			}
		}
	}
}

// M2P over the W list and L2P of the leaf's local expansion, added onto the
// near field already in the outputs: one warp per leaf at a time, lane =
// target; each
// expansion's coefficients derived once per 32 targets (derive_coefs), the
// targets evaluated by eval_cart.
template <typename real> constexpr int eval_warps() { return sizeof(real) == sizeof(float) ? 4 : 2; }

template <typename real, int LW>
__global__ void __launch_bounds__(LW * 32) eval_scaled_kernel(DevTree t, const typename V2<real>::t* __restrict__ outer,
                                                             const typename V2<real>::t* __restrict__ inner, int N,
                                                             double* __restrict__ pot_out, double* __restrict__ fld_out,
                                                             unsigned* __restrict__ next_leaf)
{
	__shared__ typename CoefStore<real>::t sC[LW][NXD];
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	// a resident grid: each warp takes the next leaf from a counter (leaves'
	// W lists differ in length, so fixed blocks of leaves finish unevenly)
	for (;;) {
		unsigned lid = 0;
		if (lane == 0) lid = atomicAdd(next_leaf, 1u);
		const size_t li = __shfl_sync(0xffffffffu, lid, 0);
		if (li >= t.nleaves) return;
		const size_t g = t.leaves[li];
		const uint32_t tb = t.tbeg[g], te = t.tend[g];
		if (tb >= te) continue;
		const int Nx2 = N * (N + 1) / 2;
		const double ihg = 1.0 / cell_size(t, g);
		const uint32_t wb = t.w_off[li], we = t.w_off[li + 1];
		const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
		for (uint32_t t0 = tb; t0 < te; t0 += 32) {
			const uint32_t i = t0 + lane;
			const bool valid = i < te;
			double xi = 0, yi = 0, zi = 0;
			if (valid) { xi = t.x[i]; yi = t.y[i]; zi = t.z[i]; }
			double pot = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
			for (uint32_t e = wb; e < we; ++e) {
				const size_t D = t.w_idx[e];
				__syncwarp();
				derive_coefs<true, real>(outer + D * Nx2, N, sC[w], lane);
				__syncwarp();
				if (valid) {
					const double ihd = 1.0 / cell_size(t, D);
					real mp, gx, gy, gz;
					eval_cart<true>(sC[w], (real)((xi - t.cx[D]) * ihd), (real)((yi - t.cy[D]) * ihd),
					                      (real)((zi - t.cz[D]) * ihd), N, mp, gx, gy, gz);
					pot += (double)mp * ihd;
					fx -= (double)gx * ihd * ihd; fy -= (double)gy * ihd * ihd; fz -= (double)gz * ihd * ihd;
				}
			}
			__syncwarp();
			derive_coefs<false, real>(inner + g * Nx2, N, sC[w], lane);
			__syncwarp();
			if (valid) {
				real lp, gx, gy, gz;
				eval_cart<false>(sC[w], (real)((xi - cx) * ihg), (real)((yi - cy) * ihg),
				                       (real)((zi - cz) * ihg), N, lp, gx, gy, gz);
				pot += (double)lp * ihg;
				fx -= (double)gx * ihg * ihg; fy -= (double)gy * ihg * ihg; fz -= (double)gz * ihg * ihg;
				const uint32_t o = t.orig[i];
				pot_out[o] += pot;
				fld_out[3 * (size_t)o] += fx; fld_out[3 * (size_t)o + 1] += fy; fld_out[3 * (size_t)o + 2] += fz;
			}
		}
	}
}

} // namespace scaled
} // namespace lfmm
