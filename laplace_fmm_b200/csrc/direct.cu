// FP64 direct sums on the device: every target against every source, with
// the reference's clamp of r at 1e-4 and its self term (reference
// common/simple_math.h:130-216 pair kernels, simple_math.cu:9-23 the GPU
// ComputeExact).  Thread per target, sources staged through shared memory.
//
// With few targets (the sampled accuracy check: thousands of targets against
// millions of sources) one block per 128 targets would leave most SMs idle, so
// the sources are split into S chunks: block (tile, chunk) writes its partial
// sums to scratch [S][nt][4] and a second kernel adds the S partials of each
// target in chunk order (deterministic).
#include "direct.cuh"

namespace lfmm {

namespace {

constexpr int DT = 128;

// 1 / sqrt(x) for the sampled checks (x = the clamped r^2 >= 1e-8): the
// hardware's FP64 reciprocal square root approximation (rsqrt.approx.ftz.f64,
// no FP32 round trip) refined by one third-order step of the binomial series
// (1 - r)^(-1/2) = 1 + r/2 + 3r^2/8 + ..., r = 1 - x y^2: a seed error e
// leaves ~(5/16)(2e)^3, below FP64 rounding for e < 2^-18.  The FP64 square
// root and divide above 1e300.
__device__ __forceinline__ double rsqrt_refined(double x)
{
	if (!(x < 1e300)) return 1.0 / sqrt(x);
	double y;
	asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
	const double r = fma(-x * y, y, 1.0);
	return fma(y * r, fma(r, 0.375, 0.5), y);
}

// Sums of target i over sources [s_lo, s_hi): out[0] = potential, out[1..dim] = field.
// FAST (3D, the sampled accuracy checks): 1/r from rsqrt_refined of the
// clamped r^2 instead of a square root and a divide.
template <int DIM, bool FAST = false>
__device__ __forceinline__ void direct_range(size_t s_lo, size_t s_hi, const double* __restrict__ src,
                                             const double* __restrict__ q, double xi, double yi, double zi,
                                             double out[4])
{
	__shared__ double sx[DT], sy[DT], sz[DT], sq[DT];
	double p = 0, fx = 0, fy = 0, fz = 0;
	for (size_t s0 = s_lo; s0 < s_hi; s0 += DT) {
		int cnt = (int)min((size_t)DT, s_hi - s0);
		__syncthreads();
		if (threadIdx.x < cnt) {
			size_t j = s0 + threadIdx.x;
			sx[threadIdx.x] = src[DIM * j]; sy[threadIdx.x] = src[DIM * j + 1];
			if (DIM == 3) sz[threadIdx.x] = src[DIM * j + 2];
			sq[threadIdx.x] = q[j];
		}
		__syncthreads();
		if (DIM == 3 && FAST) {
			for (int j = 0; j < cnt; ++j) {
				double dx = xi - sx[j], dy = yi - sy[j], dz = zi - sz[j];
				const double inv = rsqrt_refined(fmax(dx * dx + dy * dy + dz * dz, FORCE_EPS2));
				const double qr = sq[j] * inv;
				const double qr3 = qr * inv * inv;
				p += qr;
				fx = fma(dx, qr3, fx); fy = fma(dy, qr3, fy); fz = fma(dz, qr3, fz);
			}
		} else if (DIM == 3) {
			for (int j = 0; j < cnt; ++j) {
				double dx = xi - sx[j], dy = yi - sy[j], dz = zi - sz[j];
				double r = fmax(sqrt(dx * dx + dy * dy + dz * dz), FORCE_EPS);
				double qr = sq[j] / r;
				double qr3 = qr / (r * r);
				p += qr;
				fx = fma(dx, qr3, fx); fy = fma(dy, qr3, fy); fz = fma(dz, qr3, fz);
			}
		} else {
			for (int j = 0; j < cnt; ++j) {
				double dx = xi - sx[j], dy = yi - sy[j];
				double r2 = fmax(dx * dx + dy * dy, FORCE_EPS2);
				p += sq[j] * 0.5 * log(r2);
				double qr = sq[j] / r2;
				fx = fma(dx, qr, fx); fy = fma(-dy, qr, fy);
			}
		}
	}
	out[0] = p; out[1] = fx; out[2] = fy; out[3] = fz;
}

// grid (target tiles, source chunks).  part == nullptr: one chunk, results
// straight to pot/fld; else partials to part[(chunk * nt + i) * 4 + k].
template <int DIM, bool FAST = false>
__global__ void __launch_bounds__(DT) direct_kernel(size_t ns, size_t chunk, const double* __restrict__ src,
                                                    const double* __restrict__ q, size_t nt,
                                                    const double* __restrict__ tgt, double* __restrict__ pot,
                                                    double* __restrict__ fld, double* __restrict__ part)
{
	const size_t i = (size_t)blockIdx.x * DT + threadIdx.x;
	const bool valid = i < nt;
	double xi = 0, yi = 0, zi = 0;
	if (valid) {
		xi = tgt[DIM * i]; yi = tgt[DIM * i + 1];
		if (DIM == 3) zi = tgt[DIM * i + 2];
	}
	const size_t lo = (size_t)blockIdx.y * chunk, hi = min(ns, lo + chunk);
	double r[4];
	direct_range<DIM, FAST>(lo, hi, src, q, xi, yi, zi, r);
	if (!valid) return;
	if (part) {
		double2* o = reinterpret_cast<double2*>(part + ((size_t)blockIdx.y * nt + i) * 4);
		o[0] = make_double2(r[0], r[1]);
		o[1] = make_double2(r[2], r[3]);
	} else {
		pot[i] = r[0];
		for (int k = 0; k < DIM; ++k) fld[DIM * i + k] = r[1 + k];
	}
}

template <int DIM>
__global__ void direct_reduce_kernel(size_t nt, int S, const double* __restrict__ part, double* __restrict__ pot,
                                     double* __restrict__ fld)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nt) return;
	double a[4] = {0, 0, 0, 0};
	for (int s = 0; s < S; ++s) {
		const double2* o = reinterpret_cast<const double2*>(part + ((size_t)s * nt + i) * 4);
		double2 u = o[0], v = o[1];
		a[0] += u.x; a[1] += u.y; a[2] += v.x; a[3] += v.y;
	}
	pot[i] = a[0];
	for (int k = 0; k < DIM; ++k) fld[DIM * i + k] = a[1 + k];
}

// Target i against the sources of its own segment [poff[seg[i]], poff[seg[i] + 1])
// (the sampled checks of a batch of problems in one launch): one block per
// target, the threads splitting the segment's sources, then a block
// reduction in fixed order.  3D, 1/r as in the FAST sums.
__global__ void __launch_bounds__(DT) direct_segments_kernel(const double* __restrict__ src,
                                                             const double* __restrict__ q,
                                                             const uint32_t* __restrict__ poff,
                                                             const int32_t* __restrict__ seg, size_t m,
                                                             const double* __restrict__ tgt,
                                                             double* __restrict__ pot, double* __restrict__ fld)
{
	const size_t i = blockIdx.x;
	if (i >= m) return;
	const int k = seg[i];
	const size_t lo = poff[k], hi = poff[k + 1];
	const double xi = tgt[3 * i], yi = tgt[3 * i + 1], zi = tgt[3 * i + 2];
	double v[4] = {0, 0, 0, 0};
	for (size_t j = lo + threadIdx.x; j < hi; j += DT) {
		const double dx = xi - src[3 * j], dy = yi - src[3 * j + 1], dz = zi - src[3 * j + 2];
		const double inv = rsqrt_refined(fmax(dx * dx + dy * dy + dz * dz, FORCE_EPS2));
		const double qr = q[j] * inv;
		const double qr3 = qr * inv * inv;
		v[0] += qr;
		v[1] = fma(dx, qr3, v[1]); v[2] = fma(dy, qr3, v[2]); v[3] = fma(dz, qr3, v[3]);
	}
	__shared__ double red[DT / 32][4];
#pragma unroll
	for (int c = 0; c < 4; ++c) {
		double x = v[c];
		for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
		if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][c] = x;
	}
	__syncthreads();
	if (threadIdx.x < 4) {
		double x = 0.0;
		for (int w = 0; w < DT / 32; ++w) x += red[w][threadIdx.x];
		if (threadIdx.x == 0) pot[i] = x;
		else fld[3 * i + threadIdx.x - 1] = x;
	}
}

} // namespace

int direct_segments_device(Context& ctx, const double* src, const double* q, const uint32_t* poff,
                           const int32_t* seg, size_t m, const double* tgt, double* pot, double* fld)
{
	if (m == 0) return OK;
	direct_segments_kernel<<<(unsigned)m, DT, 0, ctx.stream>>>(src, q, poff, seg, m, tgt, pot, fld);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

int direct_chunks(size_t ns, size_t nt, int num_sms, size_t max_chunks)
{
	const size_t tiles = (nt + DT - 1) / DT;
	const size_t want = (size_t)num_sms * 8;           // blocks for a full GPU (several per SM)
	if (tiles >= want || ns < 4 * (size_t)DT) return 1;
	size_t s = (want + tiles - 1) / tiles;
	s = std::min(s, (ns + 4 * DT - 1) / (4 * DT));     // at least 4 source tiles per chunk
	s = std::min(s, max_chunks);
	return (int)std::max<size_t>(s, 1);
}

int direct_launch(Context& ctx, int dim, size_t ns, const double* src, const double* q, size_t nt,
                  const double* tgt, double* pot, double* fld, double* part, int S, bool fast)
{
	if (nt == 0) return OK;
	if (S <= 1 || !part) S = 1, part = nullptr;
	const size_t chunk = S > 1 ? ((ns + S - 1) / S + DT - 1) / DT * DT : std::max<size_t>(ns, 1);
	S = S > 1 ? (int)((ns + chunk - 1) / chunk) : 1;
	if (S <= 1) part = nullptr;
	dim3 grid(div_up(nt, DT), S);
	if (dim == 3 && fast) direct_kernel<3, true><<<grid, DT, 0, ctx.stream>>>(ns, chunk, src, q, nt, tgt, pot, fld, part);
	else if (dim == 3) direct_kernel<3><<<grid, DT, 0, ctx.stream>>>(ns, chunk, src, q, nt, tgt, pot, fld, part);
	else direct_kernel<2><<<grid, DT, 0, ctx.stream>>>(ns, chunk, src, q, nt, tgt, pot, fld, part);
	if (part) {
		if (dim == 3) direct_reduce_kernel<3><<<div_up(nt, 256), 256, 0, ctx.stream>>>(nt, S, part, pot, fld);
		else direct_reduce_kernel<2><<<div_up(nt, 256), 256, 0, ctx.stream>>>(nt, S, part, pot, fld);
	}
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

int direct_preload3(Context& ctx)
{
	cudaFuncAttributes a;
	LFMM_CUDA(ctx, cudaFuncGetAttributes(&a, direct_kernel<3>));
	LFMM_CUDA(ctx, cudaFuncGetAttributes(&a, direct_reduce_kernel<3>));
	return OK;
}

int direct_device(Context& ctx, int dim, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                  double* pot, double* fld, bool fast)
{
	if (nt == 0) return OK;
	int S = direct_chunks(ns, nt, ctx.num_sms, 1024);
	double* part = nullptr;
	if (S > 1) {
		part = static_cast<double*>(ctx.arena.take(sizeof(double) * 4 * nt * (size_t)S));
		if (!part) S = 1;       // fall back to one chunk (no scratch)
	}
	return direct_launch(ctx, dim, ns, src, q, nt, tgt, pot, fld, part, S, fast);
}

} // namespace lfmm
