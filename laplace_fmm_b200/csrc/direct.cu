// FP64 direct sums on the device: every target against every source, with
// the reference's clamp of r at 1e-4 and its self term (reference
// common/simple_math.h:130-216 pair kernels, simple_math.cu:9-23 the GPU
// ComputeExact).  Thread per target, sources staged through shared memory.
#include "direct.cuh"

namespace lfmm {

namespace {

constexpr int DT = 128;

__global__ void __launch_bounds__(DT) direct3d_kernel(size_t ns, const double* __restrict__ src,
                                                      const double* __restrict__ q, size_t nt,
                                                      const double* __restrict__ tgt, double* __restrict__ pot,
                                                      double* __restrict__ fld)
{
	__shared__ double sx[DT], sy[DT], sz[DT], sq[DT];
	size_t i = (size_t)blockIdx.x * DT + threadIdx.x;
	const bool valid = i < nt;
	double xi = 0, yi = 0, zi = 0;
	if (valid) { xi = tgt[3 * i]; yi = tgt[3 * i + 1]; zi = tgt[3 * i + 2]; }
	double p = 0, fx = 0, fy = 0, fz = 0;
	for (size_t s0 = 0; s0 < ns; s0 += DT) {
		int cnt = (int)min((size_t)DT, ns - s0);
		__syncthreads();
		if (threadIdx.x < cnt) {
			size_t j = s0 + threadIdx.x;
			sx[threadIdx.x] = src[3 * j]; sy[threadIdx.x] = src[3 * j + 1]; sz[threadIdx.x] = src[3 * j + 2];
			sq[threadIdx.x] = q[j];
		}
		__syncthreads();
		for (int j = 0; j < cnt; ++j) {
			double dx = xi - sx[j], dy = yi - sy[j], dz = zi - sz[j];
			double r = fmax(sqrt(dx * dx + dy * dy + dz * dz), FORCE_EPS);
			double qr = sq[j] / r;
			double qr3 = qr / (r * r);
			p += qr;
			fx = fma(dx, qr3, fx); fy = fma(dy, qr3, fy); fz = fma(dz, qr3, fz);
		}
	}
	if (valid) { pot[i] = p; fld[3 * i] = fx; fld[3 * i + 1] = fy; fld[3 * i + 2] = fz; }
}

__global__ void __launch_bounds__(DT) direct2d_kernel(size_t ns, const double* __restrict__ src,
                                                      const double* __restrict__ q, size_t nt,
                                                      const double* __restrict__ tgt, double* __restrict__ pot,
                                                      double* __restrict__ fld)
{
	__shared__ double sx[DT], sy[DT], sq[DT];
	size_t i = (size_t)blockIdx.x * DT + threadIdx.x;
	const bool valid = i < nt;
	double xi = 0, yi = 0;
	if (valid) { xi = tgt[2 * i]; yi = tgt[2 * i + 1]; }
	double p = 0, fr = 0, fi = 0;
	for (size_t s0 = 0; s0 < ns; s0 += DT) {
		int cnt = (int)min((size_t)DT, ns - s0);
		__syncthreads();
		if (threadIdx.x < cnt) {
			size_t j = s0 + threadIdx.x;
			sx[threadIdx.x] = src[2 * j]; sy[threadIdx.x] = src[2 * j + 1]; sq[threadIdx.x] = q[j];
		}
		__syncthreads();
		for (int j = 0; j < cnt; ++j) {
			double dx = xi - sx[j], dy = yi - sy[j];
			double r2 = fmax(dx * dx + dy * dy, FORCE_EPS2);
			p += sq[j] * 0.5 * log(r2);
			double qr = sq[j] / r2;
			fr = fma(dx, qr, fr); fi = fma(-dy, qr, fi);
		}
	}
	if (valid) { pot[i] = p; fld[2 * i] = fr; fld[2 * i + 1] = fi; }
}

} // namespace

int direct_device(Context& ctx, int dim, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                  double* pot, double* fld)
{
	if (nt == 0) return OK;
	unsigned grid = div_up(nt, DT);
	if (dim == 3) direct3d_kernel<<<grid, DT, 0, ctx.stream>>>(ns, src, q, nt, tgt, pot, fld);
	else direct2d_kernel<<<grid, DT, 0, ctx.stream>>>(ns, src, q, nt, tgt, pot, fld);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

} // namespace lfmm
