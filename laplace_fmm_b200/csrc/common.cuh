// Shared device/host helpers for the B200 Laplace FMM (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace lfmm {

constexpr int WARP = 32;
constexpr double FORCE_EPS = 1.0e-4;            // distance clamp (reference common/defs.h:24)
constexpr double FORCE_EPS2 = FORCE_EPS * FORCE_EPS;
constexpr int MAXN3 = 18;                       // max degrees in 3D (reference common/defs.h:33)
constexpr int MAXN2 = 30;                       // max degrees in 2D (reference common/defs.h:32)
constexpr int AUTO = 0x7fffffff;                // FMM_AUTO (reference common/defs.h:22)
constexpr double PI = 3.14159265358979323846;

// Triangular (n,m) index, 0 <= m <= n (reference common/utils.h:130-147).
__host__ __device__ constexpr inline int tix(int n, int m) { return n * (n + 1) / 2 + m; }
// The degree n of triangular index c = tix(n, m) (m = c - tix(n, 0)), computed
// rather than looked up: lanes of a warp ask for different c, which a
// constant-memory table would serialise.
__device__ __forceinline__ int tri_row(int c)
{
	// n = (sqrt(8c + 1) - 1) / 2 from the hardware reciprocal square root
	// (r >= 1); the estimate is within one of n, which the two steps correct
	const float r = 8.f * (float)c + 1.f;
	int n = (int)((r * rsqrtf(r) - 1.f) * 0.5f);
	if (tix(n + 1, 0) <= c) ++n;
	if (tix(n, 0) > c) --n;
	return n;
}
// Wigner-d (n,m,k) index, |k| <= n (reference common/special_functions.cpp:216-221).
__host__ __device__ constexpr inline int dix(int n, int m, int k)
{ return n * (n + 1) * (4 * n - 1) / 6 + m * (2 * n + 1) + (k + n); }
__host__ __device__ constexpr inline int dsize(int N) { return N * (N + 1) * (4 * N - 1) / 6; }
__host__ __device__ constexpr inline double sgn_n(int n) { return (n & 1) ? -1.0 : 1.0; }

// Status codes returned across the C ABI.
enum Status : int {
	OK = 0,
	ERR_ARG = -1,
	ERR_CUDA = -2,
	ERR_OOM = -3,
	ERR_DEVICE = -4,     // a device-side check failed (error flag set by a kernel)
	ERR_UNSUPPORTED = -5,
};

// Device-side error flags, OR-ed by kernels that detect a broken invariant;
// the host reads them after a solve and turns them into ERR_DEVICE.
enum DeviceError : unsigned {
	DEV_ERR_LIST_OVERFLOW = 1u,
	DEV_ERR_DIRECTION = 2u,
	DEV_ERR_RANGE = 4u,
};

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// (-1)^n as a double
__device__ __forceinline__ double dsgn(int n) { return (n & 1) ? -1.0 : 1.0; }

struct cplxd { double re, im; };

// Spherical coordinates with the reference's conventions
// (common/simple_math.h:101-117): r gets +1e-12, phi = 0 on the z-axis,
// +-pi/2 when |x| < 1e-12.
template <typename real>
__device__ __forceinline__ void dec_to_sph(real x, real y, real z, real& r, real& th, real& ph)
{
	const real e = real(1e-12);
	r = sqrt(x * x + y * y + z * z) + e;
	th = acos(z / r);
	if (fabs(x) + fabs(y) < e) ph = real(0);
	else if (fabs(x) < e) ph = y / fabs(y) * real(PI * 0.5);
	else ph = atan2(y, x);
}

// Morton helpers: spread / gather every dim-th bit.
__host__ __device__ inline uint64_t spread3(uint64_t v)
{
	v &= 0x1fffffull;
	v = (v | (v << 32)) & 0x001f00000000ffffull;
	v = (v | (v << 16)) & 0x001f0000ff0000ffull;
	v = (v | (v << 8)) & 0x100f00f00f00f00full;
	v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
	v = (v | (v << 2)) & 0x1249249249249249ull;
	return v;
}
__host__ __device__ inline uint32_t compact3(uint64_t v)
{
	v &= 0x1249249249249249ull;
	v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
	v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
	v = (v ^ (v >> 8)) & 0x001f0000ff0000ffull;
	v = (v ^ (v >> 16)) & 0x001f00000000ffffull;
	v = (v ^ (v >> 32)) & 0x1fffffull;
	return (uint32_t)v;
}
__host__ __device__ inline uint64_t spread2(uint64_t v)
{
	v &= 0xffffffffull;
	v = (v | (v << 16)) & 0x0000ffff0000ffffull;
	v = (v | (v << 8)) & 0x00ff00ff00ff00ffull;
	v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0full;
	v = (v | (v << 2)) & 0x3333333333333333ull;
	v = (v | (v << 1)) & 0x5555555555555555ull;
	return v;
}
__host__ __device__ inline uint32_t compact2(uint64_t v)
{
	v &= 0x5555555555555555ull;
	v = (v ^ (v >> 1)) & 0x3333333333333333ull;
	v = (v ^ (v >> 2)) & 0x0f0f0f0f0f0f0f0full;
	v = (v ^ (v >> 4)) & 0x00ff00ff00ff00ffull;
	v = (v ^ (v >> 8)) & 0x0000ffff0000ffffull;
	v = (v ^ (v >> 16)) & 0x00000000ffffffffull;
	return (uint32_t)v;
}

inline unsigned div_up(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

} // namespace lfmm
