// Vector charges: the reference's fmm::FastMultipole3d<Vector3d>
// (cpu/multipole3d.h:10-24 with value = Vector3d, leaves and field at
// cpu/multipole3d.cpp:414-853, instantiated at :1397).  At every target
//   B_j = sum_i q_i x (x_j - x_i) / max(r, 1e-4)^3
// (the reference's cross products in the near field, and in the far field
// f += (g_y)_z - (g_z)_y, ... of its three expansions' gradients); it
// computes no potential for vector charges.  Since q x d = sum_c q^c (e_c x d),
// B = sum_c e_c x E^(c) with E^(c) the scalar field of the charges'
// component c: one tree (its sources are the particles with q != 0, the
// reference's zero-charge rule for vectors, cpu/morton_tree.cpp:433-448),
// three scalar passes on it, and a cross product.
#include "fmm3d.cuh"
#include "m2l_gemm.cuh"
#include <algorithm>

namespace lfmm {

namespace {

// 1 where the particle's vector charge is nonzero: the tree's source /
// target split
__global__ void nonzero_kernel(const double* __restrict__ q3, size_t n, double* __restrict__ s)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) s[i] = (q3[3 * i] != 0.0 || q3[3 * i + 1] != 0.0 || q3[3 * i + 2] != 0.0) ? 1.0 : 0.0;
}

// component c of the charges into the tree's charge array (targets: 0)
__global__ void component_kernel(DevTree t, size_t nt, const double* __restrict__ q3, int c)
{
	const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= t.n) return;
	const uint32_t o = t.orig[s];
	t.q[s] = o < nt ? 0.0 : q3[3 * (o - nt) + c];
}

// B = e_x x E^(x) + e_y x E^(y) + e_z x E^(z); E: [3][n][3]
__global__ void curl_kernel(const double* __restrict__ E, size_t n, double* __restrict__ B)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const double* ex = E + 3 * i;
	const double* ey = E + 3 * (n + i);
	const double* ez = E + 3 * (2 * n + i);
	B[3 * i] = ey[2] - ez[1];
	B[3 * i + 1] = ez[0] - ex[2];
	B[3 * i + 2] = ex[1] - ey[0];
}

} // namespace

int fmm3d_solve_vector(Context& ctx, const ParticleInput& in, int N, int depth, int max_leaf, int precision,
                       double* field, SolveStats* stats)
{
	if (N < 1 || N > MAXN3) { ctx.last_error = "order out of range (1 <= N <= 18)"; return ERR_ARG; }
	if (!m2l_gemm_supported(N)) { ctx.last_error = "vector charges use the scaled form: N <= 18"; return ERR_UNSUPPORTED; }
	if (max_leaf < 0) { ctx.last_error = "max_leaf must be >= 0"; return ERR_ARG; }
	cudaStream_t s = ctx.stream;
	const size_t n_out = in.nt ? in.nt : in.ns;
	double* sur = static_cast<double*>(ctx.arena.take(sizeof(double) * std::max<size_t>(in.ns, 1)));
	double* E = static_cast<double*>(ctx.arena.take(sizeof(double) * 9 * n_out));
	double* pot = static_cast<double*>(ctx.arena.take(sizeof(double) * n_out));
	if (!sur || !E || !pot) { ctx.last_error = "vector solve: allocation failed"; return ERR_OOM; }
	if (in.ns) nonzero_kernel<<<div_up(in.ns, 256), 256, 0, s>>>(in.srcq, in.ns, sur);
	ParticleInput split = in;
	split.srcq = sur;
	DevTree t;
	int st = tree_build_adaptive(ctx, split, depth, max_leaf, t);
	if (st) return st;
	for (int c = 0; c < 3; ++c) {
		if (c == 2 && stats && ctx.timing) {
			// the statistics' phases and kernel times describe the last pass
			ctx.kev_used = 0;
			LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[0], s));
			LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[1], s));
		}
		component_kernel<<<div_up(t.n, 256), 256, 0, s>>>(t, in.nt, in.srcq, c);
		if ((st = fmm3d_scaled_on_tree(ctx, t, N, precision, pot, E + 3 * n_out * c, c == 2 ? stats : nullptr)))
			return st;
	}
	curl_kernel<<<div_up(n_out, 256), 256, 0, s>>>(E, n_out, field);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

} // namespace lfmm
