// Rotation and translation tables for the 3D rotation-based FMM.
//
// The reference keys its rotation tables by int(100 * angle) over the 316 far
// offsets of the 7x7x7 block minus its 3x3x3 core, last writer winning
// (reference common/special_functions.cpp:363-381), and looks them up with the
// angles of each runtime offset (cpu/multipole3d.cpp:152-165).  Here the same
// key -> canonical angle map is built on the host, every integer direction is
// resolved to its table slots once, and the Wigner small-d matrices are
// generated on the GPU in FP64 from that canonical angle with the reference's
// three-stage recurrence (special_functions.cpp:211-351).
#include "context.cuh"
#include <cmath>
#include <map>

namespace lfmm {

namespace {

void host_dec_to_sph(double x, double y, double z, double& r, double& th, double& ph)
{
	const double e = 1e-12;
	r = std::sqrt(x * x + y * y + z * z) + e;
	th = std::acos(z / r);
	if (std::fabs(x) + std::fabs(y) < e) ph = 0.0;
	else if (std::fabs(x) < e) ph = y / std::fabs(y) * PI * 0.5;
	else ph = std::atan2(y, x);
}

// One thread per degree n: fills d^n_{m,k}(theta) for all m >= 0, |k| <= n.
__global__ void wignerd_kernel(const double* __restrict__ thetas, int nslots, double* __restrict__ out)
{
	int slot = blockIdx.x;
	int n = threadIdx.x;
	if (slot >= nslots || n >= MAXN3) return;
	double* D = out + (size_t)slot * dsize(MAXN3);
	double theta = thetas[slot];
	bool isneg = theta < 0;
	theta = fabs(theta);
	bool closetopi = false;
	if (theta > PI / 2) { theta = PI - theta; closetopi = true; }
	for (int m = 0; m <= n; ++m)
		for (int k = -n; k <= n; ++k) D[dix(n, m, k)] = 0.0;
	if (fabs(theta) < 1e-3) {
		for (int m = 0; m <= n; ++m) D[dix(n, m, m)] = 1.0;
	} else {
		// g(n,0) = prod sqrt((2i-1)/(2i)); g(n,m) = g(n,m-1) sqrt((n-m+1)/(n+m))
		double g0 = 1.0;
		for (int i = 1; i <= n; ++i) g0 = sqrt((2 * i - 1.) / (2 * i)) * g0;
		double s = sin(theta), c = 1.0 + cos(theta), f = s / c;
		// stage 1: column k = n, d = (-1)^(n+m) g(n,m) c^m s^(n-m)
		double g = g0;
		for (int m = 0; m <= n; ++m) {
			if (m > 0) g = sqrt((n - m + 1.) / (n + m)) * g;
			double cp = 1.0, sp = 1.0;
			for (int i = 0; i < m; ++i) cp *= c;
			for (int i = 0; i < n - m; ++i) sp *= s;
			D[dix(n, m, n)] = sgn_n(n + m) * g * cp * sp;
		}
		// stage 2: row m = n, k descending
		for (int k = n; k > -n; --k)
			D[dix(n, n, k - 1)] = (n + k) / sqrt(n * (n + 1.) - k * (k - 1.)) * f * D[dix(n, n, k)];
		// stage 3: rows m < n from row m + 1
		for (int m = n - 1; m >= 0; --m)
			for (int k = n; k > -n; --k)
				D[dix(n, m, k - 1)] =
					sqrt((n * (n + 1.) - m * (m + 1.)) / (n * (n + 1.) - k * (k - 1.))) * D[dix(n, m + 1, k)] +
					(m + k) / sqrt(n * (n + 1.) - k * (k - 1.)) * f * D[dix(n, m, k)];
	}
	if (n == 0) return;
	if (closetopi) {   // d(pi - t)[n,m,k] = (-1)^(n+m) d(t)[n,m,-k]
		for (int m = 0; m <= n; ++m) {
			for (int k = 1; k <= n; ++k) {
				double a = D[dix(n, m, k)], b = D[dix(n, m, -k)];
				D[dix(n, m, k)] = b; D[dix(n, m, -k)] = a;
			}
			double sg = sgn_n(n + m);
			for (int k = -n; k <= n; ++k) D[dix(n, m, k)] *= sg;
		}
	}
	for (int m = 0; m <= n; ++m)
		for (int k = -n; k <= n; ++k) {
			double v = D[dix(n, m, k)];
			if (k < 0) v *= sgn_n(k);            // eps(k) convention of the reference's harmonics
			if (isneg) v *= sgn_n(m - k);        // d(-t) = (-1)^(m-k) d(t)
			D[dix(n, m, k)] = v;
		}
}

__global__ void to_float_kernel(const double* __restrict__ in, float* __restrict__ out, size_t n)
{
	size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (float)in[i];
}

__global__ void exp_kernel(const double* __restrict__ phis, int nslots, double2* __restrict__ out)
{
	int slot = blockIdx.x, m = threadIdx.x;
	if (slot >= nslots || m >= MAXN3) return;
	double a = m * phis[slot];
	out[slot * MAXN3 + m] = make_double2(cos(a), sin(a));
}

} // namespace

int tables_build(Context& ctx)
{
	Tables& TH = ctx.tables;
	DevTables& T = TH.d;
	// key -> canonical angle, in the reference's insertion order
	std::map<int, double> th_of_key, ph_of_key;
	for (int i = -3; i < 4; ++i)
		for (int j = -3; j < 4; ++j)
			for (int k = -3; k < 4; ++k) {
				if (std::abs(i) <= 1 && std::abs(j) <= 1 && std::abs(k) <= 1) continue;
				double r, th, ph;
				host_dec_to_sph(i, j, k, r, th, ph);
				int key = (int)(th * 100);
				th_of_key[key] = th;
				th_of_key[-key] = -th;
				key = (int)(ph * 100);
				ph_of_key[key] = ph;
				ph_of_key[-key] = -ph;
			}
	std::map<int, int> dslot, eslot;
	TH.theta_of_slot.clear(); TH.phi_of_slot.clear();
	for (auto& kv : th_of_key) { dslot[kv.first] = (int)TH.theta_of_slot.size(); TH.theta_of_slot.push_back(kv.second); }
	for (auto& kv : ph_of_key) { eslot[kv.first] = (int)TH.phi_of_slot.size(); TH.phi_of_slot.push_back(kv.second); }
	T.n_dslots = (int)TH.theta_of_slot.size();
	T.n_eslots = (int)TH.phi_of_slot.size();
	auto find = [](const std::map<int, int>& m, int key) { auto it = m.find(key); return it == m.end() ? -1 : it->second; };
	TH.dirinfo_host.assign(343, make_int4(-1, -1, -1, -1));
	for (int dx = -3; dx <= 3; ++dx)
		for (int dy = -3; dy <= 3; ++dy)
			for (int dz = -3; dz <= 3; ++dz) {
				if (!dx && !dy && !dz) continue;
				double r, th, ph;
				host_dec_to_sph(dx, dy, dz, r, th, ph);
				int id = (dx + 3) * 49 + (dy + 3) * 7 + (dz + 3);
				TH.dirinfo_host[id] = make_int4(find(dslot, (int)(th * 100)), find(dslot, (int)(-th * 100)),
				                               find(eslot, (int)(ph * 100)), find(eslot, (int)(-ph * 100)));
			}
	// normalisation constants, reference special_functions.h:56-116 recurrences
	std::vector<double> K(MAXN3 * (MAXN3 + 1) / 2), A(2 * MAXN3 * (2 * MAXN3 + 1) / 2);
	K[0] = 1.0;
	for (int n = 1; n < MAXN3; ++n) {
		for (int m = 0; m <= n - 1; ++m) K[tix(n, m)] = K[tix(n - 1, m)] * (n - m) / (n + m);
		K[tix(n, n)] = K[tix(n, n - 1)] / (2 * n);
	}
	for (int n = 1; n < MAXN3; ++n)
		for (int m = 0; m <= n; ++m) K[tix(n, m)] = std::sqrt(K[tix(n, m)]);
	A[0] = 1.0;
	for (int n = 1; n < 2 * MAXN3; ++n) {
		for (int m = 0; m <= n - 1; ++m) A[tix(n, m)] = A[tix(n - 1, m)] * (n - m) * (n + m);
		A[tix(n, n)] = A[tix(n, n - 1)] * 2 * n;
	}
	for (int n = 1; n < 2 * MAXN3; ++n)
		for (int m = 0; m <= n; ++m) A[tix(n, m)] = sgn_n(n) / std::sqrt(A[tix(n, m)]);
	auto An = [&](int n, int m) { return A[tix(n, m)]; };
	const int C = MAXN3 * MAXN3 * MAXN3;
	std::vector<double> m2l(C, 0.0), m2m(C, 0.0), l2l(C, 0.0);
	for (int j = 0; j < MAXN3; ++j)
		for (int k = 0; k <= j; ++k)
			for (int n = 0; n < MAXN3; ++n) {
				int idx = (j * MAXN3 + k) * MAXN3 + n;
				if (n >= k) m2l[idx] = An(n, k) * An(j, k) * sgn_n(n + k) / An(j + n, 0);
				if (j - n >= k) m2m[idx] = An(n, 0) * An(j - n, k) / An(j, k);
				if (n >= j) l2l[idx] = An(n - j, 0) * An(j, k) * sgn_n(n + j) / An(n, k);
			}
	size_t dbytes = sizeof(double) * dsize(MAXN3) * T.n_dslots;
	LFMM_CUDA(ctx, cudaMalloc(&T.dmat, dbytes));
	LFMM_CUDA(ctx, cudaMalloc(&T.emat, sizeof(double2) * MAXN3 * T.n_eslots));
	LFMM_CUDA(ctx, cudaMalloc(&T.dirinfo, sizeof(int4) * 343));
	LFMM_CUDA(ctx, cudaMalloc(&T.knm, sizeof(double) * K.size()));
	LFMM_CUDA(ctx, cudaMalloc(&T.m2l, sizeof(double) * C));
	LFMM_CUDA(ctx, cudaMalloc(&T.m2m, sizeof(double) * C));
	LFMM_CUDA(ctx, cudaMalloc(&T.l2l, sizeof(double) * C));
	double *d_th = nullptr, *d_ph = nullptr;
	LFMM_CUDA(ctx, cudaMalloc(&d_th, sizeof(double) * T.n_dslots));
	LFMM_CUDA(ctx, cudaMalloc(&d_ph, sizeof(double) * T.n_eslots));
	cudaStream_t s = ctx.stream;
	LFMM_CUDA(ctx, cudaMemcpyAsync(d_th, TH.theta_of_slot.data(), sizeof(double) * T.n_dslots, cudaMemcpyHostToDevice, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(d_ph, TH.phi_of_slot.data(), sizeof(double) * T.n_eslots, cudaMemcpyHostToDevice, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(T.dirinfo, TH.dirinfo_host.data(), sizeof(int4) * 343, cudaMemcpyHostToDevice, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(T.knm, K.data(), sizeof(double) * K.size(), cudaMemcpyHostToDevice, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(T.m2l, m2l.data(), sizeof(double) * C, cudaMemcpyHostToDevice, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(T.m2m, m2m.data(), sizeof(double) * C, cudaMemcpyHostToDevice, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(T.l2l, l2l.data(), sizeof(double) * C, cudaMemcpyHostToDevice, s));
	wignerd_kernel<<<T.n_dslots, 32, 0, s>>>(d_th, T.n_dslots, T.dmat);
	exp_kernel<<<T.n_eslots, 32, 0, s>>>(d_ph, T.n_eslots, T.emat);
	LFMM_CUDA(ctx, cudaGetLastError());
	// FP32 copies (mixed form)
	size_t nd = (size_t)dsize(MAXN3) * T.n_dslots, ne = (size_t)2 * MAXN3 * T.n_eslots;
	LFMM_CUDA(ctx, cudaMalloc(&T.dmat_f, sizeof(float) * nd));
	LFMM_CUDA(ctx, cudaMalloc(&T.emat_f, sizeof(float) * ne));
	LFMM_CUDA(ctx, cudaMalloc(&T.knm_f, sizeof(float) * K.size()));
	LFMM_CUDA(ctx, cudaMalloc(&T.m2l_f, sizeof(float) * C));
	LFMM_CUDA(ctx, cudaMalloc(&T.m2m_f, sizeof(float) * C));
	LFMM_CUDA(ctx, cudaMalloc(&T.l2l_f, sizeof(float) * C));
	to_float_kernel<<<div_up(nd, 256), 256, 0, s>>>(T.dmat, T.dmat_f, nd);
	to_float_kernel<<<div_up(ne, 256), 256, 0, s>>>(reinterpret_cast<const double*>(T.emat),
	                                                 reinterpret_cast<float*>(T.emat_f), ne);
	to_float_kernel<<<div_up(K.size(), 256), 256, 0, s>>>(T.knm, T.knm_f, K.size());
	to_float_kernel<<<div_up(C, 256), 256, 0, s>>>(T.m2l, T.m2l_f, C);
	to_float_kernel<<<div_up(C, 256), 256, 0, s>>>(T.m2m, T.m2m_f, C);
	to_float_kernel<<<div_up(C, 256), 256, 0, s>>>(T.l2l, T.l2l_f, C);
	LFMM_CUDA(ctx, cudaGetLastError());
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	cudaFree(d_th);
	cudaFree(d_ph);
	return OK;
}

void tables_free(Tables& TH)
{
	DevTables& T = TH.d;
	cudaFree(T.dmat); cudaFree(T.emat); cudaFree(T.dirinfo); cudaFree(T.knm);
	cudaFree(T.m2l); cudaFree(T.m2m); cudaFree(T.l2l);
	cudaFree(T.dmat_f); cudaFree(T.emat_f); cudaFree(T.knm_f);
	cudaFree(T.m2l_f); cudaFree(T.m2m_f); cudaFree(T.l2l_f);
	TH = Tables();
}

} // namespace lfmm
