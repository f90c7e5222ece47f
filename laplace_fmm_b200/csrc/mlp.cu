// Order-selection MLP: 16 features -> 64 -> 64 -> 14 outputs (FP32, ReLU),
// trained on the GPU by these kernels (forward, masked-MSE backward, Adam).
// Outputs 0-6 predict log10 of a leaf box's potential error at the orders
// p = 4, 6, 8, 10, 12, 14, 16; outputs 7-13 its field error at the same orders.
//
// Parameter layout (floats): W1[64][16] b1[64] W2[64][64] b2[64] W3[14][64] b3[14].
#include "learned.cuh"

namespace lfmm {

namespace {

constexpr int F = LFMM_MLP_IN, H = LFMM_MLP_HIDDEN, O = LFMM_MLP_OUT;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * F, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + O * H, NPARAM = OFF_B3 + O;
static_assert(NPARAM == LFMM_MLP_PARAMS, "parameter count");

constexpr int MT = 32;   // rows (samples) per block (static shared memory <= 48 KB)

// Forward for a block of 32 samples; thread t < 64 computes hidden unit t for
// every sample of the block (weights in shared memory, activations too).  The
// first two layers' weights are stored transposed ([input][unit]), so a warp's
// reads of one input's weights fall in distinct banks (row-major, units 64
// floats apart all hit one bank); the same values in the same order.
__global__ void __launch_bounds__(64) mlp_forward_kernel(const float* __restrict__ P, int n, const float* __restrict__ X,
                                                         float* __restrict__ Y, float* __restrict__ A1,
                                                         float* __restrict__ A2)
{
	__shared__ float sW1t[F * H], sb1[H], sW2t[H * H], sb2[H], sW3[O * H], sb3[O];
	__shared__ float sX[MT][F];
	__shared__ float sA1[MT][H + 1], sA2[MT][H + 1];
	const int t = threadIdx.x;
	for (int i = t; i < H * F; i += 64) sW1t[(i % F) * H + i / F] = P[OFF_W1 + i];
	for (int i = t; i < H * H; i += 64) sW2t[(i % H) * H + i / H] = P[OFF_W2 + i];
	for (int i = t; i < O * H; i += 64) sW3[i] = P[OFF_W3 + i];
	sb1[t] = P[OFF_B1 + t]; sb2[t] = P[OFF_B2 + t];
	if (t < O) sb3[t] = P[OFF_B3 + t];
	const int r0 = blockIdx.x * MT;
	for (int i = t; i < MT * F; i += 64) {
		int r = i / F, c = i % F;
		sX[r][c] = r0 + r < n ? X[(size_t)(r0 + r) * F + c] : 0.f;
	}
	__syncthreads();
	for (int r = 0; r < MT; ++r) {
		float a = sb1[t];
		for (int c = 0; c < F; ++c) a = fmaf(sW1t[c * H + t], sX[r][c], a);
		sA1[r][t] = fmaxf(a, 0.f);
	}
	__syncthreads();
	for (int r = 0; r < MT; ++r) {
		float a = sb2[t];
		for (int c = 0; c < H; ++c) a = fmaf(sW2t[c * H + t], sA1[r][c], a);
		sA2[r][t] = fmaxf(a, 0.f);
	}
	__syncthreads();
	for (int i = t; i < MT * O; i += 64) {
		int r = i / O, k = i % O;
		float a = sb3[k];
		for (int c = 0; c < H; ++c) a = fmaf(sW3[k * H + c], sA2[r][c], a);
		if (r0 + r < n) Y[(size_t)(r0 + r) * O + k] = a;
	}
	if (A1)
		for (int i = t; i < MT * H; i += 64) {
			int r = i / H, c = i % H;
			if (r0 + r < n) { A1[(size_t)(r0 + r) * H + c] = sA1[r][c]; A2[(size_t)(r0 + r) * H + c] = sA2[r][c]; }
		}
}

// Backward of the masked mean-squared error L = sum M (Y - T)^2 / sum M.
// Each block handles 32 samples and accumulates its parameter gradients with
// atomics into G (zeroed by the host); the loss numerator and mask count go to
// acc[0], acc[1].
__global__ void __launch_bounds__(64) mlp_backward_kernel(const float* __restrict__ P, int n, const float* __restrict__ X,
                                                          const float* __restrict__ Y, const float* __restrict__ A1,
                                                          const float* __restrict__ A2, const float* __restrict__ T,
                                                          const float* __restrict__ M, float inv_count,
                                                          float* __restrict__ G, float* __restrict__ acc)
{
	__shared__ float sW3[O * H];
	__shared__ float sD3[MT][O], sD2[MT][H + 1], sD1[MT][H + 1];
	const float* sW2 = P + OFF_W2;      // read through L1
	__shared__ float sX[MT][F], sA1[MT][H + 1], sA2[MT][H + 1];
	const int t = threadIdx.x;
	for (int i = t; i < O * H; i += 64) sW3[i] = P[OFF_W3 + i];
	const int r0 = blockIdx.x * MT;
	float lsum = 0.f, msum = 0.f;
	for (int i = t; i < MT * O; i += 64) {
		int r = i / O, k = i % O;
		float d = 0.f;
		if (r0 + r < n) {
			size_t j = (size_t)(r0 + r) * O + k;
			float m = M[j], e = Y[j] - T[j];
			d = 2.f * m * e * inv_count;
			lsum += m * e * e; msum += m;
		}
		sD3[r][k] = d;
	}
	for (int i = t; i < MT * H; i += 64) {
		int r = i / H, c = i % H;
		bool ok = r0 + r < n;
		sA1[r][c] = ok ? A1[(size_t)(r0 + r) * H + c] : 0.f;
		sA2[r][c] = ok ? A2[(size_t)(r0 + r) * H + c] : 0.f;
	}
	for (int i = t; i < MT * F; i += 64) {
		int r = i / F, c = i % F;
		sX[r][c] = r0 + r < n ? X[(size_t)(r0 + r) * F + c] : 0.f;
	}
	atomicAdd(&acc[0], lsum);
	atomicAdd(&acc[1], msum);
	__syncthreads();
	// dA2 = D3 W3, masked by ReLU
	for (int r = 0; r < MT; ++r) {
		float a = 0.f;
		for (int k = 0; k < O; ++k) a = fmaf(sD3[r][k], sW3[k * H + t], a);
		sD2[r][t] = sA2[r][t] > 0.f ? a : 0.f;
	}
	__syncthreads();
	for (int r = 0; r < MT; ++r) {
		float a = 0.f;
		for (int k = 0; k < H; ++k) a = fmaf(sD2[r][k], sW2[k * H + t], a);
		sD1[r][t] = sA1[r][t] > 0.f ? a : 0.f;
	}
	__syncthreads();
	// parameter gradients (block partial sums, then atomics)
	for (int i = t; i < O * H; i += 64) {
		int k = i / H, c = i % H;
		float g = 0.f;
		for (int r = 0; r < MT; ++r) g = fmaf(sD3[r][k], sA2[r][c], g);
		atomicAdd(&G[OFF_W3 + i], g);
	}
	if (t < O) {
		float g = 0.f;
		for (int r = 0; r < MT; ++r) g += sD3[r][t];
		atomicAdd(&G[OFF_B3 + t], g);
	}
	for (int i = t; i < H * H; i += 64) {
		int k = i / H, c = i % H;
		float g = 0.f;
		for (int r = 0; r < MT; ++r) g = fmaf(sD2[r][k], sA1[r][c], g);
		atomicAdd(&G[OFF_W2 + i], g);
	}
	{
		float g = 0.f;
		for (int r = 0; r < MT; ++r) g += sD2[r][t];
		atomicAdd(&G[OFF_B2 + t], g);
	}
	for (int i = t; i < H * F; i += 64) {
		int k = i / F, c = i % F;
		float g = 0.f;
		for (int r = 0; r < MT; ++r) g = fmaf(sD1[r][k], sX[r][c], g);
		atomicAdd(&G[OFF_W1 + i], g);
	}
	{
		float g = 0.f;
		for (int r = 0; r < MT; ++r) g += sD1[r][t];
		atomicAdd(&G[OFF_B1 + t], g);
	}
}

__global__ void adam_kernel(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ m, float* __restrict__ v,
                            int np, float lr, float b1, float b2, float eps, float c1, float c2)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= np) return;
	float g = G[i];
	float mi = b1 * m[i] + (1.f - b1) * g;
	float vi = b2 * v[i] + (1.f - b2) * g * g;
	m[i] = mi; v[i] = vi;
	P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

} // namespace

} // namespace lfmm

namespace lfmm {

int mlp_forward_device(Context& c, const float* params, int n, const float* X, float* Y)
{
	if (n <= 0) return OK;
	mlp_forward_kernel<<<(n + MT - 1) / MT, 64, 0, c.stream>>>(params, n, X, Y, nullptr, nullptr);
	LFMM_CUDA(c, cudaGetLastError());
	return OK;
}

} // namespace lfmm

struct lfmm_ctx;
namespace lfmm { Context& ctx_of(lfmm_ctx* c); }

using namespace lfmm;

extern "C" {

int lfmm_mlp_forward(lfmm_ctx* h, const float* params, int n, const float* X, float* Y)
{
	if (!h || !params || !X || !Y || n < 0) return LFMM_ERR_ARG;
	Context& c = ctx_of(h);
	if (n == 0) return LFMM_OK;
	mlp_forward_kernel<<<(n + MT - 1) / MT, 64, 0, c.stream>>>(params, n, X, Y, nullptr, nullptr);
	LFMM_CUDA(c, cudaGetLastError());
	return LFMM_OK;
}

int lfmm_mlp_grad(lfmm_ctx* h, const float* params, int n, const float* X, const float* T, const float* M,
                  float* grad, float* work, float* loss)
{
	if (!h || !params || !X || !T || !M || !grad || !work || n <= 0) return LFMM_ERR_ARG;
	Context& c = ctx_of(h);
	cudaStream_t s = c.stream;
	// work: Y[n*14] A1[n*64] A2[n*64] acc[2]
	float* Y = work;
	float* A1 = Y + (size_t)n * O;
	float* A2 = A1 + (size_t)n * H;
	float* acc = A2 + (size_t)n * H;
	LFMM_CUDA(c, cudaMemsetAsync(grad, 0, sizeof(float) * NPARAM, s));
	LFMM_CUDA(c, cudaMemsetAsync(acc, 0, sizeof(float) * 2, s));
	const unsigned blocks = (n + MT - 1) / MT;
	mlp_forward_kernel<<<blocks, 64, 0, s>>>(params, n, X, Y, A1, A2);
	// mask count first, for the mean
	float hm[2] = {0, 0};
	{
		// the count of labelled outputs is needed before the gradients: a
		// first pass over M with the loss accumulator
		mlp_backward_kernel<<<blocks, 64, 0, s>>>(params, n, X, Y, A1, A2, T, M, 0.f, grad, acc);
		LFMM_CUDA(c, cudaMemcpyAsync(hm, acc, sizeof(hm), cudaMemcpyDeviceToHost, s));
		LFMM_CUDA(c, cudaStreamSynchronize(s));
	}
	const float cnt = hm[1] > 0 ? hm[1] : 1.f;
	LFMM_CUDA(c, cudaMemsetAsync(grad, 0, sizeof(float) * NPARAM, s));
	LFMM_CUDA(c, cudaMemsetAsync(acc, 0, sizeof(float) * 2, s));
	mlp_backward_kernel<<<blocks, 64, 0, s>>>(params, n, X, Y, A1, A2, T, M, 1.f / cnt, grad, acc);
	if (loss) *loss = hm[0] / cnt;
	LFMM_CUDA(c, cudaGetLastError());
	return LFMM_OK;
}

int lfmm_mlp_adam(lfmm_ctx* h, float* params, const float* grad, float* m, float* v, int step, float lr, float beta1,
                  float beta2, float eps)
{
	if (!h || !params || !grad || !m || !v || step < 1) return LFMM_ERR_ARG;
	Context& c = ctx_of(h);
	float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
	adam_kernel<<<(NPARAM + 255) / 256, 256, 0, c.stream>>>(params, grad, m, v, NPARAM, lr, beta1, beta2, eps, c1, c2);
	LFMM_CUDA(c, cudaGetLastError());
	return LFMM_OK;
}

} // extern "C"
