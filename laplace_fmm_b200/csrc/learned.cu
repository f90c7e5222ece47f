// Learned order selection (no counterpart in the reference, which derives one
// order from eps by a fixed formula, cpu/multipole3d.cpp:1328-1331).
//
//   tree (adaptive form) -> per-leaf features (16) -> MLP (mlp.cu) -> log10
//   of each leaf's error at p = 4, 6, ..., 14 -> predicted rel-L2 of the
//   potential per order = sqrt(sum_leaf w 10^(2 y) / sum_leaf w), w = the
//   leaf's output particles -> the lowest order p (interpolated between the
//   six) whose prediction is within the tolerance -> one solve at N = p + 1 on
//   the same tree -> optional sampled check against the FP64 direct sum; a
//   solve that misses the tolerance is rerun at the fixed fallback order.
#include "learned.cuh"
#include "direct.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

namespace lfmm {

namespace {

constexpr int NF = LFMM_MLP_IN, NO = LFMM_MLP_OUT;
constexpr int FB_N = 15;            // fallback order (degrees): the highest the scaled solver runs
constexpr double LEARNED_MARGIN = 1.0;   // the calibrated prediction must be within tol

__device__ __forceinline__ float lg(double x) { return (float)log10(x); }

__device__ __forceinline__ void cell_coords(uint64_t code, int* c)
{ c[0] = (int)compact3(code >> 2); c[1] = (int)compact3(code >> 1); c[2] = (int)compact3(code); }

// Far-field strength of the cells of level L (>= 2): over the cell's V list
// (children of the parent and of its close cells that are not adjacent, the
// same enumeration as the M2L slot table), fs = sum sqrt(n) / h and
// fl = sum n / h, n = particles of the source cell, h = the cell size.
__global__ void far_strength_kernel(DevTree t, int L, double* __restrict__ fs, double* __restrict__ fl)
{
	const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= t.lsize[L]) return;
	const size_t off = t.loff[L], poff = t.loff[L - 1];
	int me[3];
	cell_coords(t.code[off + c], me);
	const int32_t p = t.parent[off + c];
	const int npc = t.close_cnt[poff + p];
	const int32_t* pl = t.close_idx + (poff + p) * t.close_stride;
	double s1 = 0.0, s2 = 0.0;
	for (int e = 0; e <= npc; ++e) {
		const int32_t pn = e < npc ? pl[e] : p;
		for (uint32_t k = t.beg[poff + pn]; k < t.end[poff + pn]; ++k) {
			if (k == c) continue;
			int o[3];
			cell_coords(t.code[off + k], o);
			if (max(max(abs(o[0] - me[0]), abs(o[1] - me[1])), abs(o[2] - me[2])) <= 1) continue;
			const double n = (double)(t.pend[off + k] - t.pbeg[off + k]);
			s1 += sqrt(n); s2 += n;
		}
	}
	const double h = cell_size(t, off + c);
	fs[off + c] = s1 / h;
	fl[off + c] = s2 / h;
}

// fs, fl += the parent's (accumulated) values: the far field of a cell's
// whole ancestry
__global__ void accumulate_down_kernel(DevTree t, int L, double* __restrict__ fs, double* __restrict__ fl)
{
	const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= t.lsize[L]) return;
	const size_t g = t.loff[L] + c, gp = t.loff[L - 1] + (size_t)t.parent[g];
	fs[g] += fs[gp];
	fl[g] += fl[gp];
}

// One warp per leaf: features[li][16] and the leaf's output count w[li].
__global__ void features_kernel(DevTree t, size_t n_total, const double* __restrict__ fs,
                                const double* __restrict__ fl, float* __restrict__ feats, float* __restrict__ w)
{
	const size_t li = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (li >= t.nleaves) return;
	const size_t g = (size_t)t.leaves[li];
	const int L = t.lev[g];
	const double h = cell_size(t, g);
	const double cx = t.cx[g], cy = t.cy[g], cz = t.cz[g];
	double aq = 0, dx = 0, dy = 0, dz = 0, r2 = 0, rmax = 0;
	for (uint32_t s = t.pbeg[g] + lane; s < t.pend[g]; s += 32) {
		const double q = t.q[s], x = t.x[s] - cx, y = t.y[s] - cy, z = t.z[s] - cz;
		const double rr = x * x + y * y + z * z;
		aq += fabs(q); dx += q * x; dy += q * y; dz += q * z; r2 += rr;
		rmax = fmax(rmax, rr);
	}
	unsigned long long near = 0;
	for (uint32_t e = t.u_off[li] + lane; e < t.u_off[li + 1]; e += 32) {
		const size_t k = (size_t)t.u_idx[e];
		near += t.pend[k] - t.pbeg[k];
	}
	for (int o = 16; o; o >>= 1) {
		aq += __shfl_xor_sync(0xffffffffu, aq, o);
		dx += __shfl_xor_sync(0xffffffffu, dx, o); dy += __shfl_xor_sync(0xffffffffu, dy, o);
		dz += __shfl_xor_sync(0xffffffffu, dz, o); r2 += __shfl_xor_sync(0xffffffffu, r2, o);
		rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
		near += __shfl_xor_sync(0xffffffffu, near, o);
	}
	if (lane != 0) return;
	const double np = (double)(t.pend[g] - t.pbeg[g]);
	double anc = (double)t.far_cnt[g], npar = np;
	size_t A = g;
	for (int l = L; l > 0; --l) {
		A = t.loff[l - 1] + (size_t)t.parent[A];
		anc += (double)t.far_cnt[A];
		if (l == L) npar = (double)(t.pend[A] - t.pbeg[A]);
	}
	float* f = feats + li * NF;
	f[0] = lg(1.0 + np);
	f[1] = lg(fs[g] + 1e-30);
	f[2] = (float)L / (float)max(t.depth, 1);
	f[3] = lg(1.0 + (double)(t.u_off[li + 1] - t.u_off[li]));
	f[4] = lg(1.0 + (double)(t.w_off[li + 1] - t.w_off[li]));
	f[5] = lg(1.0 + (double)(t.x_off[g + 1] - t.x_off[g]));
	f[6] = lg(1.0 + (double)t.far_cnt[g]);
	f[7] = lg(1.0 + anc);
	f[8] = lg(aq + 1e-30);
	f[9] = lg(fl[g] + 1e-30);
	f[10] = np > 0 ? (float)(sqrt(r2 / np) / h) : 0.f;
	f[11] = (float)(sqrt(rmax) / h);
	f[12] = lg(1.0 + npar);
	f[13] = lg(1.0 + (double)n_total);
	f[14] = lg(1.0 + (double)near);
	f[15] = lg(sqrt(dx * dx + dy * dy + dz * dz) / (h * aq + 1e-300) + 1e-12);
	w[li] = (float)(t.tend[g] - t.tbeg[g]);
}

// leaf_of[input index] = leaf (inputs: targets first, then sources)
__global__ void leaf_of_kernel(DevTree t, int32_t* __restrict__ leaf_of)
{
	const size_t li = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (li >= t.nleaves) return;
	const size_t g = (size_t)t.leaves[li];
	for (uint32_t s = t.pbeg[g] + lane; s < t.pend[g]; s += 32) leaf_of[t.orig[s]] = (int32_t)li;
}

// acc[k] += w 10^(2 y[k]) over the leaves, acc[NO] += w (FP64 atomics)
__global__ void predict_reduce_kernel(const float* __restrict__ Y, const float* __restrict__ w, size_t nl,
                                      double* __restrict__ acc)
{
	double a[NO + 1] = {};
	for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += (size_t)gridDim.x * blockDim.x) {
		const double wi = w[i];
#pragma unroll
		for (int k = 0; k < NO; ++k) a[k] += wi * exp10(2.0 * fmin((double)Y[i * NO + k], 10.0));
		a[NO] += wi;
	}
#pragma unroll
	for (int k = 0; k <= NO; ++k) {
		double v = a[k];
		for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
		if ((threadIdx.x & 31) == 0) atomicAdd(&acc[k], v);
	}
}

// Sampled check: positions of the sampled outputs (every stride-th output).
__global__ void sample_points_kernel(const double* __restrict__ pts, size_t stride, size_t m, double* __restrict__ out)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m) return;
	for (int d = 0; d < 3; ++d) out[3 * i + d] = pts[3 * (i * stride) + d];
}

// acc: [0] sum (pot - direct)^2, [1] sum (direct - self)^2, [2] sum |dfield|^2,
// [3] sum |field|^2 over the sampled outputs.  q: the outputs' charges (null
// in target mode: no self term).
__global__ void check_kernel(const double* __restrict__ pot, const double* __restrict__ fld, size_t stride, size_t m,
                             const double* __restrict__ q, const double* __restrict__ ep,
                             const double* __restrict__ ef, double* __restrict__ acc)
{
	double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
	for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
		const size_t j = i * stride;
		const double self = q ? q[j] / FORCE_EPS : 0.0;
		const double d = pot[j] - ep[i], r = ep[i] - self;
		a0 += d * d; a1 += r * r;
		for (int k = 0; k < 3; ++k) {
			const double e = fld[3 * j + k] - ef[3 * i + k];
			a2 += e * e; a3 += ef[3 * i + k] * ef[3 * i + k];
		}
	}
	for (int o = 16; o; o >>= 1) {
		a0 += __shfl_xor_sync(0xffffffffu, a0, o); a1 += __shfl_xor_sync(0xffffffffu, a1, o);
		a2 += __shfl_xor_sync(0xffffffffu, a2, o); a3 += __shfl_xor_sync(0xffffffffu, a3, o);
	}
	if ((threadIdx.x & 31) == 0) {
		atomicAdd(&acc[0], a0); atomicAdd(&acc[1], a1); atomicAdd(&acc[2], a2); atomicAdd(&acc[3], a3);
	}
}

// acc[0] += sum over the samples of (direct potential - self term)^2
__global__ void rms_kernel(const double* __restrict__ ep, size_t stride, size_t m, const double* __restrict__ q,
                           double* __restrict__ acc)
{
	double a = 0;
	for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
		const double r = ep[i] - (q ? q[i * stride] / FORCE_EPS : 0.0);
		a += r * r;
	}
	for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
	if ((threadIdx.x & 31) == 0) atomicAdd(acc, a);
}

// Forest: acc[prob * (NO + 1) + k] += w 10^(2 y[k]) per leaf, by the leaf's problem
__global__ void predict_reduce_forest_kernel(DevTree t, const float* __restrict__ Y, const float* __restrict__ w,
                                             double* __restrict__ acc)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= t.nleaves) return;
	const size_t g = (size_t)t.leaves[i];
	const size_t prob = (size_t)(t.code[g] >> (3 * t.lev[g]));
	const double wi = w[i];
	for (int k = 0; k < NO; ++k) atomicAdd(&acc[prob * (NO + 1) + k], wi * exp10(2.0 * fmin((double)Y[i * NO + k], 10.0)));
	atomicAdd(&acc[prob * (NO + 1) + NO], wi);
}

__global__ void gather_points_kernel(const double* __restrict__ pts, const uint32_t* __restrict__ idx, size_t m,
                                     double* __restrict__ out)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m) return;
	for (int d = 0; d < 3; ++d) out[3 * i + d] = pts[3 * (size_t)idx[i] + d];
}

// Forest samples: acc[4 prob + 0..3] += (pot - direct)^2, (direct - self)^2,
// |dfield|^2, |field|^2; pot == nullptr: only the reference sums (the RMS).
__global__ void check_forest_kernel(const double* __restrict__ pot, const double* __restrict__ fld,
                                    const uint32_t* __restrict__ idx, const int32_t* __restrict__ prob, size_t m,
                                    const double* __restrict__ q, const double* __restrict__ ep,
                                    const double* __restrict__ ef, double* __restrict__ acc)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m) return;
	const size_t j = idx[i];
	double* a = acc + 4 * (size_t)prob[i];
	const double r = ep[i] - q[j] / FORCE_EPS;
	atomicAdd(&a[1], r * r);
	double f2 = 0.0;
	for (int k = 0; k < 3; ++k) f2 += ef[3 * i + k] * ef[3 * i + k];
	atomicAdd(&a[3], f2);
	if (!pot) return;
	const double d = pot[j] - ep[i];
	atomicAdd(&a[0], d * d);
	double e2 = 0.0;
	for (int k = 0; k < 3; ++k) { const double e = fld[3 * j + k] - ef[3 * i + k]; e2 += e * e; }
	atomicAdd(&a[2], e2);
}

template <typename T>
T* take(Context& ctx, size_t n) { return static_cast<T*>(ctx.arena.take(sizeof(T) * std::max<size_t>(n, 1))); }

int features_device(Context& ctx, const DevTree& t, float* feats, float* w)
{
	const size_t nl = t.nleaves;
	if (nl == 0) return OK;
	cudaStream_t s = ctx.stream;
	double* fs = take<double>(ctx, t.ncells);
	double* fl = take<double>(ctx, t.ncells);
	if (!fs || !fl) { ctx.last_error = "features: allocation failed"; return ERR_OOM; }
	LFMM_CUDA(ctx, cudaMemsetAsync(fs, 0, sizeof(double) * t.ncells, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(fl, 0, sizeof(double) * t.ncells, s));
	for (int L = 2; L < t.depth; ++L)
		if (t.lsize[L]) far_strength_kernel<<<div_up(t.lsize[L], 128), 128, 0, s>>>(t, L, fs, fl);
	for (int L = 1; L < t.depth; ++L)
		if (t.lsize[L]) accumulate_down_kernel<<<div_up(t.lsize[L], 256), 256, 0, s>>>(t, L, fs, fl);
	features_kernel<<<div_up(nl * 32, 256), 256, 0, s>>>(t, t.n, fs, fl, feats, w);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

// log10 of the predicted rel-L2 at order p (4 <= p <= 14), interpolated
// between the network's six orders.
double predicted_log10(const double* e, int p)
{
	const double x = (p - 4) / 2.0;
	const int k = std::min(4, (int)x);
	const double f = x - k;
	return e[k] * (1.0 - f) + e[k + 1] * f;
}

// Features -> MLP -> the lowest order whose predicted rel-L2 (absolute
// per-leaf errors aggregated over the leaves, divided by the RMS potential
// rms) is within tol * margin (N = p + 1), or the fallback order when none
// is.  Synchronises (reads six sums).
// The network's per-order error sums over the leaves (device, NO + 1
// doubles): features, forward pass and reduction, launched on the stream.
int learned_predict_launch(Context& ctx, const DevTree& t, const float* params, double*& acc)
{
	const size_t nl = t.nleaves;
	float* feats = take<float>(ctx, nl * NF);
	float* w = take<float>(ctx, nl);
	float* Y = take<float>(ctx, nl * NO);
	acc = take<double>(ctx, NO + 1);
	if (!feats || !w || !Y || !acc) { ctx.last_error = "learned order: allocation failed"; return ERR_OOM; }
	int st = features_device(ctx, t, feats, w);
	if (st) return st;
	if ((st = mlp_forward_device(ctx, params, (int)nl, feats, Y))) return st;
	LFMM_CUDA(ctx, cudaMemsetAsync(acc, 0, sizeof(double) * (NO + 1), ctx.stream));
	const unsigned blocks = (unsigned)std::min<size_t>(div_up(std::max<size_t>(nl, 1), 256), 4 * (size_t)ctx.num_sms);
	predict_reduce_kernel<<<blocks, 256, 0, ctx.stream>>>(Y, w, nl, acc);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

// The order from the sums of learned_predict_launch and the RMS of the
// sampled potential.  Synchronises.
int learned_pick(Context& ctx, const double* acc, double tol, double rms, int& N, double& pred)
{
	double h[NO + 1];
	LFMM_CUDA(ctx, cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, ctx.stream));
	LFMM_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
	double e[NO];
	const double lrms = std::log10(std::max(rms, 1e-300));
	for (int k = 0; k < NO; ++k) e[k] = 0.5 * std::log10(std::max(h[k], 1e-300) / std::max(h[NO], 1.0)) - lrms;
	const double target = std::log10(tol * LEARNED_MARGIN);
	N = FB_N;
	pred = std::pow(10.0, predicted_log10(e, 14));
	for (int p = 4; p <= 14; ++p) {
		const double lp = predicted_log10(e, p);
		if (lp <= target) { N = p + 1; pred = std::pow(10.0, lp); break; }
	}
	return OK;
}

// The FP64 direct sum at m outputs spread evenly through the output range:
// positions sp, potential ep and field ef at them, and the sum of squares of
// the potential without the self term in acc[0].  Launched on the context's
// lowest-priority side stream, forked from the main stream, so that it runs
// beside the tree build and the order prediction; samples_join makes the
// main stream wait for it and returns the RMS.
struct Samples {
	size_t m = 0, stride = 1;
	double *sp = nullptr, *ep = nullptr, *ef = nullptr, *acc = nullptr;
};

// Swaps the context's stream for the side stream while in scope.
struct OnSideStream {
	Context& c;
	cudaStream_t main;
	explicit OnSideStream(Context& c_) : c(c_), main(c_.stream) { c.stream = c.side; }
	~OnSideStream() { c.stream = main; }
};

int direct_samples_launch(Context& ctx, const ParticleInput& in, size_t m, Samples& S)
{
	const size_t n_out = in.nt ? in.nt : in.ns;
	S.m = std::min(m, n_out);
	S.stride = n_out / S.m;
	const double* pts = in.nt ? in.tgt : in.src;
	S.sp = take<double>(ctx, 3 * S.m);
	S.ep = take<double>(ctx, S.m);
	S.ef = take<double>(ctx, 3 * S.m);
	S.acc = take<double>(ctx, 4);
	if (!S.sp || !S.ep || !S.ef || !S.acc) { ctx.last_error = "sampled check: allocation failed"; return ERR_OOM; }
	LFMM_CUDA(ctx, cudaEventRecord(ctx.fork_ev, ctx.stream));
	LFMM_CUDA(ctx, cudaStreamWaitEvent(ctx.side, ctx.fork_ev, 0));
	int st = OK;
	{
		OnSideStream on_side(ctx);
		cudaStream_t s = ctx.stream;
		sample_points_kernel<<<div_up(S.m, 256), 256, 0, s>>>(pts, S.stride, S.m, S.sp);
		st = direct_device(ctx, 3, in.ns, in.src, in.srcq, S.m, S.sp, S.ep, S.ef, /*fast=*/true);
		if (st == OK) {
			// the RMS: the check against the direct sum itself (pot = direct, zero error)
			cudaError_t e = cudaMemsetAsync(S.acc, 0, sizeof(double) * 4, s);
			if (e == cudaSuccess) {
				rms_kernel<<<(unsigned)std::min<size_t>(div_up(S.m, 256), 64), 256, 0, s>>>(
					S.ep, S.stride, S.m, in.nt ? nullptr : in.srcq, S.acc);
				e = cudaGetLastError();
			}
			if (e == cudaSuccess) e = cudaEventRecord(ctx.join_ev, s);
			if (e != cudaSuccess) st = cuda_fail(ctx, e, "sampled direct sums");
		}
	}
	if (st) cudaStreamSynchronize(ctx.side);   // nothing of it outlives the failed solve
	return st;
}

int samples_join(Context& ctx, const Samples& S, double* rms)
{
	LFMM_CUDA(ctx, cudaStreamWaitEvent(ctx.stream, ctx.join_ev, 0));
	double h;
	LFMM_CUDA(ctx, cudaMemcpyAsync(&h, S.acc, sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
	LFMM_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
	*rms = std::sqrt(h / (double)S.m);
	return OK;
}

// rel-L2 of the potential (self term removed) and of the field at the samples.
int sampled_error(Context& ctx, const ParticleInput& in, const Samples& S, const double* pot, const double* field,
                  double out[2])
{
	cudaStream_t s = ctx.stream;
	LFMM_CUDA(ctx, cudaMemsetAsync(S.acc, 0, sizeof(double) * 4, s));
	check_kernel<<<(unsigned)std::min<size_t>(div_up(S.m, 256), 64), 256, 0, s>>>(
		pot, field, S.stride, S.m, in.nt ? nullptr : in.srcq, S.ep, S.ef, S.acc);
	double h[4];
	LFMM_CUDA(ctx, cudaMemcpyAsync(h, S.acc, sizeof(h), cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	out[0] = std::sqrt(h[0] / std::max(h[1], 1e-300));
	out[1] = std::sqrt(h[2] / std::max(h[3], 1e-300));
	return OK;
}

} // namespace

int solve_learned_device(Context& ctx, const ParticleInput& in, int depth, int max_leaf, int precision,
                         const float* params, double tol, int check_targets, double* pot, double* field,
                         lfmm_learned_info* info, SolveStats* stats)
{
	if (!params || !(tol > 0.0)) { ctx.last_error = "learned solve: params and tol > 0 required"; return ERR_ARG; }
	if (max_leaf < 0) { ctx.last_error = "learned solve: negative max_leaf"; return ERR_ARG; }
	if (check_targets < 1) {
		ctx.last_error = "learned solve: check_targets >= 1 required (the sampled direct sum normalises the "
		                 "prediction and judges the result)";
		return ERR_ARG;
	}
	cudaStream_t s = ctx.stream;
	const bool timing = ctx.timing != 0;
	ctx.kev_used = 0;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[0], s));
	Samples S;
	int st = direct_samples_launch(ctx, in, (size_t)check_targets, S);
	if (st) return st;
	DevTree t;
	double* pacc = nullptr;
	double rms = 0.0;
	if ((st = tree_build_adaptive(ctx, in, depth, max_leaf, t)) ||
	    (timing && (st = cudaEventRecord(ctx.ev[1], s) == cudaSuccess ? OK : ERR_CUDA)) ||
	    (st = learned_predict_launch(ctx, t, params, pacc)) || (st = samples_join(ctx, S, &rms))) {
		cudaStreamSynchronize(ctx.side);
		return st;
	}
	int N = FB_N;
	double pred = 0.0;
	if ((st = learned_pick(ctx, pacc, tol, rms, N, pred))) return st;
	lfmm_learned_info li{};
	li.predicted_N = N;
	li.predicted_error = pred;
	if ((st = fmm3d_scaled_on_tree(ctx, t, N, precision, pot, field, stats))) return st;
	double e[2];
	if ((st = sampled_error(ctx, in, S, pot, field, e))) return st;
	if (e[0] > tol && N < FB_N) {
		// the fixed-order fallback judges and replaces a prediction that missed
		N = FB_N;
		li.fallback = 1;
		if ((st = fmm3d_scaled_on_tree(ctx, t, N, precision, pot, field, stats))) return st;
		if ((st = sampled_error(ctx, in, S, pot, field, e))) return st;
	}
	if (e[0] > tol && precision == LFMM_PRECISION_MIXED) {
		// the mixed form cannot reach tol even at N = 15: the FP64 form
		if ((st = fmm3d_scaled_on_tree(ctx, t, FB_N, LFMM_PRECISION_FP64, pot, field, stats))) return st;
		if ((st = sampled_error(ctx, in, S, pot, field, e))) return st;
		N = FB_N;
		li.fp64_resolved = 1;
	}
	li.checked_error = e[0];
	li.checked_error_field = e[1];
	li.order_N = N;
	if (info) *info = li;
	return OK;
}

// Batched learned solve (forest of in.nprob problems, hoff: host offsets).
int solve_learned_batch_device(Context& ctx, const ParticleInput& in, const size_t* hoff, int depth, int max_leaf,
                               int precision, const float* params, double tol, int check_targets, double* pot,
                               double* field, lfmm_learned_info* info, SolveStats* stats)
{
	if (!params || !(tol > 0.0) || check_targets < 1 || max_leaf < 0) {
		ctx.last_error = "learned batch: params, tol > 0, check_targets >= 1 required";
		return ERR_ARG;
	}
	const int P = in.nprob;
	cudaStream_t s = ctx.stream;
	DevTree t;
	int st = tree_build_adaptive(ctx, in, depth, max_leaf, t);
	if (st) return st;
	// samples: up to check_targets outputs of every problem, evenly spaced
	std::vector<uint32_t> hidx;
	std::vector<int32_t> hprob;
	std::vector<size_t> soff(P + 1, 0);
	for (int k = 0; k < P; ++k) {
		const size_t nk = hoff[k + 1] - hoff[k];
		const size_t mk = std::min<size_t>((size_t)check_targets, nk);
		for (size_t j = 0; j < mk; ++j) { hidx.push_back((uint32_t)(hoff[k] + j * (nk / mk))); hprob.push_back(k); }
		soff[k + 1] = hidx.size();
	}
	const size_t m = hidx.size();
	uint32_t* idx = take<uint32_t>(ctx, m);
	int32_t* prob = take<int32_t>(ctx, m);
	double* sp = take<double>(ctx, 3 * m);
	double* ep = take<double>(ctx, m);
	double* ef = take<double>(ctx, 3 * m);
	double* acc = take<double>(ctx, 4 * (size_t)P);
	double* accp = take<double>(ctx, (size_t)(NO + 1) * P);
	if (!idx || !prob || !sp || !ep || !ef || !acc || !accp) { ctx.last_error = "learned batch: allocation failed"; return ERR_OOM; }
	LFMM_CUDA(ctx, cudaMemcpyAsync(idx, hidx.data(), sizeof(uint32_t) * m, cudaMemcpyHostToDevice, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(prob, hprob.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice, s));
	gather_points_kernel<<<div_up(m, 256), 256, 0, s>>>(in.src, idx, m, sp);
	for (int k = 0; k < P; ++k) {
		const size_t mk = soff[k + 1] - soff[k];
		if (!mk) continue;
		if ((st = direct_device(ctx, 3, hoff[k + 1] - hoff[k], in.src + 3 * hoff[k], in.srcq + hoff[k], mk,
		                        sp + 3 * soff[k], ep + soff[k], ef + 3 * soff[k], /*fast=*/true)))
			return st;
	}
	LFMM_CUDA(ctx, cudaMemsetAsync(acc, 0, sizeof(double) * 4 * P, s));
	check_forest_kernel<<<div_up(m, 256), 256, 0, s>>>(nullptr, nullptr, idx, prob, m, in.srcq, ep, ef, acc);
	// per-problem predictions
	const size_t nl = t.nleaves;
	float* feats = take<float>(ctx, nl * NF);
	float* w = take<float>(ctx, nl);
	float* Y = take<float>(ctx, nl * NO);
	if (!feats || !w || !Y) { ctx.last_error = "learned batch: allocation failed"; return ERR_OOM; }
	if ((st = features_device(ctx, t, feats, w))) return st;
	if ((st = mlp_forward_device(ctx, params, (int)nl, feats, Y))) return st;
	LFMM_CUDA(ctx, cudaMemsetAsync(accp, 0, sizeof(double) * (NO + 1) * P, s));
	predict_reduce_forest_kernel<<<div_up(std::max<size_t>(nl, 1), 256), 256, 0, s>>>(t, Y, w, accp);
	std::vector<double> ha(4 * (size_t)P), hp((size_t)(NO + 1) * P);
	LFMM_CUDA(ctx, cudaMemcpyAsync(ha.data(), acc, sizeof(double) * ha.size(), cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(hp.data(), accp, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	int N = 5;
	double pred = 0.0;
	for (int k = 0; k < P; ++k) {
		const size_t mk = soff[k + 1] - soff[k];
		if (!mk || hp[(size_t)k * (NO + 1) + NO] <= 0.0) continue;
		const double rms = std::sqrt(ha[4 * (size_t)k + 1] / (double)mk);
		if (!(rms > 0.0)) continue;    // nothing but self terms (one particle): no far-field error
		double e[NO];
		for (int j = 0; j < NO; ++j)
			e[j] = 0.5 * std::log10(std::max(hp[(size_t)k * (NO + 1) + j], 1e-300) / hp[(size_t)k * (NO + 1) + NO]) -
			       std::log10(std::max(rms, 1e-300));
		int Nk = FB_N;
		double pk = std::pow(10.0, predicted_log10(e, 14));
		for (int p = 4; p <= 14; ++p) {
			const double lp = predicted_log10(e, p);
			if (lp <= std::log10(tol * LEARNED_MARGIN)) { Nk = p + 1; pk = std::pow(10.0, lp); break; }
		}
		if (Nk > N || (Nk == N && pk > pred)) { N = Nk; pred = pk; }
	}
	lfmm_learned_info li{};
	li.predicted_N = N;
	li.predicted_error = pred;
	for (int pass = 0; pass < 2; ++pass) {
		if ((st = fmm3d_scaled_on_tree(ctx, t, N, precision, pot, field, stats))) return st;
		LFMM_CUDA(ctx, cudaMemsetAsync(acc, 0, sizeof(double) * 4 * P, s));
		check_forest_kernel<<<div_up(m, 256), 256, 0, s>>>(pot, field, idx, prob, m, in.srcq, ep, ef, acc);
		LFMM_CUDA(ctx, cudaMemcpyAsync(ha.data(), acc, sizeof(double) * ha.size(), cudaMemcpyDeviceToHost, s));
		LFMM_CUDA(ctx, cudaStreamSynchronize(s));
		double ep_max = 0.0, ef_max = 0.0;
		for (int k = 0; k < P; ++k) {
			if (soff[k + 1] == soff[k]) continue;
			ep_max = std::max(ep_max, std::sqrt(ha[4 * (size_t)k] / std::max(ha[4 * (size_t)k + 1], 1e-300)));
			ef_max = std::max(ef_max, std::sqrt(ha[4 * (size_t)k + 2] / std::max(ha[4 * (size_t)k + 3], 1e-300)));
		}
		li.checked_error = ep_max;
		li.checked_error_field = ef_max;
		if (ep_max <= tol || N >= FB_N) break;
		N = FB_N;                      // the fixed-order fallback for the whole batch
		li.fallback = 1;
	}
	if (precision == LFMM_PRECISION_MIXED && li.checked_error > tol) {
		// problems the mixed form cannot bring within tol even at N = 15:
		// each rerun alone in the FP64 form, into its slice of the outputs
		for (int k = 0; k < P; ++k) {
			if (soff[k + 1] == soff[k]) continue;
			if (std::sqrt(ha[4 * (size_t)k] / std::max(ha[4 * (size_t)k + 1], 1e-300)) <= tol) continue;
			ParticleInput pk;
			pk.dim = 3; pk.ns = hoff[k + 1] - hoff[k]; pk.nt = 0;
			pk.src = in.src + 3 * hoff[k]; pk.srcq = in.srcq + hoff[k];
			const size_t mark = ctx.arena.mark();
			st = fmm3d_solve_scaled(ctx, pk, FB_N, depth, max_leaf, LFMM_PRECISION_FP64, pot + hoff[k], field + 3 * hoff[k],
			                        nullptr, nullptr);
			ctx.arena.rewind(mark);
			if (st) return st;
			++li.fp64_resolved;
		}
		if (li.fp64_resolved) {
			LFMM_CUDA(ctx, cudaMemsetAsync(acc, 0, sizeof(double) * 4 * P, s));
			check_forest_kernel<<<div_up(m, 256), 256, 0, s>>>(pot, field, idx, prob, m, in.srcq, ep, ef, acc);
			LFMM_CUDA(ctx, cudaMemcpyAsync(ha.data(), acc, sizeof(double) * ha.size(), cudaMemcpyDeviceToHost, s));
			LFMM_CUDA(ctx, cudaStreamSynchronize(s));
			double ep_max = 0.0, ef_max = 0.0;
			for (int k = 0; k < P; ++k) {
				if (soff[k + 1] == soff[k]) continue;
				ep_max = std::max(ep_max, std::sqrt(ha[4 * (size_t)k] / std::max(ha[4 * (size_t)k + 1], 1e-300)));
				ef_max = std::max(ef_max, std::sqrt(ha[4 * (size_t)k + 2] / std::max(ha[4 * (size_t)k + 3], 1e-300)));
			}
			li.checked_error = ep_max;
			li.checked_error_field = ef_max;
		}
	}
	li.order_N = N;
	if (info) *info = li;
	return OK;
}

int features_tree(Context& ctx, const ParticleInput& in, int depth, int max_leaf, float* feats_host, size_t cap,
                  int32_t* leaf_of_host, size_t* n_leaves)
{
	DevTree t;
	int st = tree_build_adaptive(ctx, in, depth, max_leaf, t);
	if (st) return st;
	const size_t nl = t.nleaves;
	if (n_leaves) *n_leaves = nl;
	if (nl > cap) { ctx.last_error = "features: more leaves than the buffer holds"; return ERR_ARG; }
	float* feats = take<float>(ctx, nl * NF);
	float* w = take<float>(ctx, nl);
	int32_t* lo = take<int32_t>(ctx, t.n);
	if (!feats || !w || !lo) { ctx.last_error = "features: allocation failed"; return ERR_OOM; }
	if ((st = features_device(ctx, t, feats, w))) return st;
	cudaStream_t s = ctx.stream;
	if (feats_host && nl) LFMM_CUDA(ctx, cudaMemcpyAsync(feats_host, feats, sizeof(float) * nl * NF, cudaMemcpyDeviceToHost, s));
	if (leaf_of_host) {
		if (nl) leaf_of_kernel<<<div_up(nl * 32, 256), 256, 0, s>>>(t, lo);
		LFMM_CUDA(ctx, cudaGetLastError());
		LFMM_CUDA(ctx, cudaMemcpyAsync(leaf_of_host, lo, sizeof(int32_t) * t.n, cudaMemcpyDeviceToHost, s));
	}
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	return OK;
}

} // namespace lfmm
