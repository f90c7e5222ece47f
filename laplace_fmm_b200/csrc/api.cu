// C ABI (include/lfmm.h): contexts, host/device solves, direct sums, tree
// inspection.  No exceptions cross this boundary; every entry returns a
// status and records a message for lfmm_last_error.
#include "../../include/lfmm.h"
#include "fmm2d.cuh"
#include "direct.cuh"
#include "learned.cuh"
#include "m2l_gemm.cuh"
#include <cmath>
#include <cstring>
#include <new>
#include <algorithm>
#include <cstdlib>

struct lfmm_ctx {
	lfmm::Context c;
	lfmm::DevTree tree;
	bool has_tree = false;
	// adaptive tree inspection: the V lists of every cell (global indices,
	// CSR), read from the M2L slot tables when the tree is built
	std::vector<long long> v_off, v_idx;
};

namespace lfmm {

Arena::~Arena() { release(); }

void Arena::release()
{
	for (void* p : extra_) cudaFree(p);
	extra_.clear();
	if (base_) cudaFree(base_);
	base_ = nullptr; cap_ = used_ = extra_total_ = 0;
}

void* Arena::take(size_t bytes)
{
	bytes = (bytes + 255) & ~size_t(255);
	if (used_ + bytes <= cap_) {
		void* p = base_ + used_;
		used_ += bytes;
		high_ = std::max(high_, used_ + extra_total_);
		return p;
	}
	void* p = nullptr;
	if (cudaMalloc(&p, bytes) != cudaSuccess) { cudaGetLastError(); return nullptr; }
	extra_.push_back(p);
	extra_total_ += bytes;
	high_ = std::max(high_, used_ + extra_total_);
	return p;
}

void Arena::settle()
{
	if (!extra_.empty()) {
		cudaDeviceSynchronize();
		for (void* p : extra_) cudaFree(p);
		extra_.clear();
		size_t want = high_ + (high_ >> 3);
		if (base_) cudaFree(base_);
		base_ = nullptr; cap_ = 0;
		if (cudaMalloc(&base_, want) == cudaSuccess) cap_ = want;
		else { cudaGetLastError(); base_ = nullptr; }
	}
	extra_total_ = 0;
	used_ = 0;
}

int cuda_fail(Context& ctx, cudaError_t e, const char* where)
{
	ctx.last_error = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") at " + where;
	return ERR_CUDA;
}

Context& ctx_of(lfmm_ctx* c) { return c->c; }

__global__ void latch_flags_kernel(unsigned* dev, volatile unsigned* host)
{
	const unsigned f = *dev;
	if (f) {
		*host |= f;
		*dev = 0u;
	}
}

// Stream-ordered: at the end of an asynchronous solve, move its device error
// flags into the context's pinned host word (cleared on the device, so the
// next solve starts clean); lfmm_check reports them.
int latch_flags(Context& c)
{
	latch_flags_kernel<<<1, 1, 0, c.stream>>>(c.dev_flags, c.host_flags_dev);
	LFMM_CUDA(c, cudaGetLastError());
	return OK;
}

} // namespace lfmm

using namespace lfmm;

namespace {

int resolve_order(int dim, int N, double eps)
{
	if (dim == 3) {
		eps = std::max(eps, 1.e-11);
		if (N == AUTO) return std::min(MAXN3, (int)(54.2 - 10.73 * std::sqrt(std::log(2.4 * eps) + 25.5)));
		return std::min(MAXN3, N);
	}
	if (N == AUTO) return std::min(MAXN2, (int)(-1.18 * std::log(1.65 * eps)));
	return std::min(MAXN2, N);
}

int resolve_depth(int dim, int depth, size_t n)
{
	if (depth != AUTO) return depth;
	if (dim == 3) return (int)std::max(2.0, 1 + std::log((double)n / 100.0) / std::log(8.0));
	return (int)std::max(3.0, 2 + std::log((double)n / 100.0) / std::log(4.0));
}

int check_flags(Context& c)
{
	unsigned f = 0;
	LFMM_CUDA(c, cudaMemcpyAsync(&f, c.dev_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
	LFMM_CUDA(c, cudaStreamSynchronize(c.stream));
	if (f) {
		cudaMemsetAsync(c.dev_flags, 0, sizeof(unsigned), c.stream);
		c.last_error = "device-side check failed (flags " + std::to_string(f) + ")";
		return ERR_DEVICE;
	}
	return OK;
}

void fill_stats(lfmm_stats* out, const SolveStats& s)
{
	if (!out) return;
	out->order_N = s.N; out->depth = s.depth;
	out->n_particles = s.n_particles; out->n_cells = s.n_cells; out->n_leaves = s.n_leaves;
	out->targets_num = s.targets_num; out->n_far_pairs = s.n_far_pairs; out->n_close_pairs = s.n_close_pairs;
	out->n_p2p_pairs = s.n_p2p_pairs;
	out->n_m2p = s.n_m2p; out->n_w = s.n_w; out->n_x = s.n_x;
	out->ms_tree = s.ms_tree; out->ms_upward = s.ms_upward; out->ms_m2l = s.ms_m2l; out->ms_l2l = s.ms_l2l;
	out->ms_leaves = s.ms_leaves; out->ms_total = s.ms_total;
	out->ms_m2l_kernel = s.ms_m2l_kernel; out->n_m2l_kernel = s.n_m2l_kernel;
}

int select_device(lfmm_ctx* ctx)
{
	cudaError_t e = cudaSetDevice(ctx->c.device);
	if (e != cudaSuccess) return cuda_fail(ctx->c, e, "cudaSetDevice");
	return OK;
}

// Device solve shared by the host and device entry points.
int solve_device(lfmm_ctx* ctx, int dim, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                 int N, int depth, double eps, int precision, double* pot, double* field, lfmm_stats* stats,
                 bool arena_reset, int max_leaf = 0, const int* level_N = nullptr)
{
	Context& c = ctx->c;
	if (ns == 0 && nt == 0) { c.last_error = "no particles"; return ERR_ARG; }
	if ((ns && (!src || !q)) || (nt && !tgt) || !pot || !field) { c.last_error = "null buffer"; return ERR_ARG; }
	if (precision != LFMM_PRECISION_FP64 && precision != LFMM_PRECISION_MIXED) { c.last_error = "unknown precision"; return ERR_ARG; }
	int Nr = resolve_order(dim, N, eps);
	int Dr = resolve_depth(dim, depth, ns + nt);
	if (Nr < 1) { c.last_error = "order must be >= 1"; return ERR_ARG; }
	if (Dr < 1) { c.last_error = "tree depth must be >= 1"; return ERR_ARG; }
	if (arena_reset) c.arena.reset();
	ctx->has_tree = false;
	ParticleInput in;
	in.dim = dim; in.ns = ns; in.nt = nt; in.src = src; in.srcq = q; in.tgt = tgt;
	SolveStats ss;
	int st;
	if (dim == 2 && max_leaf > 0)   // 2D: one FP64 form (the mixed request runs it too)
		st = fmm2d_solve_adaptive(c, in, Nr, Dr, max_leaf, pot, field, stats ? &ss : nullptr);
	else if (dim == 3 && (precision == LFMM_PRECISION_MIXED || max_leaf > 0))
		st = fmm3d_solve_scaled(c, in, Nr, Dr, max_leaf, precision, pot, field, stats ? &ss : nullptr, nullptr,
		                        level_N);
	else if (dim == 3)
		st = fmm3d_solve_device(c, in, Nr, Dr, pot, field, stats ? &ss : nullptr);
	else   // 2D: one FP64 form (the mixed request runs it too)
		st = fmm2d_solve_device(c, in, Nr, Dr, pot, field, stats ? &ss : nullptr);
	if (st) return st;
	fill_stats(stats, ss);
	return OK;
}

int solve_host(lfmm_ctx* ctx, int dim, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
               int N, int depth, double eps, int precision, double* pot, double* field, lfmm_stats* stats,
               int max_leaf = 0, const int* level_N = nullptr)
{
	Context& c = ctx->c;
	if (select_device(ctx)) return ERR_CUDA;
	if (ns == 0 && nt == 0) { c.last_error = "no particles"; return ERR_ARG; }
	if ((ns && (!src || !q)) || (nt && !tgt) || !pot || !field) { c.last_error = "null buffer"; return ERR_ARG; }
	c.arena.reset();
	const size_t nout = nt ? nt : ns;
	double* dsrc = static_cast<double*>(c.arena.take(sizeof(double) * dim * std::max<size_t>(ns, 1)));
	double* dq = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(ns, 1)));
	double* dtgt = static_cast<double*>(c.arena.take(sizeof(double) * dim * std::max<size_t>(nt, 1)));
	double* dpot = static_cast<double*>(c.arena.take(sizeof(double) * nout));
	double* dfld = static_cast<double*>(c.arena.take(sizeof(double) * dim * nout));
	if (!dsrc || !dq || !dtgt || !dpot || !dfld) { c.last_error = "device allocation failed"; return ERR_OOM; }
	cudaStream_t s = c.stream;
	if (ns) {
		LFMM_CUDA(c, cudaMemcpyAsync(dsrc, src, sizeof(double) * dim * ns, cudaMemcpyHostToDevice, s));
		LFMM_CUDA(c, cudaMemcpyAsync(dq, q, sizeof(double) * ns, cudaMemcpyHostToDevice, s));
	}
	if (nt) LFMM_CUDA(c, cudaMemcpyAsync(dtgt, tgt, sizeof(double) * dim * nt, cudaMemcpyHostToDevice, s));
	int st = solve_device(ctx, dim, ns, dsrc, dq, nt, dtgt, N, depth, eps, precision, dpot, dfld, stats, false,
	                      max_leaf, level_N);
	if (st == OK) {
		LFMM_CUDA(c, cudaMemcpyAsync(pot, dpot, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
		LFMM_CUDA(c, cudaMemcpyAsync(field, dfld, sizeof(double) * dim * nout, cudaMemcpyDeviceToHost, s));
		st = check_flags(c);
	}
	c.arena.settle();
	return st;
}

int direct_host(lfmm_ctx* ctx, int dim, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                double* pot, double* field)
{
	Context& c = ctx->c;
	if (select_device(ctx)) return ERR_CUDA;
	if ((ns && (!src || !q)) || (nt && (!tgt || !pot || !field))) { c.last_error = "null buffer"; return ERR_ARG; }
	c.arena.reset();
	double* dsrc = static_cast<double*>(c.arena.take(sizeof(double) * dim * std::max<size_t>(ns, 1)));
	double* dq = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(ns, 1)));
	double* dtgt = static_cast<double*>(c.arena.take(sizeof(double) * dim * std::max<size_t>(nt, 1)));
	double* dpot = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(nt, 1)));
	double* dfld = static_cast<double*>(c.arena.take(sizeof(double) * dim * std::max<size_t>(nt, 1)));
	if (!dsrc || !dq || !dtgt || !dpot || !dfld) { c.last_error = "device allocation failed"; return ERR_OOM; }
	cudaStream_t s = c.stream;
	if (ns) {
		LFMM_CUDA(c, cudaMemcpyAsync(dsrc, src, sizeof(double) * dim * ns, cudaMemcpyHostToDevice, s));
		LFMM_CUDA(c, cudaMemcpyAsync(dq, q, sizeof(double) * ns, cudaMemcpyHostToDevice, s));
	}
	if (nt) LFMM_CUDA(c, cudaMemcpyAsync(dtgt, tgt, sizeof(double) * dim * nt, cudaMemcpyHostToDevice, s));
	int st = direct_device(c, dim, ns, dsrc, dq, nt, dtgt, dpot, dfld);
	if (st == OK && nt) {
		LFMM_CUDA(c, cudaMemcpyAsync(pot, dpot, sizeof(double) * nt, cudaMemcpyDeviceToHost, s));
		LFMM_CUDA(c, cudaMemcpyAsync(field, dfld, sizeof(double) * dim * nt, cudaMemcpyDeviceToHost, s));
		LFMM_CUDA(c, cudaStreamSynchronize(s));
	}
	c.arena.settle();
	return st;
}

int need_tree(lfmm_ctx* ctx, int level)
{
	if (!ctx) return LFMM_ERR_ARG;
	if (!ctx->has_tree) { ctx->c.last_error = "no tree: call lfmm_tree_build first"; return LFMM_ERR_ARG; }
	if (level < 0 || level >= ctx->tree.depth) { ctx->c.last_error = "level out of range"; return LFMM_ERR_ARG; }
	return LFMM_OK;
}

// Inputs validated as for a solve; device pointers.
int check_inputs(Context& c, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                 const lfmm_solve_opts* o)
{
	if (!o) { c.last_error = "null options"; return ERR_ARG; }
	if (ns == 0 && nt == 0) { c.last_error = "no particles"; return ERR_ARG; }
	if ((ns && (!src || !q)) || (nt && !tgt)) { c.last_error = "null buffer"; return ERR_ARG; }
	if (o->precision != LFMM_PRECISION_FP64 && o->precision != LFMM_PRECISION_MIXED) {
		c.last_error = "unknown precision";
		return ERR_ARG;
	}
	return OK;
}

int learned_dev(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                const lfmm_solve_opts* o, const float* params, double tol, int check, double* pot, double* field,
                lfmm_learned_info* info, lfmm_stats* stats)
{
	Context& c = ctx->c;
	int st = check_inputs(c, ns, src, q, nt, tgt, o);
	if (st) return st;
	if (!pot || !field) { c.last_error = "null buffer"; return ERR_ARG; }
	ctx->has_tree = false;
	ParticleInput in;
	in.dim = 3; in.ns = ns; in.nt = nt; in.src = src; in.srcq = q; in.tgt = tgt;
	SolveStats ss;
	st = solve_learned_device(c, in, resolve_depth(3, o->tree_depth, ns + nt), o->max_leaf, o->precision, params,
	                          tol, check, pot, field, info, stats ? &ss : nullptr);
	if (st) return st;
	fill_stats(stats, ss);
	return OK;
}

// The learned order for a batch (params == nullptr: the order of opts).
struct BatchLearned {
	const float* params = nullptr;
	double tol = 0.0;
	int check = 0;
	lfmm_learned_info* info = nullptr;
};

// Batched solve on device buffers (see lfmm3d_solve_batch).
int batch_dev(lfmm_ctx* ctx, int nprob, const size_t* offsets, const double* src, const double* q,
              const lfmm_solve_opts* o, double* pot, double* field, lfmm_stats* stats,
              const BatchLearned& learned = BatchLearned())
{
	Context& c = ctx->c;
	if (!o || !offsets || nprob < 1 || !pot || !field) { c.last_error = "batch: bad arguments"; return ERR_ARG; }
	if (offsets[0] != 0) { c.last_error = "batch: offsets[0] must be 0"; return ERR_ARG; }
	size_t big = 0;
	for (int k = 0; k < nprob; ++k) {
		if (offsets[k + 1] < offsets[k]) { c.last_error = "batch: offsets must not decrease"; return ERR_ARG; }
		big = std::max(big, offsets[k + 1] - offsets[k]);
	}
	const size_t n = offsets[nprob];
	if (n == 0 || n >= 0xffffffffull) { c.last_error = "batch: total particle count out of range"; return ERR_ARG; }
	if (!src || !q) { c.last_error = "null buffer"; return ERR_ARG; }
	if (o->precision != LFMM_PRECISION_FP64 && o->precision != LFMM_PRECISION_MIXED) {
		c.last_error = "unknown precision";
		return ERR_ARG;
	}
	std::vector<uint32_t> h(nprob + 1);
	for (int k = 0; k <= nprob; ++k) h[k] = (uint32_t)offsets[k];
	uint32_t* poff = static_cast<uint32_t*>(c.arena.take(sizeof(uint32_t) * (nprob + 1)));
	if (!poff) { c.last_error = "device allocation failed"; return ERR_OOM; }
	LFMM_CUDA(c, cudaMemcpyAsync(poff, h.data(), sizeof(uint32_t) * (nprob + 1), cudaMemcpyHostToDevice, c.stream));
	ctx->has_tree = false;
	ParticleInput in;
	in.dim = 3; in.ns = n; in.nt = 0; in.src = src; in.srcq = q; in.poff = poff; in.nprob = nprob;
	SolveStats ss;
	int st = learned.params
	             ? solve_learned_batch_device(c, in, offsets, resolve_depth(3, o->tree_depth, big), o->max_leaf,
	                                          o->precision, learned.params, learned.tol, learned.check, pot, field,
	                                          learned.info, stats ? &ss : nullptr)
	             : fmm3d_solve_scaled(c, in, resolve_order(3, o->N, o->eps), resolve_depth(3, o->tree_depth, big),
	                                  o->max_leaf, o->precision, pot, field, stats ? &ss : nullptr);
	// the host copy of offsets must outlive the async copy
	LFMM_CUDA(c, cudaStreamSynchronize(c.stream));
	if (st) return st;
	fill_stats(stats, ss);
	return OK;
}

template <typename D, typename S>
int fetch(Context& c, D* dst, const S* src, size_t n)
{
	std::vector<S> tmp(n);
	if (n) LFMM_CUDA(c, cudaMemcpy(tmp.data(), src, sizeof(S) * n, cudaMemcpyDeviceToHost));
	for (size_t i = 0; i < n; ++i) dst[i] = (D)tmp[i];
	return OK;
}

} // namespace

extern "C" {

int lfmm_version(void) { return 100; }

int lfmm_create(lfmm_ctx** out, const lfmm_options* opt)
{
	if (!out) return LFMM_ERR_ARG;
	*out = nullptr;
	lfmm_ctx* ctx = new (std::nothrow) lfmm_ctx();
	if (!ctx) return LFMM_ERR_OOM;
	Context& c = ctx->c;
	if (opt) { c.device = opt->device; c.verbose = opt->verbose; c.timing = opt->timing; }
	// M2L engine (LFMM_M2L): tc (default) = tcgen05 hi/lo GEMMs on the FP32
	// levels and SIMT GEMMs elsewhere; simt = SIMT GEMMs only; rotation =
	// per-pair rotations on the plain path.  LFMM_M2L_TYPE: f16 (default) or
	// tf32, the tcgen05 M2L's operand type; LFMM_M2L_GATHER: tma (default) or
	// ldg, how the FP16 form's producers bring the sources in.
	c.m2l_engine = 3;
	if (const char* e = std::getenv("LFMM_M2L_TUNE")) c.tune_m2l = std::strcmp(e, "0") != 0;
	if (const char* e = std::getenv("LFMM_M2L_TYPE")) c.m2l_f16 = std::strcmp(e, "tf32") != 0;
	if (const char* e = std::getenv("LFMM_M2L_GATHER")) c.m2l_tma = std::strcmp(e, "ldg") != 0;
	if (const char* e = std::getenv("LFMM_M2L"))
		c.m2l_engine = std::strcmp(e, "rotation") == 0 ? 1 : (std::strcmp(e, "simt") == 0 ? 0 : 3);
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
		cudaGetLastError();
		delete ctx;
		return LFMM_ERR_CUDA;
	}
	if (c.device < 0 || c.device >= ndev || cudaSetDevice(c.device) != cudaSuccess) { delete ctx; return LFMM_ERR_ARG; }
	if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess ||
	    cudaMalloc(&c.dev_flags, sizeof(unsigned)) != cudaSuccess ||
	    cudaMemset(c.dev_flags, 0, sizeof(unsigned)) != cudaSuccess ||
	    cudaHostAlloc(&c.host_flags, sizeof(unsigned), cudaHostAllocMapped) != cudaSuccess ||
	    cudaHostGetDevicePointer(&c.host_flags_dev, c.host_flags, 0) != cudaSuccess) {
		cudaGetLastError();
		if (c.host_flags) cudaFreeHost(c.host_flags);
		if (c.dev_flags) cudaFree(c.dev_flags);
		if (c.stream) cudaStreamDestroy(c.stream);
		delete ctx;
		return LFMM_ERR_CUDA;
	}
	*c.host_flags = 0u;
	for (auto& e : c.ev) cudaEventCreate(&e);
	for (auto& e : c.kev) cudaEventCreate(&e);
	int prio_lo = 0, prio_hi = 0;
	if (cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess ||
	    cudaStreamCreateWithPriority(&c.side, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
	    cudaEventCreateWithFlags(&c.fork_ev, cudaEventDisableTiming) != cudaSuccess ||
	    cudaEventCreateWithFlags(&c.join_ev, cudaEventDisableTiming) != cudaSuccess) {
		lfmm_destroy(ctx);
		return LFMM_ERR_CUDA;
	}
	cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device);
	if (tables_build(c) != OK) {
		lfmm_destroy(ctx);
		return LFMM_ERR_CUDA;
	}
	*out = ctx;
	return LFMM_OK;
}

void lfmm_destroy(lfmm_ctx* ctx)
{
	if (!ctx) return;
	Context& c = ctx->c;
	cudaSetDevice(c.device);
	if (c.stream) cudaStreamSynchronize(c.stream);
	if (c.side) cudaStreamSynchronize(c.side);
	c.arena.release();
	for (auto& e : c.opcache) cudaFree(e.ptr);
	c.opcache.clear();
	tables_free(c.tables);
	for (auto& e : c.ev) if (e) cudaEventDestroy(e);
	for (auto& e : c.kev) if (e) cudaEventDestroy(e);
	if (c.fork_ev) cudaEventDestroy(c.fork_ev);
	if (c.join_ev) cudaEventDestroy(c.join_ev);
	if (c.dev_flags) cudaFree(c.dev_flags);
	if (c.host_flags) cudaFreeHost(c.host_flags);
	if (c.side) cudaStreamDestroy(c.side);
	if (c.stream) cudaStreamDestroy(c.stream);
	delete ctx;
}

const char* lfmm_last_error(const lfmm_ctx* ctx) { return ctx ? ctx->c.last_error.c_str() : "null context"; }

void* lfmm_stream(lfmm_ctx* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

__global__ void raise_flags_kernel(unsigned* dev, unsigned f) { atomicOr(dev, f); }

int lfmm_debug_raise_flags(lfmm_ctx* ctx, unsigned flags)
{
	if (!ctx) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	raise_flags_kernel<<<1, 1, 0, c.stream>>>(c.dev_flags, flags);
	LFMM_CUDA(c, cudaGetLastError());
	return LFMM_OK;
}

int lfmm_check(lfmm_ctx* ctx)
{
	if (!ctx) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	LFMM_CUDA(c, cudaStreamSynchronize(c.stream));
	const unsigned f = *(volatile unsigned*)c.host_flags;
	if (f) {
		*(volatile unsigned*)c.host_flags = 0u;
		c.last_error = "device-side check failed in an earlier solve (flags " + std::to_string(f) + ")";
		return LFMM_ERR_DEVICE;
	}
	return LFMM_OK;
}

int lfmm3d_solve(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt, int N,
                 int depth, double eps, int precision, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	return solve_host(ctx, 3, ns, src, q, nt, tgt, N, depth, eps, precision, pot, field, stats);
}

int lfmm3d_solve_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                        int N, int depth, double eps, int precision, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	int st = solve_device(ctx, 3, ns, src, q, nt, tgt, N, depth, eps, precision, pot, field, stats, true);
	if (st == OK) st = stats ? check_flags(ctx->c) : latch_flags(ctx->c);
	ctx->c.arena.settle();
	return st;
}

int lfmm3d_solve_ex(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                    const lfmm_solve_opts* o, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx || !o) return LFMM_ERR_ARG;
	return solve_host(ctx, 3, ns, src, q, nt, tgt, o->N, o->tree_depth, o->eps, o->precision, pot, field, stats,
	                  o->max_leaf);
}

int lfmm3d_solve_ex_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                           const lfmm_solve_opts* o, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx || !o) return LFMM_ERR_ARG;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	int st = solve_device(ctx, 3, ns, src, q, nt, tgt, o->N, o->tree_depth, o->eps, o->precision, pot, field, stats,
	                      true, o->max_leaf);
	if (st == OK) st = stats ? check_flags(ctx->c) : latch_flags(ctx->c);
	ctx->c.arena.settle();
	return st;
}

namespace {

// The per-level M2L orders of lfmm3d_solve_levels[_device], checked and
// padded to MAX_LEVELS entries (0: the solve's N).
int level_orders(lfmm_ctx* ctx, const lfmm_solve_opts* o, const int* level_N, int n_levels, int out[MAX_LEVELS])
{
	if (!o || n_levels < 0 || n_levels > MAX_LEVELS || (n_levels && !level_N)) {
		ctx->c.last_error = "per-level orders: 0 <= n_levels <= 22 entries required";
		return LFMM_ERR_ARG;
	}
	for (int L = 0; L < MAX_LEVELS; ++L) out[L] = 0;
	for (int L = 0; L < n_levels; ++L) {
		if (level_N[L] < 0) { ctx->c.last_error = "per-level orders must be >= 0"; return LFMM_ERR_ARG; }
		out[L] = level_N[L];
	}
	return LFMM_OK;
}

} // namespace

int lfmm3d_solve_levels(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                        const lfmm_solve_opts* o, const int* level_N, int n_levels, double* pot, double* field,
                        lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	int lv[MAX_LEVELS];
	if (int st = level_orders(ctx, o, level_N, n_levels, lv)) return st;
	return solve_host(ctx, 3, ns, src, q, nt, tgt, o->N, o->tree_depth, o->eps, o->precision, pot, field, stats,
	                  o->max_leaf, lv);
}

int lfmm3d_solve_levels_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt,
                               const double* tgt, const lfmm_solve_opts* o, const int* level_N, int n_levels,
                               double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	int lv[MAX_LEVELS];
	if (int st = level_orders(ctx, o, level_N, n_levels, lv)) return st;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	int st = solve_device(ctx, 3, ns, src, q, nt, tgt, o->N, o->tree_depth, o->eps, o->precision, pot, field, stats,
	                      true, o->max_leaf, lv);
	if (st == OK) st = stats ? check_flags(ctx->c) : latch_flags(ctx->c);
	ctx->c.arena.settle();
	return st;
}

namespace {

// The vector solve on device buffers.  own_arena: reset the context's arena
// before and settle it after (the device entry point); false when the host
// entry point already took its copies of the inputs from the arena.
int vector_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q3, size_t nt, const double* tgt,
                  const lfmm_solve_opts* o, double* field, lfmm_stats* stats, bool own_arena)
{
	Context& c = ctx->c;
	if (ns == 0 && nt == 0) { c.last_error = "no particles"; return LFMM_ERR_ARG; }
	if ((ns && (!src || !q3)) || (nt && !tgt) || !field) { c.last_error = "null buffer"; return LFMM_ERR_ARG; }
	if (o->precision != LFMM_PRECISION_FP64 && o->precision != LFMM_PRECISION_MIXED) {
		c.last_error = "unknown precision";
		return LFMM_ERR_ARG;
	}
	const int Nr = resolve_order(3, o->N, o->eps), Dr = resolve_depth(3, o->tree_depth, ns + nt);
	if (Nr < 1 || Dr < 1) { c.last_error = "order and tree depth must be >= 1"; return LFMM_ERR_ARG; }
	if (own_arena) c.arena.reset();
	ctx->has_tree = false;
	ParticleInput in;
	in.dim = 3; in.ns = ns; in.nt = nt; in.src = src; in.srcq = q3; in.tgt = tgt;
	SolveStats ss;
	int st = fmm3d_solve_vector(c, in, Nr, Dr, o->max_leaf, o->precision, field, stats ? &ss : nullptr);
	if (st == OK) {
		fill_stats(stats, ss);
		st = check_flags(c);
	}
	if (own_arena) c.arena.settle();
	return st;
}

} // namespace

int lfmm3d_solve_vector_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q3, size_t nt,
                               const double* tgt, const lfmm_solve_opts* o, double* field, lfmm_stats* stats)
{
	if (!ctx || !o) return LFMM_ERR_ARG;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	return vector_device(ctx, ns, src, q3, nt, tgt, o, field, stats, true);
}

int lfmm3d_solve_vector(lfmm_ctx* ctx, size_t ns, const double* src, const double* q3, size_t nt, const double* tgt,
                        const lfmm_solve_opts* o, double* field, lfmm_stats* stats)
{
	if (!ctx || !o) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	if ((ns && (!src || !q3)) || (nt && !tgt) || !field) { c.last_error = "null buffer"; return LFMM_ERR_ARG; }
	const size_t nout = nt ? nt : ns;
	// the device copies come from the context's arena (kept across the solve,
	// which then does not reset it), as in the scalar host entry points
	c.arena.reset();
	double* dsrc = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(ns, 1)));
	double* dq = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(ns, 1)));
	double* dtgt = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(nt, 1)));
	double* dfld = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(nout, 1)));
	int st = OK;
	if (!dsrc || !dq || !dtgt || !dfld) { c.last_error = "device allocation failed"; st = LFMM_ERR_OOM; }
	cudaStream_t s = c.stream;
	cudaError_t e = cudaSuccess;
	if (st == OK && ns) e = cudaMemcpyAsync(dsrc, src, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, s);
	if (st == OK && e == cudaSuccess && ns) e = cudaMemcpyAsync(dq, q3, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, s);
	if (st == OK && e == cudaSuccess && nt) e = cudaMemcpyAsync(dtgt, tgt, sizeof(double) * 3 * nt, cudaMemcpyHostToDevice, s);
	if (e != cudaSuccess) st = cuda_fail(c, e, "vector solve: copy in");
	if (st == OK) st = vector_device(ctx, ns, dsrc, dq, nt, dtgt, o, dfld, stats, false);
	if (st == OK) {
		e = cudaMemcpyAsync(field, dfld, sizeof(double) * 3 * nout, cudaMemcpyDeviceToHost, s);
		if (e == cudaSuccess) e = cudaStreamSynchronize(s);
		if (e != cudaSuccess) st = cuda_fail(c, e, "vector solve: copy out");
	}
	cudaStreamSynchronize(s);
	c.arena.settle();
	return st;
}

int lfmm2d_solve(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt, int N,
                 int depth, double eps, int precision, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	return solve_host(ctx, 2, ns, src, q, nt, tgt, N, depth, eps, precision, pot, field, stats);
}

int lfmm2d_solve_ex(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                    const lfmm_solve_opts* o, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx || !o) return LFMM_ERR_ARG;
	if (o->max_leaf < 0) { ctx->c.last_error = "max_leaf must be >= 0"; return LFMM_ERR_ARG; }
	return solve_host(ctx, 2, ns, src, q, nt, tgt, o->N, o->tree_depth, o->eps, o->precision, pot, field, stats,
	                  o->max_leaf);
}

int lfmm2d_solve_ex_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                           const lfmm_solve_opts* o, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx || !o) return LFMM_ERR_ARG;
	if (o->max_leaf < 0) { ctx->c.last_error = "max_leaf must be >= 0"; return LFMM_ERR_ARG; }
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	int st = solve_device(ctx, 2, ns, src, q, nt, tgt, o->N, o->tree_depth, o->eps, o->precision, pot, field, stats,
	                      true, o->max_leaf);
	if (st == OK) st = stats ? check_flags(ctx->c) : latch_flags(ctx->c);
	ctx->c.arena.settle();
	return st;
}

int lfmm2d_solve_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                        int N, int depth, double eps, int precision, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	int st = solve_device(ctx, 2, ns, src, q, nt, tgt, N, depth, eps, precision, pot, field, stats, true);
	if (st == OK) st = stats ? check_flags(ctx->c) : latch_flags(ctx->c);
	ctx->c.arena.settle();
	return st;
}

int lfmm3d_direct(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                  double* pot, double* field)
{
	if (!ctx) return LFMM_ERR_ARG;
	return direct_host(ctx, 3, ns, src, q, nt, tgt, pot, field);
}

int lfmm2d_direct(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                  double* pot, double* field)
{
	if (!ctx) return LFMM_ERR_ARG;
	return direct_host(ctx, 2, ns, src, q, nt, tgt, pot, field);
}

int lfmm3d_direct_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                         double* pot, double* field)
{
	if (!ctx) return LFMM_ERR_ARG;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	ctx->c.arena.reset();
	int st = direct_device(ctx->c, 3, ns, src, q, nt, tgt, pot, field);
	ctx->c.arena.settle();
	return st;
}

int lfmm2d_direct_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                         double* pot, double* field)
{
	if (!ctx) return LFMM_ERR_ARG;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	ctx->c.arena.reset();
	int st = direct_device(ctx->c, 2, ns, src, q, nt, tgt, pot, field);
	ctx->c.arena.settle();
	return st;
}

// ---- batched solves ----------------------------------------------------------

int lfmm3d_solve_batch_device(lfmm_ctx* ctx, int nprob, const size_t* offsets, const double* src, const double* q,
                              const lfmm_solve_opts* o, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	ctx->c.arena.reset();
	int st = batch_dev(ctx, nprob, offsets, src, q, o, pot, field, stats);
	if (st == OK) st = check_flags(ctx->c);
	ctx->c.arena.settle();
	return st;
}

int lfmm3d_solve_batch(lfmm_ctx* ctx, int nprob, const size_t* offsets, const double* src, const double* q,
                       const lfmm_solve_opts* o, double* pot, double* field, lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	if (!offsets || nprob < 1 || !src || !q || !pot || !field) { c.last_error = "batch: bad arguments"; return LFMM_ERR_ARG; }
	const size_t n = offsets[nprob];
	c.arena.reset();
	double* dsrc = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(n, 1)));
	double* dq = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(n, 1)));
	double* dpot = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(n, 1)));
	double* dfld = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(n, 1)));
	if (!dsrc || !dq || !dpot || !dfld) { c.last_error = "device allocation failed"; return LFMM_ERR_OOM; }
	cudaStream_t s = c.stream;
	if (n) {
		LFMM_CUDA(c, cudaMemcpyAsync(dsrc, src, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
		LFMM_CUDA(c, cudaMemcpyAsync(dq, q, sizeof(double) * n, cudaMemcpyHostToDevice, s));
	}
	int st = batch_dev(ctx, nprob, offsets, dsrc, dq, o, dpot, dfld, stats);
	if (st == OK) {
		LFMM_CUDA(c, cudaMemcpyAsync(pot, dpot, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
		LFMM_CUDA(c, cudaMemcpyAsync(field, dfld, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s));
		st = check_flags(c);
	}
	c.arena.settle();
	return st;
}

int lfmm3d_solve_batch_learned_device(lfmm_ctx* ctx, int nprob, const size_t* offsets, const double* src,
                                      const double* q, const lfmm_solve_opts* o, const float* params, double tol,
                                      int check_targets, double* pot, double* field, lfmm_learned_info* info,
                                      lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	if (!params) { ctx->c.last_error = "learned batch: null params"; return LFMM_ERR_ARG; }
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	ctx->c.arena.reset();
	BatchLearned bl;
	bl.params = params; bl.tol = tol; bl.check = check_targets; bl.info = info;
	int st = batch_dev(ctx, nprob, offsets, src, q, o, pot, field, stats, bl);
	if (st == OK) st = check_flags(ctx->c);
	ctx->c.arena.settle();
	return st;
}

// ---- learned order -----------------------------------------------------------

int lfmm3d_solve_learned_device(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt,
                                const double* tgt, const lfmm_solve_opts* o, const float* params, double tol,
                                int check_targets, double* pot, double* field, lfmm_learned_info* info,
                                lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	ctx->c.arena.reset();
	int st = learned_dev(ctx, ns, src, q, nt, tgt, o, params, tol, check_targets, pot, field, info, stats);
	if (st == OK) st = check_flags(ctx->c);
	ctx->c.arena.settle();
	return st;
}

int lfmm3d_solve_learned(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                         const lfmm_solve_opts* o, const float* params, double tol, int check_targets, double* pot,
                         double* field, lfmm_learned_info* info, lfmm_stats* stats)
{
	if (!ctx) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	int st = check_inputs(c, ns, src, q, nt, tgt, o);
	if (st) return st;
	if (!pot || !field) { c.last_error = "null buffer"; return LFMM_ERR_ARG; }
	c.arena.reset();
	const size_t nout = nt ? nt : ns;
	double* dsrc = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(ns, 1)));
	double* dq = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(ns, 1)));
	double* dtgt = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(nt, 1)));
	double* dpot = static_cast<double*>(c.arena.take(sizeof(double) * nout));
	double* dfld = static_cast<double*>(c.arena.take(sizeof(double) * 3 * nout));
	if (!dsrc || !dq || !dtgt || !dpot || !dfld) { c.last_error = "device allocation failed"; return LFMM_ERR_OOM; }
	cudaStream_t s = c.stream;
	if (ns) {
		LFMM_CUDA(c, cudaMemcpyAsync(dsrc, src, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, s));
		LFMM_CUDA(c, cudaMemcpyAsync(dq, q, sizeof(double) * ns, cudaMemcpyHostToDevice, s));
	}
	if (nt) LFMM_CUDA(c, cudaMemcpyAsync(dtgt, tgt, sizeof(double) * 3 * nt, cudaMemcpyHostToDevice, s));
	st = learned_dev(ctx, ns, dsrc, dq, nt, dtgt, o, params, tol, check_targets, dpot, dfld, info, stats);
	if (st == OK) {
		LFMM_CUDA(c, cudaMemcpyAsync(pot, dpot, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
		LFMM_CUDA(c, cudaMemcpyAsync(field, dfld, sizeof(double) * 3 * nout, cudaMemcpyDeviceToHost, s));
		st = check_flags(c);
	}
	c.arena.settle();
	return st;
}

int lfmm3d_features(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                    const lfmm_solve_opts* o, float* feats, size_t cap, int* leaf_of, size_t* n_leaves)
{
	if (!ctx) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	int st = check_inputs(c, ns, src, q, nt, tgt, o);
	if (st) return st;
	c.arena.reset();
	ctx->has_tree = false;
	double* dsrc = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(ns, 1)));
	double* dq = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(ns, 1)));
	double* dtgt = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(nt, 1)));
	if (!dsrc || !dq || !dtgt) { c.last_error = "device allocation failed"; return LFMM_ERR_OOM; }
	cudaStream_t s = c.stream;
	if (ns) {
		LFMM_CUDA(c, cudaMemcpyAsync(dsrc, src, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, s));
		LFMM_CUDA(c, cudaMemcpyAsync(dq, q, sizeof(double) * ns, cudaMemcpyHostToDevice, s));
	}
	if (nt) LFMM_CUDA(c, cudaMemcpyAsync(dtgt, tgt, sizeof(double) * 3 * nt, cudaMemcpyHostToDevice, s));
	ParticleInput in;
	in.dim = 3; in.ns = ns; in.nt = nt; in.src = dsrc; in.srcq = dq; in.tgt = dtgt;
	st = features_tree(c, in, resolve_depth(3, o->tree_depth, ns + nt), o->max_leaf, feats, cap,
	                   reinterpret_cast<int32_t*>(leaf_of), n_leaves);
	if (st == OK) st = check_flags(c);
	c.arena.settle();
	return st;
}

int lfmm3d_leaf_features(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                         int depth, int N, const int* cand, int K, float* feats)
{
	if (!ctx || !cand || !feats || K < 1 || K > LEAF_CAND_MAX) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	if (ns == 0 && nt == 0) { c.last_error = "no particles"; return LFMM_ERR_ARG; }
	if ((ns && (!src || !q)) || (nt && !tgt)) { c.last_error = "null buffer"; return LFMM_ERR_ARG; }
	c.arena.reset();
	ctx->has_tree = false;
	double* dsrc = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(ns, 1)));
	double* dq = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(ns, 1)));
	double* dtgt = static_cast<double*>(c.arena.take(sizeof(double) * 3 * std::max<size_t>(nt, 1)));
	if (!dsrc || !dq || !dtgt) { c.last_error = "device allocation failed"; return LFMM_ERR_OOM; }
	cudaStream_t s = c.stream;
	if (ns) {
		LFMM_CUDA(c, cudaMemcpyAsync(dsrc, src, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, s));
		LFMM_CUDA(c, cudaMemcpyAsync(dq, q, sizeof(double) * ns, cudaMemcpyHostToDevice, s));
	}
	if (nt) LFMM_CUDA(c, cudaMemcpyAsync(dtgt, tgt, sizeof(double) * 3 * nt, cudaMemcpyHostToDevice, s));
	ParticleInput in;
	in.dim = 3; in.ns = ns; in.nt = nt; in.src = dsrc; in.srcq = dq; in.tgt = dtgt;
	int st = leaf_features_host(c, in, resolve_depth(3, depth, ns + nt), N, cand, K, feats);
	if (st == OK) st = check_flags(c);
	c.arena.settle();
	return st;
}

// ---- tree inspection -------------------------------------------------------

int lfmm_tree_build(lfmm_ctx* ctx, int dim, size_t ns, const double* src, const double* q, size_t nt,
                    const double* tgt, int depth, size_t* level_sizes, size_t* targets_num)
{
	if (!ctx || (dim != 2 && dim != 3)) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	if (ns == 0 && nt == 0) { c.last_error = "no particles"; return LFMM_ERR_ARG; }
	c.arena.reset();
	ctx->has_tree = false;
	double* dsrc = static_cast<double*>(c.arena.take(sizeof(double) * dim * std::max<size_t>(ns, 1)));
	double* dq = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(ns, 1)));
	double* dtgt = static_cast<double*>(c.arena.take(sizeof(double) * dim * std::max<size_t>(nt, 1)));
	if (!dsrc || !dq || !dtgt) { c.last_error = "device allocation failed"; return LFMM_ERR_OOM; }
	cudaStream_t s = c.stream;
	if (ns) {
		LFMM_CUDA(c, cudaMemcpyAsync(dsrc, src, sizeof(double) * dim * ns, cudaMemcpyHostToDevice, s));
		if (q) LFMM_CUDA(c, cudaMemcpyAsync(dq, q, sizeof(double) * ns, cudaMemcpyHostToDevice, s));
		else LFMM_CUDA(c, cudaMemsetAsync(dq, 0, sizeof(double) * ns, s));
	}
	if (nt) LFMM_CUDA(c, cudaMemcpyAsync(dtgt, tgt, sizeof(double) * dim * nt, cudaMemcpyHostToDevice, s));
	ParticleInput in;
	in.dim = dim; in.ns = ns; in.nt = nt; in.src = dsrc; in.srcq = dq; in.tgt = dtgt;
	int st = tree_build(c, in, resolve_depth(dim, depth, ns + nt), ctx->tree);
	if (st) return st;
	st = check_flags(c);
	if (st) return st;
	ctx->has_tree = true;
	for (int L = 0; L < ctx->tree.depth && level_sizes; ++L) level_sizes[L] = ctx->tree.lsize[L];
	if (targets_num) *targets_num = ctx->tree.targets_num;
	return LFMM_OK;
}

int lfmm_tree_level(lfmm_ctx* ctx, int L, unsigned long long* code, long long* beg, long long* end, long long* tbeg,
                    long long* tend, long long* parent, double* center)
{
	int st = need_tree(ctx, L);
	if (st) return st;
	Context& c = ctx->c;
	DevTree& t = ctx->tree;
	size_t o = t.loff[L], m = t.lsize[L];
	if (code && (st = fetch(c, code, t.code + o, m))) return st;
	if (beg && (st = fetch(c, beg, t.beg + o, m))) return st;
	if (end && (st = fetch(c, end, t.end + o, m))) return st;
	if (tbeg && (st = fetch(c, tbeg, t.tbeg + o, m))) return st;
	if (tend && (st = fetch(c, tend, t.tend + o, m))) return st;
	if (parent && (st = fetch(c, parent, t.parent + o, m))) return st;
	if (center) {
		std::vector<double> x(m), y(m), z(m);
		if ((st = fetch(c, x.data(), t.cx + o, m)) || (st = fetch(c, y.data(), t.cy + o, m))) return st;
		if (t.dim == 3 && (st = fetch(c, z.data(), t.cz + o, m))) return st;
		for (size_t i = 0; i < m; ++i) {
			center[t.dim * i] = x[i]; center[t.dim * i + 1] = y[i];
			if (t.dim == 3) center[3 * i + 2] = z[i];
		}
	}
	return LFMM_OK;
}

int lfmm_tree_list_sizes(lfmm_ctx* ctx, int L, long long* n_close, long long* n_far)
{
	int st = need_tree(ctx, L);
	if (st) return st;
	Context& c = ctx->c;
	DevTree& t = ctx->tree;
	size_t o = t.loff[L], m = t.lsize[L];
	if (n_close && (st = fetch(c, n_close, t.close_cnt + o, m))) return st;
	if (n_far && (st = fetch(c, n_far, t.far_cnt + o, m))) return st;
	return LFMM_OK;
}

int lfmm_tree_lists(lfmm_ctx* ctx, int L, long long* close, long long* far)
{
	int st = need_tree(ctx, L);
	if (st) return st;
	Context& c = ctx->c;
	DevTree& t = ctx->tree;
	size_t o = t.loff[L], m = t.lsize[L];
	std::vector<int32_t> cnt(m);
	if ((st = fetch(c, cnt.data(), t.close_cnt + o, m))) return st;
	if (close) {
		std::vector<int32_t> idx(m * t.close_stride);
		if ((st = fetch(c, idx.data(), t.close_idx + o * t.close_stride, m * t.close_stride))) return st;
		size_t a = 0;
		for (size_t i = 0; i < m; ++i)
			for (int k = 0; k < cnt[i]; ++k) close[a++] = idx[i * t.close_stride + k];
	}
	if (far && L >= 2) {
		std::vector<int32_t> fc(m);
		if ((st = fetch(c, fc.data(), t.far_cnt + o, m))) return st;
		size_t total = 0;
		for (auto v : fc) total += (size_t)v;
		uint32_t* off = static_cast<uint32_t*>(c.arena.take(sizeof(uint32_t) * (m + 1)));
		int32_t* idx = static_cast<int32_t*>(c.arena.take(sizeof(int32_t) * (total + 1)));
		if (!off || !idx) { c.last_error = "device allocation failed"; return LFMM_ERR_OOM; }
		if ((st = tree_far_lists(c, t, L, off, idx, total))) return st;
		if ((st = check_flags(c))) return st;
		if ((st = fetch(c, far, idx, total))) return st;
	}
	return LFMM_OK;
}

int lfmm_tree_positions(lfmm_ctx* ctx, long long* positions)
{
	int st = need_tree(ctx, 0);
	if (st) return st;
	Context& c = ctx->c;
	DevTree& t = ctx->tree;
	std::vector<uint32_t> orig(t.n);
	if ((st = fetch(c, orig.data(), t.orig, t.n))) return st;
	for (size_t s = 0; s < t.n; ++s) positions[orig[s]] = (long long)s;
	return LFMM_OK;
}

namespace {

int tree_build_adaptive_host(lfmm_ctx* ctx, int dim, size_t ns, const double* src, const double* q, size_t nt,
                             const double* tgt, int depth, int max_leaf, size_t* n_cells, size_t* n_leaves,
                             size_t* list_sizes)
{
	if (!ctx || max_leaf < 0) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	if (ns == 0 && nt == 0) { c.last_error = "no particles"; return LFMM_ERR_ARG; }
	if ((ns && !src) || (nt && !tgt)) { c.last_error = "null buffer"; return LFMM_ERR_ARG; }
	c.arena.reset();
	ctx->has_tree = false;
	ctx->v_off.clear();
	ctx->v_idx.clear();
	double* dsrc = static_cast<double*>(c.arena.take(sizeof(double) * dim * std::max<size_t>(ns, 1)));
	double* dq = static_cast<double*>(c.arena.take(sizeof(double) * std::max<size_t>(ns, 1)));
	double* dtgt = static_cast<double*>(c.arena.take(sizeof(double) * dim * std::max<size_t>(nt, 1)));
	if (!dsrc || !dq || !dtgt) { c.last_error = "device allocation failed"; return LFMM_ERR_OOM; }
	cudaStream_t s = c.stream;
	if (ns) {
		LFMM_CUDA(c, cudaMemcpyAsync(dsrc, src, sizeof(double) * dim * ns, cudaMemcpyHostToDevice, s));
		if (q) LFMM_CUDA(c, cudaMemcpyAsync(dq, q, sizeof(double) * ns, cudaMemcpyHostToDevice, s));
		else LFMM_CUDA(c, cudaMemsetAsync(dq, 0, sizeof(double) * ns, s));
	}
	if (nt) LFMM_CUDA(c, cudaMemcpyAsync(dtgt, tgt, sizeof(double) * dim * nt, cudaMemcpyHostToDevice, s));
	ParticleInput in;
	in.dim = dim; in.ns = ns; in.nt = nt; in.src = dsrc; in.srcq = dq; in.tgt = dtgt;
	DevTree& t = ctx->tree;
	int st = tree_build_adaptive(c, in, resolve_depth(dim, depth, ns + nt), max_leaf, t);
	if (st || (st = check_flags(c))) return st;
	// V lists: the M2L slot table of every level (what the solver's M2L reads)
	ctx->v_off.assign(t.ncells + 1, 0);
	std::vector<std::vector<long long>> per(t.ncells);
	for (int L = 2; L < t.depth; ++L) {
		if (!t.lsize[L]) continue;
		const size_t mark = c.arena.mark();
		M2LPlan plan;
		if ((st = dim == 3 ? m2l_plan_build(c, t, L, plan) : m2l_plan_build2d(c, t, L, plan)) ||
		    (st = check_flags(c)))
			return st;
		const int slots = dim == 3 ? M2L_SLOTS : M2L_SLOTS2;
		std::vector<int32_t> vt(t.lsize[L] * (size_t)slots);
		if ((st = fetch(c, vt.data(), plan.vtab, vt.size()))) return st;
		c.arena.rewind(mark);
		for (size_t k = 0; k < t.lsize[L]; ++k)
			for (int sl = 0; sl < slots; ++sl) {
				const int32_t v = vt[k * slots + sl];
				if (v >= 0) per[t.loff[L] + k].push_back((long long)(t.loff[L] + (size_t)v));
			}
	}
	for (size_t g = 0; g < t.ncells; ++g) {
		ctx->v_off[g + 1] = ctx->v_off[g] + (long long)per[g].size();
		ctx->v_idx.insert(ctx->v_idx.end(), per[g].begin(), per[g].end());
	}
	ctx->has_tree = true;
	if (n_cells) *n_cells = t.ncells;
	if (n_leaves) *n_leaves = t.nleaves;
	if (list_sizes) {
		list_sizes[0] = t.n_u; list_sizes[1] = t.n_w; list_sizes[2] = t.n_x; list_sizes[3] = ctx->v_idx.size();
	}
	return LFMM_OK;
}

} // namespace

int lfmm_tree_build_adaptive(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt,
                             const double* tgt, int depth, int max_leaf, size_t* n_cells, size_t* n_leaves,
                             size_t* list_sizes)
{
	return tree_build_adaptive_host(ctx, 3, ns, src, q, nt, tgt, depth, max_leaf, n_cells, n_leaves, list_sizes);
}

int lfmm2d_tree_build_adaptive(lfmm_ctx* ctx, size_t ns, const double* src, const double* q, size_t nt,
                               const double* tgt, int depth, int max_leaf, size_t* n_cells, size_t* n_leaves,
                               size_t* list_sizes)
{
	return tree_build_adaptive_host(ctx, 2, ns, src, q, nt, tgt, depth, max_leaf, n_cells, n_leaves, list_sizes);
}

int lfmm_tree_adaptive_cells(lfmm_ctx* ctx, int* level, unsigned long long* code, long long* parent,
                             long long* pbeg, long long* pend, long long* send, unsigned char* is_leaf,
                             long long* leaves, long long* positions)
{
	if (!ctx) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	DevTree& t = ctx->tree;
	if (!ctx->has_tree || !t.adaptive) { c.last_error = "no adaptive tree: call lfmm_tree_build_adaptive first"; return LFMM_ERR_ARG; }
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	const size_t C = t.ncells;
	int st;
	std::vector<uint8_t> lv(C);
	if ((st = fetch(c, lv.data(), t.lev, C))) return st;
	if (level) for (size_t g = 0; g < C; ++g) level[g] = lv[g];
	if (code && (st = fetch(c, code, t.code, C))) return st;
	if (parent) {
		std::vector<int32_t> p(C);
		if ((st = fetch(c, p.data(), t.parent, C))) return st;
		for (size_t g = 0; g < C; ++g) parent[g] = lv[g] ? (long long)(t.loff[lv[g] - 1] + (size_t)p[g]) : -1;
	}
	if (pbeg && (st = fetch(c, pbeg, t.pbeg, C))) return st;
	if (pend && (st = fetch(c, pend, t.pend, C))) return st;
	if (send && (st = fetch(c, send, t.send, C))) return st;
	if (is_leaf && (st = fetch(c, is_leaf, t.is_leaf, C))) return st;
	if (leaves && (st = fetch(c, leaves, t.leaves, t.nleaves))) return st;
	if (positions) {
		std::vector<uint32_t> orig(t.n);
		if ((st = fetch(c, orig.data(), t.orig, t.n))) return st;
		for (size_t p = 0; p < t.n; ++p) positions[orig[p]] = (long long)p;
	}
	return LFMM_OK;
}

int lfmm_tree_adaptive_lists(lfmm_ctx* ctx, int kind, long long* off, long long* idx)
{
	if (!ctx || kind < 0 || kind > 3) return LFMM_ERR_ARG;
	Context& c = ctx->c;
	DevTree& t = ctx->tree;
	if (!ctx->has_tree || !t.adaptive) { c.last_error = "no adaptive tree: call lfmm_tree_build_adaptive first"; return LFMM_ERR_ARG; }
	if (select_device(ctx)) return LFMM_ERR_CUDA;
	if (kind == 3) {
		if (off) std::copy(ctx->v_off.begin(), ctx->v_off.end(), off);
		if (idx) std::copy(ctx->v_idx.begin(), ctx->v_idx.end(), idx);
		return LFMM_OK;
	}
	const uint32_t* o = kind == 0 ? t.u_off : kind == 1 ? t.w_off : t.x_off;
	const int32_t* ix = kind == 0 ? t.u_idx : kind == 1 ? t.w_idx : t.x_idx;
	const size_t rows = kind == 2 ? t.ncells : t.nleaves;
	const size_t total = kind == 0 ? t.n_u : kind == 1 ? t.n_w : t.n_x;
	int st;
	if (off && (st = fetch(c, off, o, rows + 1))) return st;
	if (idx && (st = fetch(c, idx, ix, total))) return st;
	return LFMM_OK;
}

int lfmm_wignerd_slot(lfmm_ctx* ctx, int slot, double* theta, double* d)
{
	if (!ctx) return LFMM_ERR_ARG;
	Tables& T = ctx->c.tables;
	if (slot < 0 || slot >= T.d.n_dslots) return T.d.n_dslots;
	if (theta) *theta = T.theta_of_slot[slot];
	if (d) {
		cudaError_t e = cudaMemcpy(d, T.d.dmat + (size_t)slot * dsize(MAXN3), sizeof(double) * dsize(MAXN3),
		                           cudaMemcpyDeviceToHost);
		if (e != cudaSuccess) return cuda_fail(ctx->c, e, "lfmm_wignerd_slot");
	}
	return T.d.n_dslots;
}

} // extern "C"
