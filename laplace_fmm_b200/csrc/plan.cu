// Solve plans: one geometry, many charge vectors.  The adaptive tree of the
// positions (or the forest of a batch of independent problems) is built once, every cache the solve uses is warmed (operators,
// constants, the M2L autotuner), and the FMM passes are captured in a CUDA
// graph on the context's stream; each execution copies the new charges in,
// scatters them into tree order and launches the graph.  No counterpart in
// the reference, which rebuilds the tree on every solve
// (cpu/multipole3d.cpp:1340).
#include "../../include/lfmm.h"
#include "fmm3d.cuh"
#include "m2l_gemm.cuh"
#include <algorithm>
#include <cmath>
#include <new>

struct lfmm_ctx;
namespace lfmm { Context& ctx_of(lfmm_ctx* c); int latch_flags(Context& c); }

struct lfmm_plan {
	lfmm_ctx* ctx = nullptr;
	lfmm::Arena arena;                 // the plan's device memory (tree, expansions, scratch)
	lfmm::DevTree tree;
	int N = 0, precision = 0;
	size_t n = 0;
	int nprob = 1;                     // > 1: a batch plan (forest of independent problems)
	double* q_in = nullptr;            // charges in input order (graph input)
	double* pot = nullptr;             // outputs in input order (graph output)
	double* fld = nullptr;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	std::vector<void*> pinned;         // operator cache entries the graph reads
};

namespace lfmm {

namespace {

__global__ void scatter_charges_kernel(DevTree t, const double* __restrict__ q_in)
{
	const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (s < t.n) t.q[s] = q_in[t.orig[s]];
}

// Take the plan's buffers (before the tree, so both passes lay them out alike).
int take_io(Context& c, lfmm_plan* p)
{
	p->q_in = static_cast<double*>(c.arena.take(sizeof(double) * p->n));
	p->pot = static_cast<double*>(c.arena.take(sizeof(double) * p->n));
	p->fld = static_cast<double*>(c.arena.take(sizeof(double) * 3 * p->n));
	if (!p->q_in || !p->pot || !p->fld) { c.last_error = "plan: allocation failed"; return ERR_OOM; }
	return OK;
}

// Build the plan in the context with the plan's arena swapped in.  hoff
// (host, nprob + 1 entries) for a batch plan, else null.
int build(Context& c, lfmm_plan* p, const double* src, const double* q, int depth, int max_leaf, const size_t* hoff)
{
	ParticleInput in;
	in.dim = 3; in.ns = p->n; in.nt = 0; in.src = src; in.srcq = q;
	std::vector<uint32_t> h;
	if (hoff) {
		h.resize(p->nprob + 1);
		for (int k = 0; k <= p->nprob; ++k) h[k] = (uint32_t)hoff[k];
	}
	// the forest's device offsets, taken (and re-taken in pass 2) before the
	// tree so that both passes lay the arena out alike
	auto take_offsets = [&]() -> int {
		if (!hoff) return OK;
		uint32_t* poff = static_cast<uint32_t*>(c.arena.take(sizeof(uint32_t) * (p->nprob + 1)));
		if (!poff) { c.last_error = "plan: allocation failed"; return ERR_OOM; }
		LFMM_CUDA(c, cudaMemcpyAsync(poff, h.data(), sizeof(uint32_t) * (p->nprob + 1), cudaMemcpyHostToDevice,
		                             c.stream));
		in.poff = poff;
		in.nprob = p->nprob;
		return OK;
	};
	// pass 1: sizes the arena and warms every cache (operators, autotuner)
	int st = take_io(c, p);
	if (st || (st = take_offsets())) return st;
	if ((st = tree_build_adaptive(c, in, depth, max_leaf, p->tree))) return st;
	if ((st = fmm3d_scaled_on_tree(c, p->tree, p->N, p->precision, p->pot, p->fld, nullptr))) return st;
	c.arena.settle();                  // one block of the high-water size
	// pass 2: the final layout, one more warm solve, then the capture replays it
	c.arena.reset();
	if ((st = take_io(c, p)) || (st = take_offsets())) return st;
	LFMM_CUDA(c, cudaMemcpyAsync(p->q_in, q, sizeof(double) * p->n, cudaMemcpyDeviceToDevice, c.stream));
	if ((st = tree_build_adaptive(c, in, depth, max_leaf, p->tree))) return st;
	const size_t mark = c.arena.mark();
	const size_t chunks = c.arena.chunks();
	if ((st = fmm3d_scaled_on_tree(c, p->tree, p->N, p->precision, p->pot, p->fld, nullptr))) return st;
	LFMM_CUDA(c, cudaStreamSynchronize(c.stream));
	if (c.arena.chunks() != chunks) { c.last_error = "plan: the solve outgrew its memory"; return ERR_OOM; }
	c.arena.rewind(mark);
	const int timing = c.timing;
	c.timing = 0;
	LFMM_CUDA(c, cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
	scatter_charges_kernel<<<div_up(p->n, 256), 256, 0, c.stream>>>(p->tree, p->q_in);
	st = fmm3d_scaled_on_tree(c, p->tree, p->N, p->precision, p->pot, p->fld, nullptr);
	cudaGraph_t g = nullptr;
	const cudaError_t ec = cudaStreamEndCapture(c.stream, &g);   // always end the capture
	c.timing = timing;
	if (st) { if (g) cudaGraphDestroy(g); return st; }
	if (ec != cudaSuccess) return cuda_fail(c, ec, "cudaStreamEndCapture");
	p->graph = g;
	if (c.arena.chunks() != chunks) { c.last_error = "plan: the captured solve outgrew its memory"; return ERR_OOM; }
	LFMM_CUDA(c, cudaGraphInstantiate(&p->exec, p->graph, 0));
	// the graph reads the cached operators: keep them from eviction
	for (auto& e : c.opcache) { ++e.pinned; p->pinned.push_back(e.ptr); }
	return OK;
}

} // namespace

} // namespace lfmm

using namespace lfmm;

namespace {

void unpin_and_delete(lfmm_plan* p)
{
	Context& c = ctx_of(p->ctx);
	cudaSetDevice(c.device);
	cudaStreamSynchronize(c.stream);
	if (p->exec) cudaGraphExecDestroy(p->exec);
	if (p->graph) cudaGraphDestroy(p->graph);
	for (void* ptr : p->pinned)
		for (auto& e : c.opcache)
			if (e.ptr == ptr && e.pinned > 0) --e.pinned;
	delete p;                          // the arena frees the plan's memory
}

} // namespace

extern "C" {

int lfmm3d_plan_create(lfmm_ctx* h, size_t n_src, const double* src_xyz, const double* src_q,
                       const lfmm_solve_opts* o, lfmm_plan** out)
{
	if (!h || !o || !out || !src_xyz || !src_q || n_src == 0) return LFMM_ERR_ARG;
	*out = nullptr;
	Context& c = ctx_of(h);
	if (o->max_leaf < 0 || (o->precision != LFMM_PRECISION_FP64 && o->precision != LFMM_PRECISION_MIXED)) {
		c.last_error = "plan: bad options";
		return LFMM_ERR_ARG;
	}
	if (o->N == LFMM_AUTO || o->N < 1 || !m2l_gemm_supported(o->N)) {
		c.last_error = "plan: N must be given, 1 <= N <= 18";
		return LFMM_ERR_ARG;
	}
	const int depth = o->tree_depth != LFMM_AUTO
	                      ? o->tree_depth
	                      : (int)std::max(2.0, 1 + std::log((double)n_src / 100.0) / std::log(8.0));
	cudaError_t e = cudaSetDevice(c.device);
	if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
	lfmm_plan* p = new (std::nothrow) lfmm_plan();
	if (!p) return LFMM_ERR_OOM;
	p->ctx = h; p->n = n_src; p->N = o->N; p->precision = o->precision;
	c.arena.swap(p->arena);
	int st = build(c, p, src_xyz, src_q, depth, o->max_leaf, nullptr);
	c.arena.swap(p->arena);
	if (st) {
		unpin_and_delete(p);
		return st;
	}
	*out = p;
	return LFMM_OK;
}

int lfmm3d_plan_create_batch(lfmm_ctx* h, int n_prob, const size_t* offsets, const double* src_xyz,
                             const double* src_q, const lfmm_solve_opts* o, lfmm_plan** out)
{
	if (!h || !o || !out || !offsets || !src_xyz || !src_q || n_prob < 1) return LFMM_ERR_ARG;
	*out = nullptr;
	Context& c = ctx_of(h);
	if (offsets[0] != 0) { c.last_error = "batch plan: offsets[0] must be 0"; return LFMM_ERR_ARG; }
	size_t big = 0;
	for (int k = 0; k < n_prob; ++k) {
		if (offsets[k + 1] < offsets[k]) { c.last_error = "batch plan: offsets must not decrease"; return LFMM_ERR_ARG; }
		big = std::max(big, offsets[k + 1] - offsets[k]);
	}
	const size_t n = offsets[n_prob];
	if (n == 0 || n >= 0xffffffffull) { c.last_error = "batch plan: total particle count out of range"; return LFMM_ERR_ARG; }
	if (o->max_leaf < 0 || o->max_leaf == LFMM_AUTO ||
	    (o->precision != LFMM_PRECISION_FP64 && o->precision != LFMM_PRECISION_MIXED)) {
		c.last_error = "batch plan: bad options (max_leaf must be given)";
		return LFMM_ERR_ARG;
	}
	if (o->N == LFMM_AUTO || o->N < 1 || !m2l_gemm_supported(o->N)) {
		c.last_error = "batch plan: N must be given, 1 <= N <= 18";
		return LFMM_ERR_ARG;
	}
	const int depth = o->tree_depth != LFMM_AUTO
	                      ? o->tree_depth
	                      : (int)std::max(2.0, 1 + std::log((double)big / 100.0) / std::log(8.0));
	cudaError_t e = cudaSetDevice(c.device);
	if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
	lfmm_plan* p = new (std::nothrow) lfmm_plan();
	if (!p) return LFMM_ERR_OOM;
	p->ctx = h; p->n = n; p->N = o->N; p->precision = o->precision; p->nprob = n_prob;
	c.arena.swap(p->arena);
	int st = build(c, p, src_xyz, src_q, depth, o->max_leaf, offsets);
	c.arena.swap(p->arena);
	if (st) {
		unpin_and_delete(p);
		return st;
	}
	*out = p;
	return LFMM_OK;
}

int lfmm3d_plan_execute(lfmm_plan* p, const double* src_q, double* pot, double* field)
{
	if (!p || !src_q || !pot || !field) return LFMM_ERR_ARG;
	Context& c = ctx_of(p->ctx);
	cudaError_t e = cudaSetDevice(c.device);
	if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
	LFMM_CUDA(c, cudaMemcpyAsync(p->q_in, src_q, sizeof(double) * p->n, cudaMemcpyDeviceToDevice, c.stream));
	LFMM_CUDA(c, cudaGraphLaunch(p->exec, c.stream));
	LFMM_CUDA(c, cudaMemcpyAsync(pot, p->pot, sizeof(double) * p->n, cudaMemcpyDeviceToDevice, c.stream));
	LFMM_CUDA(c, cudaMemcpyAsync(field, p->fld, sizeof(double) * 3 * p->n, cudaMemcpyDeviceToDevice, c.stream));
	return latch_flags(c);
}

void lfmm3d_plan_destroy(lfmm_plan* p)
{
	if (p) unpin_and_delete(p);
}

} // extern "C"
