// 3D FP64 direct sum whose source-chunk scratch is a file-scope device array,
// so a call allocates no device memory.  Same kernels and chunk rule as
// lfmm3d_direct_device (direct.cu); only the scratch differs.
//
// The array is one per device, shared by every context of the process on that
// device: calls that overlap in time on one device race on it.  Nothing in it
// needs to start at zero (each partial is written before it is read).  Its
// address is looked up once per device (cudaGetSymbolAddress, which may load
// the module) on the first call with that device current; the same first call
// also loads both kernels a call can launch (the chunk reduction runs only
// when the sources are split), so that no later call loads code, which can
// allocate.  A cudaDeviceReset invalidates the cached address.
#include "../../include/lfmm.h"
#include "direct.cuh"
#include <mutex>

namespace {

constexpr size_t SCRATCH_DOUBLES = LFMM_DIRECT_NOALLOC_SCRATCH_BYTES / sizeof(double);
constexpr int MAX_DEVICES = 64;

__device__ __align__(256) double g_direct_scratch[SCRATCH_DOUBLES];

std::mutex g_scratch_mu;
double* g_scratch_ptr[MAX_DEVICES] = {};

// Scratch address on ctx.device (current); nullptr with last_error set on failure.
double* scratch_of(lfmm::Context& c)
{
	if (c.device < 0 || c.device >= MAX_DEVICES) {
		c.last_error = "lfmm3d_direct_device_noalloc: device index above 63";
		return nullptr;
	}
	std::lock_guard<std::mutex> lock(g_scratch_mu);
	if (!g_scratch_ptr[c.device]) {
		void* p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_direct_scratch);
		if (e != cudaSuccess || !p) {
			lfmm::cuda_fail(c, e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress(g_direct_scratch)");
			return nullptr;
		}
		if (lfmm::direct_preload3(c) != lfmm::OK) return nullptr;
		g_scratch_ptr[c.device] = static_cast<double*>(p);
	}
	return g_scratch_ptr[c.device];
}

} // namespace

struct lfmm_ctx;
namespace lfmm { Context& ctx_of(lfmm_ctx* c); }

extern "C" int lfmm3d_direct_device_noalloc(lfmm_ctx* h, size_t ns, const double* src, const double* q, size_t nt,
                                            const double* tgt, double* pot, double* field)
{
	if (!h) return LFMM_ERR_ARG;
	lfmm::Context& c = lfmm::ctx_of(h);
	if (nt > LFMM_DIRECT_NOALLOC_MAX_TARGETS) {
		c.last_error = "lfmm3d_direct_device_noalloc: at most 65536 targets (its static scratch is sized for "
		               "that); use lfmm3d_direct_device for more";
		return LFMM_ERR_ARG;
	}
	if ((ns && (!src || !q)) || (nt && (!tgt || !pot || !field))) {
		c.last_error = "null buffer";
		return LFMM_ERR_ARG;
	}
	if (nt == 0) return LFMM_OK;
	// the caller's current device is put back on every return
	int prev = -1;
	cudaError_t e = cudaGetDevice(&prev);
	if (e != cudaSuccess) return lfmm::cuda_fail(c, e, "cudaGetDevice");
	if (prev != c.device && (e = cudaSetDevice(c.device)) != cudaSuccess) return lfmm::cuda_fail(c, e, "cudaSetDevice");
	int st = LFMM_ERR_CUDA;
	if (double* scratch = scratch_of(c)) {
		const int S = lfmm::direct_chunks(ns, nt, c.num_sms, SCRATCH_DOUBLES / (4 * nt));
		st = lfmm::direct_launch(c, 3, ns, src, q, nt, tgt, pot, field, scratch, S);
	}
	if (prev != c.device) cudaSetDevice(prev);
	return st;
}
