// Solver context: stream, device arena, math tables, error state.
#pragma once
#include "common.cuh"
#include <string>
#include <utility>
#include <vector>

namespace lfmm {

// Bump allocator over one device block.  A solve that outgrows the block
// takes extra cudaMalloc chunks; at the end of the solve they are released and
// the block is regrown to the high-water mark, so repeated solves of the same
// shape allocate nothing.
class Arena {
public:
	~Arena();
	void reset() { used_ = 0; }
	void* take(size_t bytes);               // nullptr on cudaMalloc failure
	void settle();                          // end of solve: consolidate chunks
	size_t capacity() const { return cap_; }
	size_t high_water() const { return high_; }
	void release();
	// position in the block; rewind(mark()) replays the same addresses while
	// no extra chunk was taken in between (chunks() unchanged)
	size_t mark() const { return used_; }
	void rewind(size_t m) { used_ = m; }
	size_t chunks() const { return extra_.size(); }
	void swap(Arena& o)
	{
		std::swap(base_, o.base_); std::swap(cap_, o.cap_); std::swap(used_, o.used_);
		std::swap(high_, o.high_); std::swap(extra_total_, o.extra_total_); extra_.swap(o.extra_);
	}
private:
	char* base_ = nullptr;
	size_t cap_ = 0, used_ = 0, high_ = 0, extra_total_ = 0;
	std::vector<void*> extra_;
};

// Rotation / translation tables, built once per context on the GPU (FP64).
// DevTables is the plain-pointer view passed to kernels.
struct DevTables {
	// Wigner small-d matrices (N = 18 layout) for each theta slot
	double* dmat = nullptr;
	int n_dslots = 0;
	// (cos m phi, sin m phi), m < 18, for each phi slot
	double2* emat = nullptr;
	int n_eslots = 0;
	// per integer direction (dx+3)*49+(dy+3)*7+(dz+3):
	// {dslot(theta), dslot(-theta), eslot(phi), eslot(-phi)}, -1 if absent
	int4* dirinfo = nullptr;
	// K(n,m) and the translation coefficient cubes [j][k][n] (18^3)
	double* knm = nullptr;
	double* m2l = nullptr;
	double* m2m = nullptr;
	double* l2l = nullptr;
	// FP32 copies for the mixed form (same layouts)
	float* dmat_f = nullptr;
	float2* emat_f = nullptr;
	float* knm_f = nullptr;
	float* m2l_f = nullptr;
	float* m2m_f = nullptr;
	float* l2l_f = nullptr;
};

struct Tables {
	DevTables d;
	// host copies of the canonical angles (tests)
	std::vector<double> theta_of_slot, phi_of_slot;
	std::vector<int4> dirinfo_host;
};

// Dense M2L operators [343][MT][MT] of one (order, cell size, precision),
// kept across solves (repeated solves of one geometry rebuild nothing).
struct OpCacheEntry {
	int N = 0, prec = 0;
	double h = 0.0;
	void* ptr = nullptr;
	size_t bytes = 0;
	unsigned long long stamp = 0;
	int pinned = 0;                   // > 0: a captured graph reads it (never evicted)
	float aux = 1.f;                  // FP16 tensor-core operators: the inverse of their scale
};

struct Context {
	int device = 0;
	int num_sms = 148;
	cudaStream_t stream = nullptr;
	Arena arena;
	Tables tables;
	std::vector<OpCacheEntry> opcache;
	unsigned long long opcache_clock = 0;
	int m2l_engine = 3;               // 0: dense SIMT GEMMs, 1: per-pair rotations (plain path), 3: tcgen05 on FP32 levels
	unsigned* dev_flags = nullptr;      // device error flags
	// Device errors of asynchronous solves (device buffers, no stats): latched
	// at the end of each such solve into this mapped pinned word (host view,
	// device view) and read by lfmm_check.
	unsigned* host_flags = nullptr;
	unsigned* host_flags_dev = nullptr;
	std::string last_error;
	int verbose = 0;
	cudaEvent_t ev[16] = {};
	cudaStream_t side = nullptr;        // lowest-priority stream for work that overlaps a solve
	cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
	cudaEvent_t kev[32] = {};          // pairs around the tensor-core M2L launches (timing)
	int kev_used = 0;
	// tcgen05 M2L operands: FP16 hi / lo pairs (1, the default) or TF32 hi / lo
	// pairs (0; LFMM_M2L_TYPE=tf32)
	int m2l_f16 = 1;
	// FP16 M2L sources gathered by TMA row gathers (1, the default) or by the
	// producers' loads (0; LFMM_M2L_GATHER=ldg)
	int m2l_tma = 1;
	// M2L autotuner: slot split chosen per (operand type and gather, operator rows / 16,
	// level-size bucket); 0 = not tuned yet.  tune_m2l = 0 (LFMM_M2L_TUNE=0):
	// the fixed rule.  Operator rows reach 352 (N = 18): 23 row classes.
	static constexpr int SPLIT_ROWS = 352 / 16 + 1;
	int m2l_split[3][SPLIT_ROWS][33] = {};
	int tune_m2l = 1;
	int timing = 0;
};

// With 48 entries cached (four per order: FP64 and tensor-core M2L, M2M and
// L2L operators), evict the least recently used one no graph reads.
inline void opcache_make_room(Context& ctx)
{
	if (ctx.opcache.size() < 48) return;
	auto it = ctx.opcache.end();
	for (auto j = ctx.opcache.begin(); j != ctx.opcache.end(); ++j)
		if (!j->pinned && (it == ctx.opcache.end() || j->stamp < it->stamp)) it = j;
	if (it != ctx.opcache.end()) {
		cudaStreamSynchronize(ctx.stream);
		cudaFree(it->ptr);
		ctx.opcache.erase(it);
	}
}

int tables_build(Context& ctx);
void tables_free(Tables& t);

// set last_error from a CUDA error; returns ERR_CUDA
int cuda_fail(Context& ctx, cudaError_t e, const char* where);

#define LFMM_CUDA(ctx, call)                                                   \
	do {                                                                       \
		cudaError_t e__ = (call);                                              \
		if (e__ != cudaSuccess) return ::lfmm::cuda_fail((ctx), e__, #call);  \
	} while (0)

} // namespace lfmm
