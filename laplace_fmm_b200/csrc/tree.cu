// Device tree build: bounding box, Morton codes, stable radix sort, levels,
// q == 0 target partition, close lists.  Integer results are bit-exact with
// the reference's MortonTree (reference cpu/morton_tree.cpp:286-493).
#include "tree.cuh"
#include "primitives.cuh"

namespace lfmm {

namespace {

template <int DIM>
__device__ __forceinline__ void load_point(const ParticleInput in, size_t i, double* p)
{
	const double* b = i < in.nt ? in.tgt + DIM * i : in.src + DIM * (i - in.nt);
#pragma unroll
	for (int d = 0; d < DIM; ++d) p[d] = b[d];
}

// Element e of the input coordinates read as one array: the targets' nt x DIM
// doubles followed by the sources' (both interleaved, one particle per DIM
// consecutive doubles).  Walking e with consecutive lanes makes every warp
// load 32 consecutive doubles (256 bytes).
template <int DIM>
__device__ __forceinline__ double point_elem(const ParticleInput& in, size_t e)
{
	const size_t te = in.nt * DIM;
	return e < te ? __ldg(in.tgt + e) : __ldg(in.src + (e - te));
}

// Min / max of coordinate d over the elements [e, e_end) taken with stride S by
// this thread; the coordinate of element e is e mod DIM, kept incrementally.
// Four independent loads per iteration keep enough requests in flight.
template <int DIM>
__device__ __forceinline__ void minmax_elems(const ParticleInput& in, size_t e, size_t e_end, size_t S,
                                             double* mn, double* mx)
{
	int d = (int)(e % DIM);
	const int dS = (int)(S % DIM);
	auto take = [&](double v) {
#pragma unroll
		for (int k = 0; k < DIM; ++k)
			if (d == k) { mn[k] = fmin(mn[k], v); mx[k] = fmax(mx[k], v); }
		d += dS;
		if (d >= DIM) d -= DIM;
	};
	for (; e + 3 * S < e_end; e += 4 * S) {
		const double v0 = point_elem<DIM>(in, e), v1 = point_elem<DIM>(in, e + S);
		const double v2 = point_elem<DIM>(in, e + 2 * S), v3 = point_elem<DIM>(in, e + 3 * S);
		take(v0); take(v1); take(v2); take(v3);
	}
	for (; e < e_end; e += S) take(point_elem<DIM>(in, e));
}

constexpr int BBOX_BLOCKS = 1184;               // 8 per SM
constexpr int BBOX_THREADS = 256;

template <int DIM>
__global__ void __launch_bounds__(BBOX_THREADS) bbox_partial_kernel(const ParticleInput in, size_t n, double* partial)
{
	double mn[DIM], mx[DIM];
	{
		double p[DIM];
		load_point<DIM>(in, 0, p);
#pragma unroll
		for (int d = 0; d < DIM; ++d) mn[d] = mx[d] = p[d];
	}
	minmax_elems<DIM>(in, (size_t)blockIdx.x * blockDim.x + threadIdx.x, n * DIM, (size_t)gridDim.x * blockDim.x,
	                  mn, mx);
#pragma unroll
	for (int d = 0; d < DIM; ++d)
		for (int o = 16; o > 0; o >>= 1) {
			mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
			mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
		}
	__shared__ double s[BBOX_THREADS / 32][2 * DIM];
	int w = threadIdx.x >> 5;
	if ((threadIdx.x & 31) == 0)
		for (int d = 0; d < DIM; ++d) { s[w][d] = mn[d]; s[w][DIM + d] = mx[d]; }
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int k = 1; k < BBOX_THREADS / 32; ++k)
			for (int d = 0; d < DIM; ++d) { s[0][d] = fmin(s[0][d], s[k][d]); s[0][DIM + d] = fmax(s[0][DIM + d], s[k][DIM + d]); }
		for (int d = 0; d < 2 * DIM; ++d) partial[blockIdx.x * 2 * DIM + d] = s[0][d];
	}
}

// shift = min - 1e-7, scale = largest extent + 1e-6 (reference cpu/morton_tree.cpp:293-301)
// One warp: lane l folds the partials l, l + 32, ..., then shuffles.
template <int DIM>
__global__ void bbox_final_kernel(const double* partial, int nb, double* geo)
{
	const int lane = threadIdx.x;
	if (lane >= 32) return;
	double mn[DIM], mx[DIM];
	for (int d = 0; d < DIM; ++d) { mn[d] = partial[d]; mx[d] = partial[DIM + d]; }
	for (int b = lane; b < nb; b += 32)
		for (int d = 0; d < DIM; ++d) { mn[d] = fmin(mn[d], partial[b * 2 * DIM + d]); mx[d] = fmax(mx[d], partial[b * 2 * DIM + DIM + d]); }
	for (int d = 0; d < DIM; ++d)
		for (int o = 16; o > 0; o >>= 1) {
			mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
			mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
		}
	if (lane != 0) return;
	double dw = mx[0] - mn[0];
	for (int d = 1; d < DIM; ++d) dw = fmax(dw, mx[d] - mn[d]);
	for (int d = 0; d < 3; ++d) geo[d] = d < DIM ? mn[d] - 1.e-7 : 0.0;
	geo[3] = dw + 1.e-6;
}

// Forest: the bounding box of each problem, one block per problem, with the
// same shift / scale rule.
template <int DIM>
__global__ void __launch_bounds__(BBOX_THREADS) bbox_segment_kernel(const ParticleInput in, double* geo)
{
	const uint32_t b = in.poff[blockIdx.x], e = in.poff[blockIdx.x + 1];
	double mn[DIM], mx[DIM];
#pragma unroll
	for (int d = 0; d < DIM; ++d) { mn[d] = 1e300; mx[d] = -1e300; }
	minmax_elems<DIM>(in, (size_t)b * DIM + threadIdx.x, (size_t)e * DIM, blockDim.x, mn, mx);
#pragma unroll
	for (int d = 0; d < DIM; ++d)
		for (int o = 16; o > 0; o >>= 1) {
			mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
			mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
		}
	__shared__ double s[BBOX_THREADS / 32][2 * DIM];
	const int w = threadIdx.x >> 5;
	if ((threadIdx.x & 31) == 0)
		for (int d = 0; d < DIM; ++d) { s[w][d] = mn[d]; s[w][DIM + d] = mx[d]; }
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int k = 1; k < BBOX_THREADS / 32; ++k)
			for (int d = 0; d < DIM; ++d) { s[0][d] = fmin(s[0][d], s[k][d]); s[0][DIM + d] = fmax(s[0][DIM + d], s[k][DIM + d]); }
		double dw = s[0][DIM] - s[0][0];
		for (int d = 1; d < DIM; ++d) dw = fmax(dw, s[0][DIM + d] - s[0][d]);
		double* g = geo + 4 * blockIdx.x;
		for (int d = 0; d < 3; ++d) g[d] = d < DIM ? s[0][d] - 1.e-7 : 0.0;
		g[3] = dw + 1.e-6;
	}
}

// code = interleave(trunc(2^(depth-1) * (x - shift) / scale)), x highest
// (reference cpu/morton_tree.cpp:48-99); IEEE-rounded ops, no contraction.
// Forest: the particle's problem index above the Morton bits, the problem's box.
// The block's positions are staged through shared memory with coalesced loads.
constexpr int CODES_THREADS = 256;

template <int DIM>
__global__ void __launch_bounds__(CODES_THREADS) codes_kernel(const ParticleInput in, size_t n,
                                                              const double* __restrict__ geo_all, int depth,
                                                              uint64_t* __restrict__ keys, uint32_t* __restrict__ vals)
{
	__shared__ double sp[CODES_THREADS * DIM];
	const size_t first = (size_t)blockIdx.x * CODES_THREADS;
	for (int j = threadIdx.x; j < CODES_THREADS * DIM; j += CODES_THREADS) {
		const size_t e = first * DIM + j;
		if (e < n * DIM) sp[j] = point_elem<DIM>(in, e);
	}
	__syncthreads();
	size_t i = first + threadIdx.x;
	if (i >= n) return;
	double p[DIM];
#pragma unroll
	for (int d = 0; d < DIM; ++d) p[d] = sp[threadIdx.x * DIM + d];
	uint64_t prob = 0;
	if (in.nprob > 1) {
		int lo = 0, hi = in.nprob;          // last k with poff[k] <= i
		while (hi - lo > 1) {
			const int mid = (lo + hi) >> 1;
			if (in.poff[mid] <= i) lo = mid; else hi = mid;
		}
		prob = (uint64_t)lo;
	}
	const double* geo = geo_all + 4 * prob;
	double scale = geo[3];
	double bit_shift = (double)(1ull << (depth - 1));
	uint64_t c = 0;
#pragma unroll
	for (int d = 0; d < DIM; ++d) {
		double u = __ddiv_rn(__dsub_rn(p[d], geo[d]), scale);
		uint64_t v = (uint64_t)__dmul_rn(bit_shift, u);
		c |= (DIM == 3 ? spread3(v) : spread2(v)) << (DIM - 1 - d);
	}
	keys[i] = c | (prob << (DIM * (depth - 1)));
	vals[i] = (uint32_t)i;
}

// Gather into tree order; count q == 0 particles; mark the coarsest level at
// which each particle starts a new cell (depth = none).
template <int DIM>
__global__ void gather_kernel(const ParticleInput in, size_t n, const uint64_t* __restrict__ keys,
                              const uint32_t* __restrict__ vals, DevTree t, uint8_t* __restrict__ newlev,
                              unsigned* __restrict__ level_hist)
{
	__shared__ unsigned h[MAX_LEVELS + 2];
	if (threadIdx.x < MAX_LEVELS + 2) h[threadIdx.x] = 0;
	__syncthreads();
	size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n) {
		uint32_t i = vals[s];
		double p[DIM];
		load_point<DIM>(in, i, p);
		t.x[s] = p[0]; t.y[s] = p[1];
		if (DIM == 3) t.z[s] = p[2];
		double q = i < in.nt ? 0.0 : in.srcq[i - in.nt];
		t.q[s] = q;
		uint64_t c = keys[s];
		t.pcode[s] = c;
		t.orig[s] = i;
		int lev;
		if (s == 0) lev = 0;
		else {
			uint64_t x = c ^ keys[s - 1];
			if (x == 0) lev = t.depth;
			else {
				int b = 63 - __clzll((long long)x);
				lev = max(0, t.depth - 1 - b / DIM);     // a new problem of a forest: a new root
			}
		}
		newlev[s] = (uint8_t)lev;
		atomicAdd(&h[lev], 1u);
		if (q == 0.0) atomicAdd(&h[MAX_LEVELS + 1], 1u);
	}
	__syncthreads();
	if (threadIdx.x < MAX_LEVELS + 2 && h[threadIdx.x]) atomicAdd(&level_hist[threadIdx.x], h[threadIdx.x]);
}

__global__ void leaf_flags_kernel(const uint8_t* __restrict__ newlev, size_t n, int leaf, uint32_t* __restrict__ flags)
{
	size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n) flags[s] = newlev[s] <= leaf ? 1u : 0u;
}

__global__ void leaf_cells_kernel(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ excl, size_t n,
                                  DevTree t, size_t off)
{
	size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n && flags[s]) {
		size_t c = off + excl[s];
		t.beg[c] = (uint32_t)s;
		t.code[c] = t.pcode[s];
	}
}

__global__ void cell_ends_kernel(DevTree t, size_t off, size_t m, uint32_t total)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c < m) t.end[off + c] = c + 1 < m ? t.beg[off + c + 1] : total;
}

template <int DIM>
__global__ void parent_flags_kernel(const uint64_t* __restrict__ code, size_t m, uint32_t* __restrict__ flags)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c < m) flags[c] = (c == 0 || (code[c] >> DIM) != (code[c - 1] >> DIM)) ? 1u : 0u;
}

template <int DIM>
__global__ void parent_cells_kernel(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ excl, size_t m,
                                    DevTree t, size_t child_off, size_t par_off)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= m) return;
	uint32_t p = excl[c] + flags[c] - 1;
	t.parent[child_off + c] = (int32_t)p;
	if (flags[c]) {
		t.beg[par_off + p] = (uint32_t)c;
		t.code[par_off + p] = t.code[child_off + c] >> DIM;
	}
}

// centre = shift + scale * (decoded corner + 1/2) / 2^L
// (reference cpu/morton_tree.cpp:101-145), no contraction
template <int DIM>
__global__ void centres_kernel(DevTree t, int L, size_t off, size_t m)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= m) return;
	uint64_t v = t.code[off + c];
	const double* geo = t.geo + (t.nprob > 1 ? 4 * (v >> (DIM * L)) : 0);
	double step = 1.0 / (double)(1ull << (L + 1));
	double x = step, y = step, z = step;
	step *= 2;
	for (int i = 0; i < L; ++i) {
		if (DIM == 3) { z += step * (double)(v & 1); v >>= 1; }
		y += step * (double)(v & 1); v >>= 1;
		x += step * (double)(v & 1); v >>= 1;
		step *= 2;
	}
	double scale = geo[3];
	t.cx[off + c] = __dadd_rn(__dmul_rn(x, scale), geo[0]);
	t.cy[off + c] = __dadd_rn(__dmul_rn(y, scale), geo[1]);
	if (DIM == 3) t.cz[off + c] = __dadd_rn(__dmul_rn(z, scale), geo[2]);
	t.tbeg[off + c] = 0; t.tend[off + c] = 0;
}

// Stable partition inside each leaf: q != 0 first (sources), then q == 0
// (targets).  The reference partitions by swaps (cpu/morton_tree.cpp:445-458),
// which keeps the same member sets.  One warp per leaf, out of place.
template <int DIM>
__global__ void partition_kernel(DevTree t, size_t off, size_t m, double* x2, double* y2, double* z2, double* q2,
                                 uint32_t* o2, uint64_t* c2)
{
	size_t leaf = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	unsigned lane = threadIdx.x & 31;
	if (leaf >= m) return;
	uint32_t b = t.beg[off + leaf], e = t.end[off + leaf];
	// count sources
	uint32_t nsrc = 0;
	for (uint32_t i = b + lane; i < e + 31 && i - lane < e; i += 32) {
		bool src = i < e && t.q[i] != 0.0;
		nsrc += __popc(__ballot_sync(0xffffffffu, src));
	}
	uint32_t ws = b, wt = b + nsrc;
	const unsigned lt = (1u << lane) - 1u;
	for (uint32_t base = b; base < e; base += 32) {
		uint32_t i = base + lane;
		bool valid = i < e;
		bool src = valid && t.q[i] != 0.0;
		unsigned bs = __ballot_sync(0xffffffffu, src);
		unsigned bt = __ballot_sync(0xffffffffu, valid && !src);
		if (valid) {
			uint32_t dst = src ? ws + __popc(bs & lt) : wt + __popc(bt & lt);
			x2[dst] = t.x[i]; y2[dst] = t.y[i];
			if (DIM == 3) z2[dst] = t.z[i];
			q2[dst] = t.q[i]; o2[dst] = t.orig[i]; c2[dst] = t.pcode[i];
		}
		ws += __popc(bs); wt += __popc(bt);
	}
	if (lane == 0) {
		t.tbeg[off + leaf] = b + nsrc;
		t.tend[off + leaf] = e;
		t.end[off + leaf] = b + nsrc;
	}
}

__global__ void source_targets_kernel(DevTree t, size_t off, size_t m)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c < m) { t.tbeg[off + c] = t.beg[off + c]; t.tend[off + c] = t.end[off + c]; }
}

template <int DIM>
__device__ __forceinline__ void cell_coords(uint64_t code, int* c)
{
	if (DIM == 3) { c[0] = (int)compact3(code >> 2); c[1] = (int)compact3(code >> 1); c[2] = (int)compact3(code); }
	else { c[0] = (int)compact2(code >> 1); c[1] = (int)compact2(code); c[2] = 0; }
}

// Close lists (Chebyshev distance 1 among the children of the parent's close
// cells and of the parent, in that order) and far counts; level 1: all other
// level-1 cells.  Same rule and order as reference cpu/morton_tree.cpp:147-208.
template <int DIM>
__global__ void lists_kernel(DevTree t, int L, unsigned* flags)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	size_t m = t.lsize[L];
	if (c >= m) return;
	size_t off = t.loff[L];
	int32_t* out = t.close_idx + (off + c) * t.close_stride;
	int nc = 0, nf = 0;
	if (L == 1) {
		// the other children of the root (forest: of the same root)
		const int32_t pc = t.parent[off + c];
		for (size_t k = 0; k < m; ++k)
			if (k != c && t.parent[off + k] == pc) { if (nc < t.close_stride) out[nc] = (int32_t)k; nc++; }
	} else {
		int me[3];
		cell_coords<DIM>(t.code[off + c], me);
		size_t poff = t.loff[L - 1];
		int32_t p = t.parent[off + c];
		int npc = t.close_cnt[poff + p];
		const int32_t* pl = t.close_idx + (poff + p) * t.close_stride;
		for (int e = 0; e <= npc; ++e) {
			int32_t pn = e < npc ? pl[e] : p;
			for (uint32_t k = t.beg[poff + pn]; k < t.end[poff + pn]; ++k) {
				if (k == c) continue;
				int o[3];
				cell_coords<DIM>(t.code[off + k], o);
				int d = max(abs(o[0] - me[0]), abs(o[1] - me[1]));
				if (DIM == 3) d = max(d, abs(o[2] - me[2]));
				if (d <= 1) { if (nc < t.close_stride) out[nc] = (int32_t)k; nc++; }
				else nf++;
			}
		}
	}
	if (nc > t.close_stride) { atomicOr(flags, DEV_ERR_LIST_OVERFLOW); nc = t.close_stride; }
	t.close_cnt[off + c] = nc;
	t.far_cnt[off + c] = nf;
}

template <int DIM>
__global__ void far_fill_kernel(DevTree t, int L, const uint32_t* __restrict__ far_off, int32_t* __restrict__ far_idx,
                                size_t cap, unsigned* flags)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	size_t m = t.lsize[L];
	if (c >= m || L < 2) return;
	size_t off = t.loff[L], poff = t.loff[L - 1];
	int me[3];
	cell_coords<DIM>(t.code[off + c], me);
	int32_t p = t.parent[off + c];
	int npc = t.close_cnt[poff + p];
	const int32_t* pl = t.close_idx + (poff + p) * t.close_stride;
	size_t w = far_off[c];
	for (int e = 0; e <= npc; ++e) {
		int32_t pn = e < npc ? pl[e] : p;
		for (uint32_t k = t.beg[poff + pn]; k < t.end[poff + pn]; ++k) {
			if (k == c) continue;
			int o[3];
			cell_coords<DIM>(t.code[off + k], o);
			int d = max(abs(o[0] - me[0]), abs(o[1] - me[1]));
			if (DIM == 3) d = max(d, abs(o[2] - me[2]));
			if (d > 1) {
				if (w < cap) far_idx[w] = (int32_t)k;
				else atomicOr(flags, DEV_ERR_LIST_OVERFLOW);
				w++;
			}
		}
	}
}

template <typename T>
T* take(Context& ctx, size_t count)
{
	return static_cast<T*>(ctx.arena.take(sizeof(T) * (count ? count : 1)));
}

} // namespace

int tree_build(Context& ctx, const ParticleInput& in, int depth, DevTree& t, bool partition, bool lists)
{
	const int dim = in.dim;
	const size_t n = in.ns + in.nt;
	const int nprob = std::max(in.nprob, 1);
	int pbits = 0;
	while ((1ll << pbits) < nprob) ++pbits;
	if (n == 0 || n > 0xffffffffull || depth < 1 || depth > MAX_LEVELS - 1 || dim * (depth - 1) + pbits > 62 ||
	    (nprob > 1 && (in.nt > 0 || !in.poff))) {
		ctx.last_error = "tree: unsupported particle count, depth or problem count";
		return ERR_ARG;
	}
	cudaStream_t s = ctx.stream;
	t = DevTree();
	t.dim = dim; t.depth = depth; t.n = n; t.nt = in.nt; t.nprob = nprob;
	t.close_stride = dim == 3 ? 26 : 8;
	t.geo = take<double>(ctx, 4 * (size_t)nprob);
	t.x = take<double>(ctx, n); t.y = take<double>(ctx, n); t.z = dim == 3 ? take<double>(ctx, n) : nullptr;
	t.q = take<double>(ctx, n); t.orig = take<uint32_t>(ctx, n); t.pcode = take<uint64_t>(ctx, n);
	uint64_t* keys = take<uint64_t>(ctx, n);
	uint64_t* keys2 = take<uint64_t>(ctx, n);
	uint32_t* vals = take<uint32_t>(ctx, n);
	uint32_t* vals2 = take<uint32_t>(ctx, n);
	uint32_t* scratch = take<uint32_t>(ctx, radix_scratch_words(n) + scan_scratch_words(n));
	uint8_t* newlev = take<uint8_t>(ctx, n);
	uint32_t* flags = take<uint32_t>(ctx, n);
	uint32_t* excl = take<uint32_t>(ctx, n);
	double* partial = take<double>(ctx, BBOX_BLOCKS * 6);
	unsigned* hist = take<unsigned>(ctx, MAX_LEVELS + 2);
	if (!t.geo || !t.x || !t.orig || !keys || !scratch || !excl || !hist) { ctx.last_error = "tree: device allocation failed"; return ERR_OOM; }

	LFMM_CUDA(ctx, cudaMemsetAsync(hist, 0, sizeof(unsigned) * (MAX_LEVELS + 2), s));
	const unsigned TB = 256;
	if (dim == 3 && nprob > 1) {
		bbox_segment_kernel<3><<<nprob, BBOX_THREADS, 0, s>>>(in, t.geo);
		codes_kernel<3><<<div_up(n, CODES_THREADS), CODES_THREADS, 0, s>>>(in, n, t.geo, depth, keys, vals);
	} else if (dim == 3) {
		bbox_partial_kernel<3><<<BBOX_BLOCKS, BBOX_THREADS, 0, s>>>(in, n, partial);
		bbox_final_kernel<3><<<1, 32, 0, s>>>(partial, BBOX_BLOCKS, t.geo);
		codes_kernel<3><<<div_up(n, CODES_THREADS), CODES_THREADS, 0, s>>>(in, n, t.geo, depth, keys, vals);
	} else {
		bbox_partial_kernel<2><<<BBOX_BLOCKS, BBOX_THREADS, 0, s>>>(in, n, partial);
		bbox_final_kernel<2><<<1, 32, 0, s>>>(partial, BBOX_BLOCKS, t.geo);
		codes_kernel<2><<<div_up(n, CODES_THREADS), CODES_THREADS, 0, s>>>(in, n, t.geo, depth, keys, vals);
	}
	int which = radix_sort_pairs(keys, vals, keys2, vals2, n, 0, dim * (depth - 1) + pbits, scratch, s);
	uint64_t* sk = which ? keys2 : keys;
	uint32_t* sv = which ? vals2 : vals;
	if (dim == 3) gather_kernel<3><<<div_up(n, TB), TB, 0, s>>>(in, n, sk, sv, t, newlev, hist);
	else gather_kernel<2><<<div_up(n, TB), TB, 0, s>>>(in, n, sk, sv, t, newlev, hist);
	unsigned hh[MAX_LEVELS + 2];
	LFMM_CUDA(ctx, cudaMemcpyAsync(hh, hist, sizeof(hh), cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(t.geo_host, t.geo, sizeof(t.geo_host), cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	size_t acc = 0;
	for (int L = 0; L < depth; ++L) { acc += hh[L]; t.lsize[L] = acc; }
	t.targets_num = hh[MAX_LEVELS + 1];
	t.ncells = 0;
	for (int L = 0; L < depth; ++L) { t.loff[L] = t.ncells; t.ncells += t.lsize[L]; }
	const size_t C = t.ncells;
	t.code = take<uint64_t>(ctx, C);
	t.beg = take<uint32_t>(ctx, C); t.end = take<uint32_t>(ctx, C);
	t.tbeg = take<uint32_t>(ctx, C); t.tend = take<uint32_t>(ctx, C);
	t.parent = take<int32_t>(ctx, C);
	t.cx = take<double>(ctx, C); t.cy = take<double>(ctx, C); t.cz = dim == 3 ? take<double>(ctx, C) : nullptr;
	t.close_cnt = take<int32_t>(ctx, C);
	t.close_idx = take<int32_t>(ctx, C * t.close_stride);
	t.far_cnt = take<int32_t>(ctx, C);
	if (!t.code || !t.close_idx || !t.far_cnt) { ctx.last_error = "tree: device allocation failed"; return ERR_OOM; }

	// leaves
	const int LL = depth - 1;
	uint32_t* scan_scr = scratch + radix_scratch_words(n);
	leaf_flags_kernel<<<div_up(n, TB), TB, 0, s>>>(newlev, n, LL, flags);
	scan_exclusive_u32(flags, excl, n, nullptr, scan_scr, s);
	leaf_cells_kernel<<<div_up(n, TB), TB, 0, s>>>(flags, excl, n, t, t.loff[LL]);
	cell_ends_kernel<<<div_up(t.lsize[LL], TB), TB, 0, s>>>(t, t.loff[LL], t.lsize[LL], (uint32_t)n);
	// upper levels
	for (int L = depth - 2; L >= 0; --L) {
		size_t m1 = t.lsize[L + 1];
		if (dim == 3) parent_flags_kernel<3><<<div_up(m1, TB), TB, 0, s>>>(t.code + t.loff[L + 1], m1, flags);
		else parent_flags_kernel<2><<<div_up(m1, TB), TB, 0, s>>>(t.code + t.loff[L + 1], m1, flags);
		scan_exclusive_u32(flags, excl, m1, nullptr, scan_scr, s);
		if (dim == 3) parent_cells_kernel<3><<<div_up(m1, TB), TB, 0, s>>>(flags, excl, m1, t, t.loff[L + 1], t.loff[L]);
		else parent_cells_kernel<2><<<div_up(m1, TB), TB, 0, s>>>(flags, excl, m1, t, t.loff[L + 1], t.loff[L]);
		cell_ends_kernel<<<div_up(t.lsize[L], TB), TB, 0, s>>>(t, t.loff[L], t.lsize[L], (uint32_t)m1);
	}
	LFMM_CUDA(ctx, cudaMemsetAsync(t.parent, 0xff, sizeof(int32_t) * t.lsize[0], s));   // roots have no parent
	for (int L = 0; L < depth; ++L) {
		if (dim == 3) centres_kernel<3><<<div_up(t.lsize[L], TB), TB, 0, s>>>(t, L, t.loff[L], t.lsize[L]);
		else centres_kernel<2><<<div_up(t.lsize[L], TB), TB, 0, s>>>(t, L, t.loff[L], t.lsize[L]);
	}
	// target partition
	if (partition && t.targets_num > 0) {
		double* x2 = reinterpret_cast<double*>(keys2 == sk ? keys : keys2);   // reuse the free sort buffer
		double* y2 = take<double>(ctx, n);
		double* z2 = dim == 3 ? take<double>(ctx, n) : nullptr;
		double* q2 = take<double>(ctx, n);
		uint32_t* o2 = vals2 == sv ? vals : vals2;
		uint64_t* c2 = take<uint64_t>(ctx, n);
		if (!y2 || !q2 || !c2) { ctx.last_error = "tree: device allocation failed"; return ERR_OOM; }
		size_t m = t.lsize[LL];
		if (dim == 3) partition_kernel<3><<<div_up(m * 32, TB), TB, 0, s>>>(t, t.loff[LL], m, x2, y2, z2, q2, o2, c2);
		else partition_kernel<2><<<div_up(m * 32, TB), TB, 0, s>>>(t, t.loff[LL], m, x2, y2, z2, q2, o2, c2);
		LFMM_CUDA(ctx, cudaMemcpyAsync(t.x, x2, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
		t.y = y2; t.z = z2; t.q = q2; t.orig = o2; t.pcode = c2;
	} else {
		source_targets_kernel<<<div_up(t.lsize[LL], TB), TB, 0, s>>>(t, t.loff[LL], t.lsize[LL]);
	}
	LFMM_CUDA(ctx, cudaGetLastError());
	return lists ? tree_lists(ctx, t) : OK;
}

int tree_lists(Context& ctx, DevTree& t)
{
	cudaStream_t s = ctx.stream;
	LFMM_CUDA(ctx, cudaMemsetAsync(t.close_cnt, 0, sizeof(int32_t) * t.ncells, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(t.far_cnt, 0, sizeof(int32_t) * t.ncells, s));
	for (int L = 1; L < t.depth; ++L) {
		if (t.lsize[L] == 0) continue;
		if (t.dim == 3) lists_kernel<3><<<div_up(t.lsize[L], 128), 128, 0, s>>>(t, L, ctx.dev_flags);
		else lists_kernel<2><<<div_up(t.lsize[L], 128), 128, 0, s>>>(t, L, ctx.dev_flags);
	}
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

namespace {

__global__ void count_pairs_kernel(DevTree t, unsigned long long* out)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long far = 0, close = 0, p2p = 0;
	size_t leaf0 = t.loff[t.depth - 1];
	if (c < t.ncells) {
		far = (unsigned long long)t.far_cnt[c];
		if (c >= leaf0) {
			int nc = t.close_cnt[c];
			close = (unsigned long long)nc;
			bool tmode = t.targets_num > 0;
			unsigned long long nt = tmode ? t.tend[c] - t.tbeg[c] : t.end[c] - t.beg[c];
			unsigned long long ns = t.end[c] - t.beg[c];
			for (int e = 0; e < nc; ++e) {
				size_t k = leaf0 + t.close_idx[c * t.close_stride + e];
				ns += t.end[k] - t.beg[k];
			}
			p2p = nt * ns;
		}
	}
	far = warp_sum(far); close = warp_sum(close); p2p = warp_sum(p2p);
	if ((threadIdx.x & 31) == 0) { atomicAdd(out, far); atomicAdd(out + 1, close); atomicAdd(out + 2, p2p); }
}

} // namespace

int tree_count_pairs(Context& ctx, const DevTree& t, unsigned long long* dev, unsigned long long* out)
{
	cudaStream_t s = ctx.stream;
	LFMM_CUDA(ctx, cudaMemsetAsync(dev, 0, 3 * sizeof(unsigned long long), s));
	count_pairs_kernel<<<div_up(t.ncells, 256), 256, 0, s>>>(t, dev);
	LFMM_CUDA(ctx, cudaMemcpyAsync(out, dev, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	return OK;
}

int tree_far_lists(Context& ctx, const DevTree& t, int L, uint32_t* far_off, int32_t* far_idx, size_t cap)
{
	size_t m = t.lsize[L];
	cudaStream_t s = ctx.stream;
	uint32_t* scr = static_cast<uint32_t*>(ctx.arena.take(sizeof(uint32_t) * (scan_scratch_words(m) + 1)));
	if (!scr) return ERR_OOM;
	scan_exclusive_u32(reinterpret_cast<const uint32_t*>(t.far_cnt + t.loff[L]), far_off, m, far_off + m, scr, s);
	if (t.dim == 3) far_fill_kernel<3><<<div_up(m, 128), 128, 0, s>>>(t, L, far_off, far_idx, cap, ctx.dev_flags);
	else far_fill_kernel<2><<<div_up(m, 128), 128, 0, s>>>(t, L, far_off, far_idx, cap, ctx.dev_flags);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

} // namespace lfmm
