// Adaptive octree / quadtree and its U / V / W / X interaction lists.
//
// The reference builds only uniform-depth trees (cpu/morton_tree.cpp:286-493);
// this builder starts from the same bit-exact uniform tree (all levels down to
// depth - 1) and keeps a cell when its parent is split, splitting while a cell
// holds more than max_leaf particles.  Lists, for a cell B at level L:
//   colleagues  same-level adjacent cells (close_idx, as the uniform tree)
//   V(B)        children of the parent's colleagues not adjacent to B  (M2L)
//   U(B)        leaf B: every leaf adjacent to B, any level              (P2P)
//   W(B)        leaf B: descendants D of B's colleagues with D not adjacent
//               to B and parent(D) adjacent to B                          (M2P)
//   X(B)        leaves C coarser than B, adjacent to parent(B), not
//               adjacent to B (the transpose of W)                         (P2L)
// Adjacency of cubes (squares) on different levels is exact integer arithmetic
// on the Morton coordinates (touching faces, edges or corners count).
#include "tree.cuh"
#include "primitives.cuh"

namespace lfmm {

namespace {

constexpr int STACK = 160;

template <int DIM>
__device__ __forceinline__ void coords(uint64_t code, int* c)
{
	if (DIM == 3) { c[0] = (int)compact3(code >> 2); c[1] = (int)compact3(code >> 1); c[2] = (int)compact3(code); }
	else { c[0] = (int)compact2(code >> 1); c[1] = (int)compact2(code); }
}

// Cube C (level lc, coords c) and cube B (level lb >= lc, coords b) touch or overlap.
template <int DIM>
__device__ __forceinline__ bool touch(int lc, const int* c, int lb, const int* b)
{
	int s = lb - lc;
#pragma unroll
	for (int d = 0; d < DIM; ++d) {
		int lo = c[d] << s, hi = (c[d] + 1) << s;
		if (b[d] < lo - 1 || b[d] > hi) return false;
	}
	return true;
}

__global__ void uprange_kernel(DevTree u, int L, uint32_t* __restrict__ pb, uint32_t* __restrict__ pe)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= u.lsize[L]) return;
	size_t g = u.loff[L] + c;
	if (L == u.depth - 1) { pb[g] = u.beg[g]; pe[g] = u.end[g]; }
	else {
		size_t cb = u.loff[L + 1];
		pb[g] = pb[cb + u.beg[g]];
		pe[g] = pe[cb + u.end[g] - 1];
	}
}

__global__ void keep_kernel(DevTree u, int L, const uint32_t* __restrict__ pb, const uint32_t* __restrict__ pe,
                            uint8_t* __restrict__ keep, uint8_t* __restrict__ split, uint32_t* __restrict__ keep32,
                            int max_leaf)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= u.lsize[L]) return;
	size_t g = u.loff[L] + c;
	bool in = true;
	if (L > 0) {
		size_t gp = u.loff[L - 1] + u.parent[g];
		in = keep[gp] && split[gp];
	}
	bool sp = in && L < u.depth - 1 && (max_leaf == 0 || pe[g] - pb[g] > (uint32_t)max_leaf);
	keep[g] = in; split[g] = sp;
	keep32[c] = in ? 1u : 0u;
}

__global__ void emit_kernel(DevTree u, int L, const uint8_t* __restrict__ keep, const uint8_t* __restrict__ split,
                            const uint32_t* __restrict__ map, const uint32_t* __restrict__ pb,
                            const uint32_t* __restrict__ pe, DevTree a)
{
	size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= u.lsize[L]) return;
	size_t g = u.loff[L] + c;
	if (!keep[g]) return;
	size_t ag = a.loff[L] + map[g];
	a.code[ag] = u.code[g];
	a.cx[ag] = u.cx[g]; a.cy[ag] = u.cy[g];
	if (a.cz) a.cz[ag] = u.cz[g];
	a.pbeg[ag] = pb[g]; a.pend[ag] = pe[g];
	a.lev[ag] = (uint8_t)L;
	a.is_leaf[ag] = split[g] ? 0 : 1;
	a.parent[ag] = L > 0 ? (int32_t)map[u.loff[L - 1] + u.parent[g]] : -1;
	if (split[g]) {
		size_t cb = u.loff[L + 1];
		a.beg[ag] = map[cb + u.beg[g]];
		a.end[ag] = map[cb + u.end[g] - 1] + 1;
	} else {
		a.beg[ag] = 0; a.end[ag] = 0;
	}
}

__global__ void leaf_flag_kernel(DevTree a, uint32_t* __restrict__ f)
{
	size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (g < a.ncells) f[g] = a.is_leaf[g];
}

__global__ void leaf_list_kernel(DevTree a, const uint32_t* __restrict__ f, const uint32_t* __restrict__ pos)
{
	size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (g < a.ncells && f[g]) a.leaves[pos[g]] = (int32_t)g;
}

// Stable partition of every leaf: sources (q != 0) then targets; warp per leaf.
__global__ void partition_leaves_kernel(DevTree a, double* x2, double* y2, double* z2, double* q2, uint32_t* o2,
                                        uint64_t* c2)
{
	size_t li = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	unsigned lane = threadIdx.x & 31;
	if (li >= a.nleaves) return;
	size_t g = a.leaves[li];
	uint32_t b = a.pbeg[g], e = a.pend[g];
	uint32_t nsrc = 0;
	for (uint32_t base = b; base < e; base += 32) {
		uint32_t i = base + lane;
		nsrc += __popc(__ballot_sync(0xffffffffu, i < e && a.q[i] != 0.0));
	}
	uint32_t ws = b, wt = b + nsrc;
	const unsigned lt = (1u << lane) - 1u;
	for (uint32_t base = b; base < e; base += 32) {
		uint32_t i = base + lane;
		bool valid = i < e;
		bool src = valid && a.q[i] != 0.0;
		unsigned bs = __ballot_sync(0xffffffffu, src);
		unsigned bt = __ballot_sync(0xffffffffu, valid && !src);
		if (valid) {
			uint32_t dst = src ? ws + __popc(bs & lt) : wt + __popc(bt & lt);
			x2[dst] = a.x[i]; y2[dst] = a.y[i];
			if (z2) z2[dst] = a.z[i];
			q2[dst] = a.q[i]; o2[dst] = a.orig[i]; c2[dst] = a.pcode[i];
		}
		ws += __popc(bs); wt += __popc(bt);
	}
	if (lane == 0) { a.send[g] = b + nsrc; a.tbeg[g] = b + nsrc; a.tend[g] = e; }
}

__global__ void source_ranges_kernel(DevTree a)
{
	size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (g >= a.ncells) return;
	a.send[g] = a.pend[g];
	a.tbeg[g] = a.pbeg[g];
	a.tend[g] = a.pend[g];
}

// U and W lists of one leaf (pass 0: count, pass 1: fill at the offsets).
template <int DIM>
__global__ void uw_kernel(DevTree a, int pass, uint32_t* __restrict__ ucnt, uint32_t* __restrict__ wcnt, unsigned* flags)
{
	size_t li = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (li >= a.nleaves) return;
	const int32_t g = a.leaves[li];
	const int L = a.lev[g];
	int me[3];
	coords<DIM>(a.code[g], me);
	uint32_t nu = 0, nw = 0;
	const uint32_t ub = pass ? a.u_off[li] : 0, wb = pass ? a.w_off[li] : 0;
	int32_t stack[STACK];
	const int nc = a.close_cnt[g];
	const int32_t* cl = a.close_idx + (size_t)g * a.close_stride;
	const size_t off = a.loff[L];
	for (int e = 0; e < nc; ++e) {
		int32_t C = (int32_t)(off + cl[e]);
		if (a.is_leaf[C]) {
			if (pass) a.u_idx[ub + nu] = C;
			nu++;
			continue;
		}
		int sp = 0;
		{
			size_t cb = a.loff[L + 1];
			for (uint32_t k = a.beg[C]; k < a.end[C]; ++k) stack[sp++] = (int32_t)(cb + k);
		}
		while (sp > 0) {
			int32_t D = stack[--sp];
			int ld = a.lev[D];
			int d[3];
			coords<DIM>(a.code[D], d);
			if (touch<DIM>(L, me, ld, d)) {
				if (a.is_leaf[D]) {
					if (pass) a.u_idx[ub + nu] = D;
					nu++;
				} else {
					size_t cb = a.loff[ld + 1];
					for (uint32_t k = a.beg[D]; k < a.end[D]; ++k) {
						if (sp < STACK) stack[sp++] = (int32_t)(cb + k);
						else atomicOr(flags, DEV_ERR_LIST_OVERFLOW);
					}
				}
			} else {
				if (pass) a.w_idx[wb + nw] = D;
				nw++;
			}
		}
	}
	// coarser adjacent leaves: leaf colleagues of the ancestors that touch B
	int32_t A = g;
	for (int l = L - 1; l >= 1; --l) {
		A = (int32_t)(a.loff[l] + a.parent[A]);
		const int na = a.close_cnt[A];
		const int32_t* al = a.close_idx + (size_t)A * a.close_stride;
		for (int e = 0; e < na; ++e) {
			int32_t C = (int32_t)(a.loff[l] + al[e]);
			if (!a.is_leaf[C]) continue;
			int c[3];
			coords<DIM>(a.code[C], c);
			if (touch<DIM>(l, c, L, me)) {
				if (pass) a.u_idx[ub + nu] = C;
				nu++;
			}
		}
	}
	if (!pass) { ucnt[li] = nu; wcnt[li] = nw; }
}

// X list of one cell: leaf colleagues C of an ancestor, touching parent(B)
// but not B.
template <int DIM>
__global__ void x_kernel(DevTree a, int pass, uint32_t* __restrict__ xcnt)
{
	size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (g >= a.ncells) return;
	const int L = a.lev[g];
	uint32_t nx = 0;
	const uint32_t xb = pass ? a.x_off[g] : 0;
	if (L >= 2) {
		int me[3], pc[3];
		coords<DIM>(a.code[g], me);
		int32_t A = (int32_t)(a.loff[L - 1] + a.parent[g]);
		coords<DIM>(a.code[A], pc);
		for (int l = L - 1; l >= 1; --l) {
			if (l < L - 1) A = (int32_t)(a.loff[l] + a.parent[A]);
			const int na = a.close_cnt[A];
			const int32_t* al = a.close_idx + (size_t)A * a.close_stride;
			for (int e = 0; e < na; ++e) {
				int32_t C = (int32_t)(a.loff[l] + al[e]);
				if (!a.is_leaf[C]) continue;
				int c[3];
				coords<DIM>(a.code[C], c);
				if (touch<DIM>(l, c, L - 1, pc) && !touch<DIM>(l, c, L, me)) {
					if (pass) a.x_idx[xb + nx] = C;
					nx++;
				}
			}
		}
	}
	if (!pass) xcnt[g] = nx;
}

// Candidate thresholds' counts for the uniform cells of level L (see
// LeafChooser); acc [K][LEAF_STATS].  Block row blockIdx.y = candidate k;
// each thread sums its cells (grid-stride) in registers, then one warp
// reduction and one atomic per statistic and warp.
__global__ void leaf_candidates_kernel(DevTree u, int L, const uint32_t* __restrict__ pb,
                                       const uint32_t* __restrict__ pe, const int* __restrict__ cand, int K,
                                       unsigned long long* __restrict__ acc)
{
	const int k = blockIdx.y;
	const unsigned long long m = (unsigned long long)cand[k];
	const bool last = L == u.depth - 1;
	unsigned long long v[LEAF_STATS] = {};
	for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < u.lsize[L]; c += (size_t)gridDim.x * blockDim.x) {
		const size_t g = u.loff[L] + c;
		const unsigned long long n = pe[g] - pb[g];
		unsigned long long np = 0;
		if (L > 0) {
			const size_t gp = u.loff[L - 1] + (size_t)u.parent[g];
			np = pe[gp] - pb[gp];
		}
		const bool kept = L == 0 || np > m;
		if (!kept) continue;
		const bool leaf = n <= m || last;
		v[0] += 1; v[1] += leaf; v[2] += L >= 2; v[3] += L >= 4;
		if (leaf) { v[4] += n * n; v[5] += n * np; v[6] += last ? n : 0; v[8] = v[8] > n ? v[8] : n; }
		v[7] = (unsigned long long)L;
	}
#pragma unroll
	for (int j = 0; j < LEAF_STATS; ++j) {
		unsigned long long x = v[j];
		for (int o = 16; o; o >>= 1) {
			const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
			x = j >= 7 ? (x > y ? x : y) : x + y;
		}
		if ((threadIdx.x & 31) == 0 && x) {
			if (j >= 7) atomicMax(&acc[k * LEAF_STATS + j], x);
			else atomicAdd(&acc[k * LEAF_STATS + j], x);
		}
	}
}

// Interaction counts of an adaptive tree: far (V) pairs, U entries, P2P
// particle pairs (targets x sources of the leaf and its U list), M2P
// (target, W cell) pairs.
__global__ void adaptive_counts_kernel(DevTree t, unsigned long long* out)
{
	size_t li = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long p2p = 0, m2p = 0, u = 0;
	if (li < t.nleaves) {
		size_t g = t.leaves[li];
		unsigned long long nt = t.tend[g] - t.tbeg[g];
		unsigned long long ns = t.send[g] - t.pbeg[g];
		for (uint32_t e = t.u_off[li]; e < t.u_off[li + 1]; ++e) { size_t k = t.u_idx[e]; ns += t.send[k] - t.pbeg[k]; }
		p2p = nt * ns;
		m2p = nt * (t.w_off[li + 1] - t.w_off[li]);
		u = t.u_off[li + 1] - t.u_off[li];
	}
	unsigned long long far = 0;
	for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < t.ncells; c += (size_t)gridDim.x * blockDim.x)
		far += (unsigned long long)t.far_cnt[c];
	p2p = warp_sum(p2p); m2p = warp_sum(m2p); u = warp_sum(u); far = warp_sum(far);
	if ((threadIdx.x & 31) == 0) {
		atomicAdd(out, far); atomicAdd(out + 1, u); atomicAdd(out + 2, p2p); atomicAdd(out + 3, m2p);
	}
}

template <typename T>
T* take(Context& ctx, size_t count) { return static_cast<T*>(ctx.arena.take(sizeof(T) * (count ? count : 1))); }

} // namespace

namespace {

// The uniform tree and the particle range of each of its cells (pb, pe).
int uniform_with_ranges(Context& ctx, const ParticleInput& in, int depth, DevTree& u, uint32_t*& pb, uint32_t*& pe)
{
	if (depth < 1 || depth > 16) { ctx.last_error = "adaptive tree: depth must be in [1, 16]"; return ERR_ARG; }
	int st = tree_build(ctx, in, depth, u, /*partition=*/false, /*lists=*/false);
	if (st) return st;
	pb = take<uint32_t>(ctx, u.ncells);
	pe = take<uint32_t>(ctx, u.ncells);
	if (!pb || !pe) { ctx.last_error = "adaptive tree: allocation failed"; return ERR_OOM; }
	for (int L = depth - 1; L >= 0; --L)
		uprange_kernel<<<div_up(u.lsize[L], 256), 256, 0, ctx.stream>>>(u, L, pb, pe);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

int candidate_counts(Context& ctx, const DevTree& u, const uint32_t* pb, const uint32_t* pe, const int* cand, int K,
                     unsigned long long* stats)
{
	if (K < 1 || K > LEAF_CAND_MAX) { ctx.last_error = "leaf candidates: 1 to 8 thresholds"; return ERR_ARG; }
	for (int k = 0; k < K; ++k)
		if (cand[k] < 1) { ctx.last_error = "leaf candidates: thresholds must be >= 1"; return ERR_ARG; }
	cudaStream_t s = ctx.stream;
	int* dc = take<int>(ctx, LEAF_CAND_MAX);
	unsigned long long* acc = take<unsigned long long>(ctx, LEAF_CAND_MAX * LEAF_STATS);
	if (!dc || !acc) { ctx.last_error = "leaf candidates: allocation failed"; return ERR_OOM; }
	LFMM_CUDA(ctx, cudaMemcpyAsync(dc, cand, sizeof(int) * K, cudaMemcpyHostToDevice, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * K * LEAF_STATS, s));
	for (int L = 0; L < u.depth; ++L)
		if (u.lsize[L]) {
			const dim3 grid((unsigned)std::min<size_t>(div_up(u.lsize[L], 256), 2 * (size_t)ctx.num_sms), (unsigned)K);
			leaf_candidates_kernel<<<grid, 256, 0, s>>>(u, L, pb, pe, dc, K, acc);
		}
	LFMM_CUDA(ctx, cudaMemcpyAsync(stats, acc, sizeof(unsigned long long) * K * LEAF_STATS, cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	return OK;
}

} // namespace

int leaf_candidate_stats(Context& ctx, const ParticleInput& in, int depth, const int* cand, int K,
                         unsigned long long* stats)
{
	DevTree u;
	uint32_t *pb = nullptr, *pe = nullptr;
	int st = uniform_with_ranges(ctx, in, depth, u, pb, pe);
	if (st) return st;
	return candidate_counts(ctx, u, pb, pe, cand, K, stats);
}

int tree_build_adaptive(Context& ctx, const ParticleInput& in, int depth, int max_leaf, DevTree& a,
                        LeafChooser* choose)
{
	DevTree u;
	uint32_t *pb = nullptr, *pe = nullptr;
	int st = uniform_with_ranges(ctx, in, depth, u, pb, pe);
	if (st) return st;
	if (choose) {
		unsigned long long cs[LEAF_CAND_MAX * LEAF_STATS];
		if ((st = candidate_counts(ctx, u, pb, pe, choose->cand, choose->K, cs))) return st;
		const int k = choose->pick(cs);
		if (k < 0 || k >= choose->K) { ctx.last_error = "leaf candidates: no threshold picked"; return ERR_CUDA; }
		choose->chosen = k;
		max_leaf = choose->cand[k];
	}
	cudaStream_t s = ctx.stream;
	const unsigned TB = 256;
	const size_t UC = u.ncells;
	uint8_t* keep = take<uint8_t>(ctx, UC);
	uint8_t* split = take<uint8_t>(ctx, UC);
	uint32_t* keep32 = take<uint32_t>(ctx, UC);
	uint32_t* map = take<uint32_t>(ctx, UC);
	uint32_t* tot = take<uint32_t>(ctx, MAX_LEVELS + 4);
	size_t maxl = 0;
	for (int L = 0; L < depth; ++L) maxl = std::max(maxl, u.lsize[L]);
	uint32_t* scr = take<uint32_t>(ctx, scan_scratch_words(std::max(UC, maxl)) + 64);
	if (!keep || !split || !keep32 || !map || !tot || !scr) { ctx.last_error = "adaptive tree: allocation failed"; return ERR_OOM; }
	for (int L = 0; L < depth; ++L) {
		keep_kernel<<<div_up(u.lsize[L], TB), TB, 0, s>>>(u, L, pb, pe, keep, split, keep32 + u.loff[L], max_leaf);
		scan_exclusive_u32(keep32 + u.loff[L], map + u.loff[L], u.lsize[L], tot + L, scr, s);
	}
	uint32_t ht[MAX_LEVELS];
	LFMM_CUDA(ctx, cudaMemcpyAsync(ht, tot, sizeof(uint32_t) * depth, cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	a = DevTree();
	const int dim = in.dim;
	a.dim = dim; a.depth = depth; a.n = u.n; a.nt = u.nt; a.targets_num = u.targets_num;
	a.geo = u.geo;
	a.nprob = u.nprob;
	for (int d = 0; d < 4; ++d) a.geo_host[d] = u.geo_host[d];
	a.x = u.x; a.y = u.y; a.z = u.z; a.q = u.q; a.orig = u.orig; a.pcode = u.pcode;
	a.close_stride = dim == 3 ? 26 : 8;
	a.adaptive = true; a.max_leaf = max_leaf;
	a.ncells = 0;
	int used_depth = 0;
	for (int L = 0; L < depth; ++L) {
		a.lsize[L] = ht[L];
		a.loff[L] = a.ncells;
		a.ncells += ht[L];
		if (ht[L]) used_depth = L + 1;
	}
	const size_t C = a.ncells;
	a.code = take<uint64_t>(ctx, C);
	a.beg = take<uint32_t>(ctx, C); a.end = take<uint32_t>(ctx, C);
	a.tbeg = take<uint32_t>(ctx, C); a.tend = take<uint32_t>(ctx, C);
	a.pbeg = take<uint32_t>(ctx, C); a.pend = take<uint32_t>(ctx, C); a.send = take<uint32_t>(ctx, C);
	a.parent = take<int32_t>(ctx, C);
	a.cx = take<double>(ctx, C); a.cy = take<double>(ctx, C); a.cz = dim == 3 ? take<double>(ctx, C) : nullptr;
	a.is_leaf = take<uint8_t>(ctx, C); a.lev = take<uint8_t>(ctx, C);
	a.close_cnt = take<int32_t>(ctx, C);
	a.close_idx = take<int32_t>(ctx, C * a.close_stride);
	a.far_cnt = take<int32_t>(ctx, C);
	a.x_off = take<uint32_t>(ctx, C + 1);
	uint32_t* f = take<uint32_t>(ctx, C);
	uint32_t* pos = take<uint32_t>(ctx, C + 1);
	if (!a.code || !a.close_idx || !a.x_off || !f || !pos) { ctx.last_error = "adaptive tree: allocation failed"; return ERR_OOM; }
	for (int L = 0; L < depth; ++L)
		emit_kernel<<<div_up(u.lsize[L], TB), TB, 0, s>>>(u, L, keep, split, map, pb, pe, a);
	leaf_flag_kernel<<<div_up(C, TB), TB, 0, s>>>(a, f);
	scan_exclusive_u32(f, pos, C, pos + C, scr, s);
	uint32_t nl = 0;
	LFMM_CUDA(ctx, cudaMemcpyAsync(&nl, pos + C, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	a.nleaves = nl;
	a.leaves = take<int32_t>(ctx, nl);
	a.u_off = take<uint32_t>(ctx, nl + 1);
	a.w_off = take<uint32_t>(ctx, nl + 1);
	if (!a.leaves || !a.u_off || !a.w_off) { ctx.last_error = "adaptive tree: allocation failed"; return ERR_OOM; }
	leaf_list_kernel<<<div_up(C, TB), TB, 0, s>>>(a, f, pos);
	// sources / targets inside the leaves
	if (a.targets_num > 0) {
		const size_t n = a.n;
		double* x2 = take<double>(ctx, n); double* y2 = take<double>(ctx, n);
		double* z2 = dim == 3 ? take<double>(ctx, n) : nullptr;
		double* q2 = take<double>(ctx, n); uint32_t* o2 = take<uint32_t>(ctx, n); uint64_t* c2 = take<uint64_t>(ctx, n);
		if (!x2 || !y2 || (dim == 3 && !z2) || !q2 || !o2 || !c2) { ctx.last_error = "adaptive tree: allocation failed"; return ERR_OOM; }
		source_ranges_kernel<<<div_up(C, TB), TB, 0, s>>>(a);
		partition_leaves_kernel<<<div_up(nl * 32, TB), TB, 0, s>>>(a, x2, y2, z2, q2, o2, c2);
		a.x = x2; a.y = y2; a.z = z2; a.q = q2; a.orig = o2; a.pcode = c2;
	} else {
		source_ranges_kernel<<<div_up(C, TB), TB, 0, s>>>(a);
	}
	a.depth = used_depth;   // levels below the deepest kept one are empty
	if ((st = tree_lists(ctx, a))) return st;
	// U / W per leaf, X per cell
	uint32_t* ucnt = take<uint32_t>(ctx, nl + 1);
	uint32_t* wcnt = take<uint32_t>(ctx, nl + 1);
	uint32_t* xcnt = take<uint32_t>(ctx, C + 1);
	uint32_t* tots = take<uint32_t>(ctx, 4);
	if (!ucnt || !wcnt || !xcnt || !tots) { ctx.last_error = "adaptive tree: allocation failed"; return ERR_OOM; }
	if (dim == 3) {
		uw_kernel<3><<<div_up(nl, 128), 128, 0, s>>>(a, 0, ucnt, wcnt, ctx.dev_flags);
		x_kernel<3><<<div_up(C, 128), 128, 0, s>>>(a, 0, xcnt);
	} else {
		uw_kernel<2><<<div_up(nl, 128), 128, 0, s>>>(a, 0, ucnt, wcnt, ctx.dev_flags);
		x_kernel<2><<<div_up(C, 128), 128, 0, s>>>(a, 0, xcnt);
	}
	scan_exclusive_u32(ucnt, a.u_off, nl, a.u_off + nl, scr, s);
	scan_exclusive_u32(wcnt, a.w_off, nl, a.w_off + nl, scr, s);
	scan_exclusive_u32(xcnt, a.x_off, C, a.x_off + C, scr, s);
	LFMM_CUDA(ctx, cudaMemcpyAsync(tots, a.u_off + nl, 4, cudaMemcpyDeviceToDevice, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(tots + 1, a.w_off + nl, 4, cudaMemcpyDeviceToDevice, s));
	LFMM_CUDA(ctx, cudaMemcpyAsync(tots + 2, a.x_off + C, 4, cudaMemcpyDeviceToDevice, s));
	uint32_t ht3[3];
	LFMM_CUDA(ctx, cudaMemcpyAsync(ht3, tots, 12, cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	a.n_u = ht3[0]; a.n_w = ht3[1]; a.n_x = ht3[2];
	a.u_idx = take<int32_t>(ctx, a.n_u);
	a.w_idx = take<int32_t>(ctx, a.n_w);
	a.x_idx = take<int32_t>(ctx, a.n_x);
	if (!a.u_idx || !a.w_idx || !a.x_idx) { ctx.last_error = "adaptive tree: allocation failed"; return ERR_OOM; }
	if (dim == 3) {
		uw_kernel<3><<<div_up(nl, 128), 128, 0, s>>>(a, 1, ucnt, wcnt, ctx.dev_flags);
		x_kernel<3><<<div_up(C, 128), 128, 0, s>>>(a, 1, xcnt);
	} else {
		uw_kernel<2><<<div_up(nl, 128), 128, 0, s>>>(a, 1, ucnt, wcnt, ctx.dev_flags);
		x_kernel<2><<<div_up(C, 128), 128, 0, s>>>(a, 1, xcnt);
	}
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

int tree_adaptive_counts(Context& ctx, const DevTree& t, unsigned long long* out)
{
	cudaStream_t s = ctx.stream;
	unsigned long long* dc = take<unsigned long long>(ctx, 8);
	if (!dc) { ctx.last_error = "adaptive counts: allocation failed"; return ERR_OOM; }
	LFMM_CUDA(ctx, cudaMemsetAsync(dc, 0, 32, s));
	adaptive_counts_kernel<<<div_up(std::max<size_t>(t.nleaves, 1), 256), 256, 0, s>>>(t, dc);
	LFMM_CUDA(ctx, cudaMemcpyAsync(out, dc, 32, cudaMemcpyDeviceToHost, s));
	LFMM_CUDA(ctx, cudaStreamSynchronize(s));
	return OK;
}

} // namespace lfmm
