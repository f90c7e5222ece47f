// Uniform-depth Morton quadtree / octree on the device, bit-exact with the
// reference's MortonTree (reference cpu/morton_tree.cpp:286-493).
#pragma once
#include "context.cuh"
#include <functional>

namespace lfmm {

constexpr int MAX_LEVELS = 22;

struct DevTree {
	int dim = 3, depth = 0;
	size_t n = 0;              // particles in the tree: [targets | sources]
	size_t nt = 0;             // leading input particles that are targets (q = 0)
	size_t targets_num = 0;    // particles with q == 0 (switches P2P to target mode)
	double* geo = nullptr;     // device: shift x, y, z, scale
	double geo_host[4] = {};   // host copy
	// particles in tree order (SoA)
	double *x = nullptr, *y = nullptr, *z = nullptr, *q = nullptr;
	uint32_t* orig = nullptr;  // input index of tree particle s
	uint64_t* pcode = nullptr;
	// cells of all levels, concatenated; level L occupies [loff[L], loff[L] + lsize[L])
	size_t lsize[MAX_LEVELS] = {}, loff[MAX_LEVELS] = {};
	size_t ncells = 0;
	uint64_t* code = nullptr;
	uint32_t *beg = nullptr, *end = nullptr;    // particles (leaves) or level-local children
	uint32_t *tbeg = nullptr, *tend = nullptr;  // leaf target range
	int32_t* parent = nullptr;                  // level-local parent index
	double *cx = nullptr, *cy = nullptr, *cz = nullptr;
	// close lists, fixed stride (26 in 3D, 8 in 2D), level-local indices
	int close_stride = 26;
	int32_t* close_cnt = nullptr;
	int32_t* close_idx = nullptr;
	int32_t* far_cnt = nullptr;                 // per cell, for statistics
	size_t n_far_pairs = 0, n_close_pairs = 0;
	// adaptive form (tree_build_adaptive); global cell indices unless noted
	// forest of nprob independent problems (batched solves): the problem index
	// sits above the Morton bits of every code, geo holds 4 doubles per problem
	int nprob = 1;
	bool adaptive = false;
	int max_leaf = 0;
	uint32_t *pbeg = nullptr, *pend = nullptr;  // particles of every cell
	uint32_t* send = nullptr;                   // leaves: sources are [pbeg, send)
	uint8_t* is_leaf = nullptr;
	uint8_t* lev = nullptr;
	int32_t* leaves = nullptr;                  // global indices of the leaves
	size_t nleaves = 0;
	uint32_t *u_off = nullptr, *w_off = nullptr; // per leaf (position in leaves[]), CSR
	int32_t *u_idx = nullptr, *w_idx = nullptr;  // global cell indices
	uint32_t* x_off = nullptr;                  // per cell, CSR
	int32_t* x_idx = nullptr;                   // global indices of leaves
	size_t n_u = 0, n_w = 0, n_x = 0;
};

// Input particles: targets (nt, q = 0) followed by sources (ns, with q).
// nprob > 1: the sources are nprob independent problems, problem k at
// [poff[k], poff[k + 1]) (device offsets; no separate targets).
struct ParticleInput {
	int dim = 3;
	size_t ns = 0, nt = 0;
	const double* src = nullptr;   // device, ns x dim interleaved
	const double* srcq = nullptr;  // device, ns
	const double* tgt = nullptr;   // device, nt x dim interleaved
	const uint32_t* poff = nullptr;
	int nprob = 1;
};

// Size of the box of cell g (level t.lev[g]) of an adaptive-form tree; the
// scale is per problem in a forest.
__device__ __forceinline__ double cell_size(const DevTree& t, size_t g)
{
	const int L = t.lev[g];
	const double scale = t.nprob > 1 ? t.geo[4 * (t.code[g] >> (t.dim * L)) + 3] : t.geo_host[3];
	return scale / (double)(1ull << L);
}

// partition: split each leaf into sources then q == 0 targets; lists: build
// the close lists and far counts.
int tree_build(Context& ctx, const ParticleInput& in, int depth, DevTree& t, bool partition = true,
               bool lists = true);

// Close lists (fixed stride) and far counts of every level from the child
// ranges; used by both builders.
int tree_lists(Context& ctx, DevTree& t);

// Adaptive octree from the uniform one: a cell is split while it holds more
// than max_leaf particles and is above level depth-1 (max_leaf = 0 splits
// every cell: the uniform tree in adaptive form).  Leaves may sit on any
// level; beg/end hold child ranges (empty for leaves), pbeg/pend particle
// ranges; U/W/X lists are built (quadtree or octree).
// Leaf-size candidates: the counts of the adaptive tree each candidate
// threshold would give, taken from the uniform tree in one pass per level
// (a cell is kept when its parent holds more than m particles -- counts only
// shrink down the tree -- and a kept cell is a leaf when it holds at most m
// or sits on the last level).  Per candidate, LEAF_STATS words: cells,
// leaves, cells on levels >= 2, cells on levels >= 4, sum over leaves of n^2,
// sum over leaves of n * n(parent), particles in last-level leaves, deepest
// kept level, largest leaf.
constexpr int LEAF_STATS = 9, LEAF_CAND_MAX = 8;
struct LeafChooser {
	int K = 0;
	int cand[LEAF_CAND_MAX] = {};
	// called with [K][LEAF_STATS] counts; returns the index of the candidate to build
	std::function<int(const unsigned long long* stats)> pick;
	int chosen = -1;     // set by tree_build_adaptive
};
int tree_build_adaptive(Context& ctx, const ParticleInput& in, int depth, int max_leaf, DevTree& t,
                        LeafChooser* choose = nullptr);
// The candidates' counts alone (no adaptive tree is built): stats [K][LEAF_STATS] on the host.
int leaf_candidate_stats(Context& ctx, const ParticleInput& in, int depth, const int* cand, int K,
                         unsigned long long* stats);

// Interaction counts of an adaptive tree (synchronises): out[0] V pairs,
// out[1] U entries, out[2] P2P particle pairs, out[3] M2P (target, cell) pairs.
int tree_adaptive_counts(Context& ctx, const DevTree& t, unsigned long long* out);

// Fill a CSR far list of level L (level-local source indices) in the
// reference's order; far_off must hold lsize[L] + 1 entries.
int tree_far_lists(Context& ctx, const DevTree& t, int L, uint32_t* far_off, int32_t* far_idx, size_t cap);

// Interaction counts (synchronises): out[0] far pairs, out[1] leaf close
// pairs (full lists), out[2] particle pairs in the near field.  dev: 3 words.
int tree_count_pairs(Context& ctx, const DevTree& t, unsigned long long* dev, unsigned long long* out);

} // namespace lfmm
