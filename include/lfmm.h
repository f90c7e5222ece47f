/*
 * lfmm.h -- C ABI of the B200 (sm_100a) Laplace fast multipole method.
 *
 * Drop-in boundary for the reference's solver classes: every entry point
 * takes plain pointers and sizes, returns an int status (0 = success, < 0 =
 * error, message via lfmm_last_error), never throws or aborts.  One context
 * per host thread; a context owns a CUDA stream, a device arena reused across
 * solves, and the rotation tables (the reference's process-global
 * InitMathConstants / cudaCopyMathConstants state, made per-context).
 *
 * Reference interfaces replaced (paths relative to the reference's src/):
 *   lfmm3d_solve   fmm::gpu::FastMultipole3d<double>(particles, eps, N, tree_depth)
 *                  cuda/multipole3d.h:16, and the source/target overload :17;
 *                  the CPU twins cpu/multipole3d.h:19-21
 *   lfmm2d_solve   fmm::gpu::FastMultipole(particles, eps, N, tree_depth)
 *                  cuda/multipole.h:11, source/target overload :12;
 *                  CPU twins cpu/multipole.h:13-15
 *   lfmm3d_direct / lfmm2d_direct
 *                  fmm::gpu::ComputeExact<Potential3d|Force3d|Potential2d|Force2d>
 *                  common/simple_math.h:283-313 (common/simple_math.cu:25-130)
 *   lfmm_tree_*    fmm::MortonTree<dim,...> public members (levels, level_sizes,
 *                  positions_map, closeneighbours, farneighbours),
 *                  cpu/morton_tree.h:24-45
 *
 * Conventions kept from the reference:
 *   - N is the number of degrees (order p = N - 1), clamped to 18 (3D) / 30
 *     (2D); LFMM_AUTO picks N from eps and the depth from the particle count
 *     with the reference's formulas (cpu/multipole3d.cpp:1328-1337,
 *     cpu/multipole.cpp:478-486).
 *   - Potential includes the self term q_i / 1e-4 (3D) or q_i log(1e-4) (2D);
 *     all distances are clamped at 1e-4.
 *   - Source+target solves: targets carry q = 0 and outputs are for targets
 *     only, in input order.  Source-only solves: outputs for every source in
 *     input order.  As in the reference, a source-only solve in which some
 *     charge is exactly 0 evaluates only the zero-charge particles.
 *   - 3D field = -grad(potential) = sum q (r_i - r_j) / |r_i - r_j|^3,
 *     xyz per particle; 2D "force" = sum q / (z_i - z_j) as (re, im).
 */
#ifndef LFMM_H
#define LFMM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LFMM_AUTO 2147483647

/* status codes */
#define LFMM_OK 0
#define LFMM_ERR_ARG (-1)
#define LFMM_ERR_CUDA (-2)
#define LFMM_ERR_OOM (-3)
#define LFMM_ERR_DEVICE (-4)
#define LFMM_ERR_UNSUPPORTED (-5)

/* precision: plain FP64 (the reference's arithmetic), or the mixed form */
#define LFMM_PRECISION_FP64 0
#define LFMM_PRECISION_MIXED 1

typedef struct lfmm_ctx lfmm_ctx;

typedef struct {
	int device;   /* CUDA device ordinal */
	int verbose;  /* 0: silent */
	int timing;   /* 1: record per-phase CUDA events into lfmm_stats */
} lfmm_options;

typedef struct {
	int order_N;            /* resolved number of degrees */
	int depth;              /* resolved tree depth (levels) */
	size_t n_particles;     /* particles in the tree (sources + targets) */
	size_t n_cells, n_leaves, targets_num;
	size_t n_far_pairs;     /* M2L interactions */
	size_t n_close_pairs;   /* leaf-leaf near-field interactions (full lists) */
	size_t n_p2p_pairs;     /* particle-particle evaluations in the near field */
	size_t n_m2p;           /* adaptive tree: target-particle x W-cell evaluations */
	size_t n_w, n_x;        /* adaptive tree: W and X list entries */
	float ms_tree, ms_upward, ms_m2l, ms_l2l, ms_leaves, ms_total; /* device time, when timing */
	float ms_m2l_kernel;    /* device time inside the M2L GEMMs, when timing (3D: the tensor-core
	                           launches of the mixed form; 2D: the FP64 GEMM of every level) */
	int n_m2l_kernel;       /* M2L GEMMs timed */
} lfmm_stats;

/* A context: its own stream, device arena and caches, on opt->device.  The
 * M2L engine is read from the environment when the context is created:
 * LFMM_M2L = tc (default; tcgen05 on the mixed form's FP32 levels), simt or
 * rotation; LFMM_M2L_TYPE = f16 (default; FP16 hi / lo operands) or tf32;
 * LFMM_M2L_GATHER = tma (default; the staged FP16 sources gathered by
 * tile::gather4) or ldg (loaded by the producer warps); LFMM_M2L_TUNE = 0
 * keeps the fixed launch rule instead of the autotuner. */
int lfmm_create(lfmm_ctx** ctx, const lfmm_options* opt);
void lfmm_destroy(lfmm_ctx* ctx);
const char* lfmm_last_error(const lfmm_ctx* ctx);
int lfmm_version(void);
/* the context's CUDA stream (cudaStream_t), for callers that order work on it */
void* lfmm_stream(lfmm_ctx* ctx);

/* Device-side checks (a list that overflowed its bound, a tensor-core wait
 * that gave up, an offset outside the operator set) set flags on the device.
 * A call that synchronises (host buffers, or device buffers with stats)
 * reports them itself as LFMM_ERR_DEVICE.  An asynchronous call (device
 * buffers without stats, lfmm3d_plan_execute) cannot: it latches its flags
 * into the context's pinned host memory when its work ends on the stream and
 * clears them on the device, so the next solve starts clean.  lfmm_check
 * synchronises the context's stream and returns LFMM_ERR_DEVICE (message in
 * lfmm_last_error) if any asynchronous call since the previous lfmm_check set
 * a flag; the results of that call are then incomplete.  No counterpart in
 * the reference, which checks nothing. */
int lfmm_check(lfmm_ctx* ctx);
/* Sets device error flags on the context's stream as a failing device-side
 * check would (flags: bit mask, nonzero), so that callers can test their
 * handling of LFMM_ERR_DEVICE without a real failure. */
int lfmm_debug_raise_flags(lfmm_ctx* ctx, unsigned flags);

/* ---- 3D ----------------------------------------------------------------
 * Host buffers.  src_xyz: n_src x 3, src_q: n_src, tgt_xyz: n_tgt x 3 (or
 * NULL with n_tgt = 0).  pot: n_out, field: n_out x 3, n_out = n_tgt ? n_tgt
 * : n_src.  Blocking: returns when the results are in the host buffers. */
int lfmm3d_solve(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                 const double* tgt_xyz, int N, int tree_depth, double eps, int precision, double* pot,
                 double* field, lfmm_stats* stats);
/* Same with device buffers; enqueued on the context's stream, returns after
 * the solve has been issued and its host-side sizing syncs are done (the
 * results are complete once the stream is synchronised).  With stats the call
 * synchronises and reports device-side check failures; without, they are
 * reported by lfmm_check. */
int lfmm3d_solve_device(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                        const double* tgt_xyz, int N, int tree_depth, double eps, int precision, double* pot,
                        double* field, lfmm_stats* stats);

/* Extended 3D solve: the reference's arguments plus the leaf size and the
 * precision.  max_leaf = 0 keeps the reference's uniform tree of depth
 * tree_depth; max_leaf > 0 builds an adaptive octree (cells split while they
 * hold more than max_leaf particles, at most tree_depth levels) with U, V, W, X
 * lists.  precision FP64 with max_leaf = 0 is the reference-parity path
 * (same as lfmm3d_solve); every other combination runs the scaled-expansion
 * solver (N <= 18). */
typedef struct {
	int N;            /* degrees (order p + 1), or LFMM_AUTO (from eps) */
	int tree_depth;   /* uniform depth / maximum adaptive depth, or LFMM_AUTO */
	int max_leaf;     /* 0: uniform tree; > 0: adaptive split threshold */
	int precision;    /* LFMM_PRECISION_FP64 or LFMM_PRECISION_MIXED */
	double eps;       /* tolerance used by LFMM_AUTO order selection */
} lfmm_solve_opts;

int lfmm3d_solve_ex(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                    const double* tgt_xyz, const lfmm_solve_opts* opts, double* pot, double* field, lfmm_stats* stats);
int lfmm3d_solve_ex_device(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                           const double* tgt_xyz, const lfmm_solve_opts* opts, double* pot, double* field,
                           lfmm_stats* stats);

/* Per-level M2L orders (no counterpart in the reference, whose order is one
 * number for the whole solve, cpu/multipole3d.cpp:1328-1331): opts as for
 * lfmm3d_solve_ex; level_N[L] (L < n_levels <= 22; 0 or >= opts->N: opts->N)
 * is the order of level L's M2L, the degrees of the source multipoles it uses,
 * on the mixed form's tensor-core levels (level 4 and finer); the expansions,
 * the shifts and the coarse FP64 levels keep opts->N degrees.  The fine levels
 * hold most of the M2L work and, for charges of either sign, the smallest
 * share of the far field's error, so they can run lower orders. */
int lfmm3d_solve_levels(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                        const double* tgt_xyz, const lfmm_solve_opts* opts, const int* level_N, int n_levels,
                        double* pot, double* field, lfmm_stats* stats);
int lfmm3d_solve_levels_device(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q,
                               size_t n_tgt, const double* tgt_xyz, const lfmm_solve_opts* opts, const int* level_N,
                               int n_levels, double* pot, double* field, lfmm_stats* stats);

/* ---- batched 3D solves (no counterpart in the reference, which solves one
 * problem per constructor call) ---------------------------------------------
 * n_prob independent problems in one solve: problem k is the sources
 * [offsets[k], offsets[k + 1]) of the concatenated arrays (offsets: host
 * array of n_prob + 1 entries, offsets[0] = 0, non-decreasing, total < 2^32).
 * One forest of octrees (each problem its own bounding box and root, as if
 * solved alone) built and solved together: every FMM pass is one launch over
 * all problems.  Results in input order.  opts as for lfmm3d_solve_ex (one N
 * for the batch; tree_depth LFMM_AUTO follows the largest problem; the
 * scaled-expansion solver). */
int lfmm3d_solve_batch(lfmm_ctx* ctx, int n_prob, const size_t* offsets, const double* src_xyz, const double* src_q,
                       const lfmm_solve_opts* opts, double* pot, double* field, lfmm_stats* stats);
int lfmm3d_solve_batch_device(lfmm_ctx* ctx, int n_prob, const size_t* offsets, const double* src_xyz,
                              const double* src_q, const lfmm_solve_opts* opts, double* pot, double* field,
                              lfmm_stats* stats);

/* ---- solve plans: one geometry, many charge vectors (no counterpart in the
 * reference, which rebuilds the tree on every solve) ------------------------
 * lfmm3d_plan_create builds the tree of the positions once (device buffers;
 * opts as for lfmm3d_solve_ex, N given explicitly, N <= 18), warms every
 * cache and captures the FMM passes in a CUDA graph on the context's stream.
 * lfmm3d_plan_execute (device buffers, input order, n_src each) enqueues: copy
 * the charges in, launch the graph, copy potential and field out; the results
 * are complete once the context's stream is synchronised.  The tree keeps the
 * creation charges' split into sources and zero-charge targets; later charges
 * only change values.  The plan uses the context's stream and operator cache:
 * destroy it before the context; executions of one plan must not overlap. */
typedef struct lfmm_plan lfmm_plan;
int lfmm3d_plan_create(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q,
                       const lfmm_solve_opts* opts, lfmm_plan** plan);
/* A plan for a batch: the forest of n_prob independent problems (offsets as
 * for lfmm3d_solve_batch, host array) built once and its FMM passes captured
 * in one CUDA graph, so that repeated batch solves with new charges skip the
 * forest's build and every host synchronisation.  opts->N and opts->max_leaf
 * must be given.  Executed and destroyed like any plan (charges, potential
 * and field in the concatenated input order). */
int lfmm3d_plan_create_batch(lfmm_ctx* ctx, int n_prob, const size_t* offsets, const double* src_xyz,
                             const double* src_q, const lfmm_solve_opts* opts, lfmm_plan** plan);
int lfmm3d_plan_execute(lfmm_plan* plan, const double* src_q, double* pot, double* field);
void lfmm3d_plan_destroy(lfmm_plan* plan);

/* ---- 2D ---------------------------------------------------------------- */
int lfmm2d_solve(lfmm_ctx* ctx, size_t n_src, const double* src_xy, const double* src_q, size_t n_tgt,
                 const double* tgt_xy, int N, int tree_depth, double eps, int precision, double* pot,
                 double* field, lfmm_stats* stats);
int lfmm2d_solve_device(lfmm_ctx* ctx, size_t n_src, const double* src_xy, const double* src_q, size_t n_tgt,
                        const double* tgt_xy, int N, int tree_depth, double eps, int precision, double* pot,
                        double* field, lfmm_stats* stats);
/* Extended 2D solve (the reference's uniform quadtree only,
 * cpu/multipole.cpp:473-522, is what max_leaf = 0 keeps): max_leaf > 0 builds
 * an adaptive quadtree (cells split while they hold more than max_leaf
 * particles, at most tree_depth levels) with U, V, W, X lists, so clustered
 * sets do not crowd a few leaves.  FP64 (the precision field is accepted and
 * runs the FP64 form); N <= 30; field as (re, im) pairs. */
int lfmm2d_solve_ex(lfmm_ctx* ctx, size_t n_src, const double* src_xy, const double* src_q, size_t n_tgt,
                    const double* tgt_xy, const lfmm_solve_opts* opts, double* pot, double* field, lfmm_stats* stats);
int lfmm2d_solve_ex_device(lfmm_ctx* ctx, size_t n_src, const double* src_xy, const double* src_q, size_t n_tgt,
                           const double* tgt_xy, const lfmm_solve_opts* opts, double* pot, double* field,
                           lfmm_stats* stats);

/* ---- FP64 direct sums (the accuracy oracle on the GPU) -------------------
 * Every target against every source, same clamp and self term as the FMM.
 * Host and device-buffer variants. */
int lfmm3d_direct(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                  const double* tgt_xyz, double* pot, double* field);
int lfmm3d_direct_device(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                         const double* tgt_xyz, double* pot, double* field);
int lfmm2d_direct(lfmm_ctx* ctx, size_t n_src, const double* src_xy, const double* src_q, size_t n_tgt,
                  const double* tgt_xy, double* pot, double* field);
int lfmm2d_direct_device(lfmm_ctx* ctx, size_t n_src, const double* src_xy, const double* src_q, size_t n_tgt,
                         const double* tgt_xy, double* pot, double* field);

/* ---- tree inspection (the reference's MortonTree members) ----------------
 * lfmm_tree_build builds the uniform tree of [targets | sources] on the
 * device (host input buffers, q = NULL means all targets) and keeps it in the
 * context until the next call.  Level L cells are read with
 * lfmm_tree_level (codes, particle / child ranges, target ranges, parents,
 * centres as dim doubles each); lists with lfmm_tree_lists (close lists are
 * the full symmetric lists; far lists in the reference's order);
 * positions[i] = tree position of input particle i. */
int lfmm_tree_build(lfmm_ctx* ctx, int dim, size_t n_src, const double* src_pts, const double* src_q, size_t n_tgt,
                    const double* tgt_pts, int tree_depth, size_t* level_sizes, size_t* targets_num);
int lfmm_tree_level(lfmm_ctx* ctx, int level, unsigned long long* code, long long* beg, long long* end,
                    long long* tbeg, long long* tend, long long* parent, double* center);
int lfmm_tree_list_sizes(lfmm_ctx* ctx, int level, long long* n_close, long long* n_far);
int lfmm_tree_lists(lfmm_ctx* ctx, int level, long long* close, long long* far);
int lfmm_tree_positions(lfmm_ctx* ctx, long long* positions);

/* ---- adaptive tree inspection (no counterpart in the reference, which
 * builds only the uniform tree) -------------------------------------------
 * lfmm_tree_build_adaptive builds the adaptive octree the solver uses
 * (host input buffers as lfmm_tree_build, 3D; tree_depth levels at most,
 * cells split while they hold more than max_leaf particles) with its U, W,
 * X lists and the V lists the M2L slot tables give, and keeps it in the
 * context until the next tree or solve call.  *n_cells, *n_leaves, and
 * list_sizes[4] = the entries of U, W, X, V.  Cells are numbered globally,
 * level by level.  lfmm_tree_adaptive_cells reads (any may be NULL) per
 * cell: level, Morton code at its level, parent (-1 for the root),
 * particle range [pbeg, pend) in tree order and its sources [pbeg, send)
 * (leaves; sources first), leaf flag; the leaves' cell indices
 * (n_leaves); positions[i] = tree position of input particle i (targets
 * first, then sources).  lfmm_tree_adaptive_lists reads one list kind in
 * CSR form: kind 0 U (rows = leaves in the order of the leaves array:
 * adjacent leaves of any level, the leaf itself excluded; P2P), 1 W (rows =
 * leaves: cells whose multipole is evaluated at the leaf's targets; M2P),
 * 2 X (rows = cells: leaves whose sources form the cell's local expansion;
 * P2L), 3 V (rows = cells: M2L sources); off has rows + 1 entries, idx
 * holds global cell indices. */
int lfmm_tree_build_adaptive(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                             const double* tgt_xyz, int tree_depth, int max_leaf, size_t* n_cells, size_t* n_leaves,
                             size_t* list_sizes);
/* The same for the adaptive quadtree of lfmm2d_solve_ex (2D points; the
 * cells and lists are read with the two calls below). */
int lfmm2d_tree_build_adaptive(lfmm_ctx* ctx, size_t n_src, const double* src_xy, const double* src_q, size_t n_tgt,
                               const double* tgt_xy, int tree_depth, int max_leaf, size_t* n_cells,
                               size_t* n_leaves, size_t* list_sizes);
int lfmm_tree_adaptive_cells(lfmm_ctx* ctx, int* level, unsigned long long* code, long long* parent,
                             long long* pbeg, long long* pend, long long* send, unsigned char* is_leaf,
                             long long* leaves, long long* positions);
int lfmm_tree_adaptive_lists(lfmm_ctx* ctx, int kind, long long* off, long long* idx);

/* ---- direct sum without allocation (no counterpart in the reference) -----
 * Same result as lfmm3d_direct_device, but the call allocates no device
 * memory: its source-chunk scratch is a static device array of
 * LFMM_DIRECT_NOALLOC_SCRATCH_BYTES per device, so calls with more than
 * LFMM_DIRECT_NOALLOC_MAX_TARGETS targets are rejected (LFMM_ERR_ARG).  For
 * callers that must not allocate inside their step (an allocator that has
 * reserved the device's memory, or a loop where cudaMalloc / cudaFree would
 * synchronise the device).  The first call on each device looks up the
 * array's address and loads the kernels a call can launch (either may load
 * the module): make it before any stream capture.  The address is cached per
 * device for the life of the process; a cudaDeviceReset invalidates it.  The
 * caller's current device is unchanged on return.  The array is shared by every context on the device, so calls
 * that overlap in time on one device race; serialise them.  Nothing in the
 * scratch needs to start at zero.  All pointers are device pointers. */
#define LFMM_DIRECT_NOALLOC_MAX_TARGETS 65536
#define LFMM_DIRECT_NOALLOC_SCRATCH_BYTES (8u << 20)
int lfmm3d_direct_device_noalloc(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q,
                                 size_t n_tgt, const double* tgt_xyz, double* pot, double* field);

/* ---- learned order selection (no counterpart in the reference) -----------
 * The reference picks one order from eps by a fixed formula
 * (cpu/multipole3d.cpp:1328-1331).  Here a small MLP (16 per-leaf features ->
 * 64 -> 64 -> 14, FP32, ReLU) predicts, for each leaf box, log10 of the RMS
 * absolute error of its outputs at the orders p = 4, 6, 8, 10, 12, 14, 16:
 * outputs 0-6 the potential's, outputs 7-13 the field's (magnitude of the
 * error vector); a solve takes the lowest p whose predicted
 * particle-weighted errors of both meet the tolerance.  All pointers to MLP
 * data are device pointers (FP32); parameters are W1[64][16] b1[64]
 * W2[64][64] b2[64] W3[14][64] b3[14]. */
#define LFMM_MLP_IN 16
#define LFMM_MLP_HIDDEN 64
#define LFMM_MLP_OUT 14
#define LFMM_MLP_PARAMS (64 * 16 + 64 + 64 * 64 + 64 + 14 * 64 + 14)

/* Y[n][14] = MLP(X[n][16]) */
int lfmm_mlp_forward(lfmm_ctx* ctx, const float* params, int n, const float* X, float* Y);
/* Masked mean-squared-error loss sum M (Y - T)^2 / sum M over T, M [n][14];
 * grad[LFMM_MLP_PARAMS]; work >= n * (14 + 128) + 2 floats; *loss on the host.
 * Synchronises. */
int lfmm_mlp_grad(lfmm_ctx* ctx, const float* params, int n, const float* X, const float* T, const float* M,
                  float* grad, float* work, float* loss);
/* One Adam step (step >= 1) on params with moments m, v. */
int lfmm_mlp_adam(lfmm_ctx* ctx, float* params, const float* grad, float* m, float* v, int step, float lr,
                  float beta1, float beta2, float eps);

/* Per-leaf features of the tree that opts describes (its tree_depth and
 * max_leaf; host buffers): feats [cap][16] in leaf order, leaf_of[n_src +
 * n_tgt] = the leaf of every input particle (targets first, then sources);
 * either may be NULL.  *n_leaves = the leaves of the tree (fails with
 * LFMM_ERR_ARG when above cap).  The features: log10 particles; log10 of
 * the far-field strength sum sqrt(n) / h over the V lists of the leaf and its
 * ancestors (n = particles of the source cell, h = cell size); level / depth;
 * log10 |U|, |W|, |X|, |V|, V-list entries of the leaf and its ancestors;
 * log10 sum |q|; log10 of sum n / h over the same V lists; rms and max
 * particle distance from the centre / cell size; log10 particles in the
 * parent, in the problem, in the U cells; log10 |dipole| / (h sum |q|). */
int lfmm3d_features(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                    const double* tgt_xyz, const lfmm_solve_opts* opts, float* feats, size_t cap, int* leaf_of,
                    size_t* n_leaves);

/* Vector charges: the reference's fmm::FastMultipole3d<Vector3d>
 * (cpu/multipole3d.h:10-24 with value = Vector3d; cpu/multipole3d.cpp:414-853):
 * field[3 i + c] = (sum_j q_j x (x_i - x_j) / max(r, 1e-4)^3)_c at every
 * target, q_j = (src_q3[3 j], src_q3[3 j + 1], src_q3[3 j + 2]).  No
 * potential (the reference computes none for vector charges).  Sources are
 * the particles with q != 0 (the reference's zero-charge rule); one tree,
 * three scalar passes combined by a cross product.  opts as lfmm3d_solve_ex
 * (max_leaf 0: the uniform tree; N <= 18); stats describe the tree and the
 * last of the three passes.  Host and device-buffer variants; the host one
 * synchronises. */
int lfmm3d_solve_vector(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q3, size_t n_tgt,
                        const double* tgt_xyz, const lfmm_solve_opts* opts, double* field, lfmm_stats* stats);
int lfmm3d_solve_vector_device(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q3,
                               size_t n_tgt, const double* tgt_xyz, const lfmm_solve_opts* opts, double* field,
                               lfmm_stats* stats);

typedef struct {
	int order_N;                /* degrees of the final solve */
	int predicted_N;            /* degrees the network chose */
	int fallback;               /* 0: the prediction passed the judge; 1: it did not, and the solve was
	                               rerun at the order picked again from predictions shifted by the
	                               measured shortfall, which passed; 2: that missed too (or no such
	                               order) and the solve was rerun at the fixed order N = 18 */
	double predicted_error;     /* the network's rel-L2 estimate of the potential at predicted_N */
	double checked_error;       /* sampled rel-L2 of the potential, self term removed (-1: no check) */
	double checked_error_field; /* the same for the field */
	int fp64_resolved;          /* problems rerun in the FP64 form at N = 18 because the mixed form
	                               missed tol even there (0 or 1 for a single solve) */
	double predicted_error_field; /* the network's rel-L2 estimate of the field at predicted_N */
	double judged_error;        /* what the judge compared with tol: the larger of the two upper
	                               confidence bounds (mean + 2 standard errors) of the sampled
	                               rel-L2 of potential and field (batches: the largest over problems) */
	int max_leaf;               /* the leaf-size threshold of the tree (picked by the threshold
	                               network when opts->max_leaf is LFMM_AUTO) */
	int order_groups;           /* batches: the distinct orders the problems were solved at (each
	                               order's problems as one forest); 1 for a single solve */
	int checked_targets;        /* the sampled outputs the final judgement used (batches: over all
	                               problems) */
} lfmm_learned_info;

/* 3D solve at the order the network picks for tolerance tol, which bounds
 * the rel-L2 of both outputs: the potential (self term removed) and the
 * field.  The FP64 direct sum is first evaluated at check_targets (>= 1)
 * outputs spread through the output range; the network predicts each leaf's
 * absolute potential and field errors at p = 4, 6, ..., 14, 16, the leaves'
 * errors over the samples' RMS potential and RMS field give the predicted
 * rel-L2 of each, and the lowest p in 4..17 at which both are within
 * 0.6 tol is solved (else N = 18).  The same samples then judge the result
 * on an upper confidence bound of each sampled rel-L2 (the ratio estimate
 * plus two standard errors, so a sample too small or too uneven to certify
 * tol does not pass).  When the bound exceeds tol while the estimate is
 * within 0.75 tol, three times more outputs (between the first ones) are
 * summed directly and the result judged again on all of them.  A solve
 * whose bound still exceeds tol is rerun once at the
 * order picked again from the predictions shifted by the shortfall measured
 * (bound over prediction), then, if that misses too, at the fixed order
 * N = 18 (the fallback); a mixed-precision solve still above tol there is
 * rerun in the FP64 form (fp64_resolved).  params: device pointer to the
 * network (LFMM_MLP_PARAMS floats, inputs unnormalised).  opts gives the
 * tree (tree_depth, max_leaf) and precision; opts->N and opts->eps are
 * ignored.  opts->max_leaf = LFMM_AUTO: the leaf-size threshold is learned
 * too -- params then holds the order network followed by the threshold
 * network (2 LFMM_MLP_PARAMS floats), which predicts the solve's time for
 * each threshold in {16, 24, 32, 48, 64, 96, 128, 192} from the counts of the
 * adaptive tree it would give (lfmm3d_leaf_features) at the reference's
 * automatic order for tol, and the fastest is built (info->max_leaf).  The
 * reference has a uniform tree and no leaf size (cpu/multipole3d.cpp:1334-1337).
 * Synchronises.  Host and device-buffer variants. */
int lfmm3d_solve_learned(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                         const double* tgt_xyz, const lfmm_solve_opts* opts, const float* params, double tol,
                         int check_targets, double* pot, double* field, lfmm_learned_info* info, lfmm_stats* stats);
int lfmm3d_solve_learned_device(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q,
                                size_t n_tgt, const double* tgt_xyz, const lfmm_solve_opts* opts,
                                const float* params, double tol, int check_targets, double* pot, double* field,
                                lfmm_learned_info* info, lfmm_stats* stats);
/* The batch at the orders the network picks for tolerance tol (as
 * lfmm3d_solve_learned; device buffers): up to check_targets sampled outputs
 * per problem, every output of a problem of at most 8192 particles (their
 * FP64 direct sums in one launch), normalise each
 * problem's prediction and judge its result (the same upper confidence
 * bounds, per problem, and the same threefold extension of the samples of a
 * problem whose estimate is within 0.75 tol but whose bound is not).  Every problem runs at its own predicted order: when
 * the problems need several, the problems of each order are solved together
 * as their own forest (order_groups in info), and the problems an order
 * left above tol are solved again together at N = 18; a problem still above
 * tol there (mixed form) is rerun alone in the FP64 form into its slice of
 * the outputs.  opts->max_leaf LFMM_AUTO: the threshold network picks the
 * leaf size for the whole batch (params as for lfmm3d_solve_learned).  info:
 * the highest order used, the largest predicted, checked and judged errors
 * over the problems, the number of FP64 reruns. */
int lfmm3d_solve_batch_learned_device(lfmm_ctx* ctx, int n_prob, const size_t* offsets, const double* src_xyz,
                                      const double* src_q, const lfmm_solve_opts* opts, const float* params,
                                      double tol, int check_targets, double* pot, double* field,
                                      lfmm_learned_info* info, lfmm_stats* stats);

/* The threshold network's inputs: for each candidate leaf-size threshold
 * cand[k] (K <= 8), 16 features of the adaptive tree it would give (counts of
 * cells, leaves, sums of squared leaf sizes ...) for a solve at order N;
 * feats [K][16] (host buffers).  No counterpart in the reference. */
int lfmm3d_leaf_features(lfmm_ctx* ctx, size_t n_src, const double* src_xyz, const double* src_q, size_t n_tgt,
                         const double* tgt_xyz, int tree_depth, int N, const int* cand, int K, float* feats);

/* ---- rotation tables (tests) --------------------------------------------
 * Wigner small-d matrix for table slot `slot` (layout n(n+1)(4n-1)/6 +
 * m(2n+1) + k + n, N = 18) and its canonical angle; returns the number of
 * slots, or < 0. */
int lfmm_wignerd_slot(lfmm_ctx* ctx, int slot, double* theta, double* d);

#ifdef __cplusplus
}
#endif

#endif /* LFMM_H */
