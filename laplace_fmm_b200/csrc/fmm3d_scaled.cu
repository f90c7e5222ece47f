// 3D FMM in scaled expansions on the adaptive-form tree (uniform when
// max_leaf = 0): plain FP64 or mixed (FP32 expansions and near field, FP64
// M2L accumulation on levels 2-3, FP64 tile sums and self term).
// Passes: P2M (every leaf, any level) -> M2M -> M2L (V, direction GEMMs) ->
// P2L (X) -> L2L -> leaves: P2P (self + U), M2P (W), L2P.
#include <cmath>
#include "scaled_kernels.cuh"
#include "m2l_tc.cuh"
#include <algorithm>

namespace lfmm {

using namespace scaled;

namespace {

bool g_scaled_const_ready[64] = {};

int upload_scaled_constants(Context& ctx)
{
	if (ctx.device < 0 || ctx.device >= 64) { ctx.last_error = "device index above 63"; return ERR_ARG; }
	if (g_scaled_const_ready[ctx.device]) return OK;
	float2 rec_f[NXD];
	double2 rec_d[NXD];
	float sig_f[MAXN3 + 2];
	double sig_d[MAXN3 + 2];
	for (int n = 0; n <= MAXN3; ++n)
		for (int m = 0; m <= n; ++m) {
			const int i = tix(n, m);
			const double d1 = (double)(n + 1) * (n + 1) - (double)m * m;
			rec_d[i] = make_double2((2.0 * n + 1.0) / std::sqrt(d1), std::sqrt(((double)n * n - (double)m * m) / d1));
			rec_f[i] = make_float2((float)rec_d[i].x, (float)rec_d[i].y);
		}
	sig_d[0] = 0.0;
	for (int m = 1; m <= MAXN3 + 1; ++m) sig_d[m] = -std::sqrt((2.0 * m - 1.0) / (2.0 * m));
	for (int m = 0; m <= MAXN3 + 1; ++m) sig_f[m] = (float)sig_d[m];
	float inv_f[NINV];
	double inv_d[NINV];
	inv_f[0] = 0.f; inv_d[0] = 0.0;
	for (int k = 1; k < NINV; ++k) { inv_d[k] = 1.0 / k; inv_f[k] = 1.0f / (float)k; }
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_inv_f, inv_f, sizeof(inv_f)));
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_inv_d, inv_d, sizeof(inv_d)));
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_rec_f, rec_f, sizeof(rec_f)));
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_rec_d, rec_d, sizeof(rec_d)));
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_sig_f, sig_f, sizeof(sig_f)));
	LFMM_CUDA(ctx, cudaMemcpyToSymbol(c_sig_d, sig_d, sizeof(sig_d)));
	g_scaled_const_ready[ctx.device] = true;
	return OK;
}

template <typename real> Tab<real> tables_of(const DevTables& T);
template <> Tab<double> tables_of<double>(const DevTables& T) { return Tab<double>{T.dmat, T.emat, T.m2m, T.l2l, T.knm, T.dirinfo}; }
template <> Tab<float> tables_of<float>(const DevTables& T) { return Tab<float>{T.dmat_f, T.emat_f, T.m2m_f, T.l2l_f, T.knm_f, T.dirinfo}; }

template <typename real> const real* ops_of(Context& ctx, int N);
template <> const double* ops_of<double>(Context& ctx, int N) { return m2l_ops_fp64(ctx, N, 1.0); }
template <> const float* ops_of<float>(Context& ctx, int N) { return m2l_ops_fp32(ctx, N); }

// Dense FP64 scaled M2M (OP = SOP_M2M) or L2L operators, one per child octant
// o (the octant bits of the child's code): column r is translate_scaled, the
// rotation-based shift of the SIMT kernels, applied to the r-th unit vector.
// out: [8][MT][MT], pre-zeroed.
template <int OP>
__global__ void __launch_bounds__(WPB * 32) shift_ops_kernel(int N, int MT, Tab<double> T, double* __restrict__ out,
                                                             unsigned* flags)
{
	__shared__ SmemT<double> sm[WPB];
	__shared__ double2 unit[WPB][NX2MAX];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int Nx2 = N * (N + 1) / 2, R = 2 * Nx2;
	const size_t task = (size_t)blockIdx.x * WPB + w;
	const int o = (int)(task / R), r = (int)(task % R);
	if (o >= 8) return;
	const int bx = (o >> 2) & 1, by = (o >> 1) & 1, bz = o & 1;
	const int d = OP == SOP_M2M ? dir_id(2 * bx - 1, 2 * by - 1, 2 * bz - 1) : dir_id(1 - 2 * bx, 1 - 2 * by, 1 - 2 * bz);
	for (int c = lane; c < Nx2; c += 32)
		unit[w][c] = make_double2(c == r / 2 && !(r & 1) ? 1.0 : 0.0, c == r / 2 && (r & 1) ? 1.0 : 0.0);
	__syncwarp();
	double2 acc[CMAX];
#pragma unroll
	for (int k = 0; k < CMAX; ++k) acc[k] = make_double2(0.0, 0.0);
	translate_scaled<OP, double>(unit[w], d, acc, N, Nx2, sm[w], T, flags);
	double* op = out + (size_t)o * MT * MT;
#pragma unroll
	for (int k = 0; k < CMAX; ++k) {
		const int c = lane + 32 * k;
		if (c < Nx2) {
			op[(size_t)(2 * c) * MT + r] = acc[k].x;
			op[(size_t)(2 * c + 1) * MT + r] = acc[k].y;
		}
	}
}

// Moves the diagonal of the 8 FP64 operators [8][MT][MT] into diag [8][MT]
// (FP32; zero past R) and zeroes it in the operators.
__global__ void split_diag_kernel(double* __restrict__ ops64, int MT, int R, float* __restrict__ diag)
{
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= 8 * MT) return;
	const int o = e / MT, c = e % MT;
	double* p = ops64 + ((size_t)o * MT + c) * MT + c;
	diag[e] = c < R ? (float)*p : 0.f;
	*p = 0.0;
}

// The tensor-core M2M (op 0) or L2L (op 1, followed by its diagonal) operators
// of order N, cached in the context (built once; the plan's warm solves build
// them before capture).  nullptr on failure, with st = ERR_OOM or ERR_CUDA.
const uint4* shift_ops_tc(Context& ctx, int N, int op, int& st)
{
	st = OK;
	const int tag = 30 + op;
	for (auto& e : ctx.opcache)
		if (e.N == N && e.prec == tag) { e.stamp = ++ctx.opcache_clock; return static_cast<const uint4*>(e.ptr); }
	const int MT = m2l_padded(N), R = N * (N + 1);
	const size_t bytes64 = sizeof(double) * 8 * (size_t)MT * MT;
	const size_t bytes_tc = tc_ops_bytes(8, N) + (op == 1 ? sizeof(float) * 8 * MT : 0);
	opcache_make_room(ctx);
	double* d = nullptr;
	void* tc = nullptr;
	if (cudaMalloc(&d, bytes64) != cudaSuccess || cudaMalloc(&tc, bytes_tc) != cudaSuccess) {
		cudaGetLastError();
		if (d) cudaFree(d);
		ctx.last_error = "shift operators: out of memory";
		st = ERR_OOM;
		return nullptr;
	}
	const Tab<double> T = tables_of<double>(ctx.tables.d);
	const size_t tasks = (size_t)8 * R;
	cudaMemsetAsync(d, 0, bytes64, ctx.stream);
	if (op == 0) {
		shift_ops_kernel<SOP_M2M><<<div_up(tasks, WPB), WPB * 32, 0, ctx.stream>>>(N, MT, T, d, ctx.dev_flags);
	} else {
		shift_ops_kernel<SOP_L2L><<<div_up(tasks, WPB), WPB * 32, 0, ctx.stream>>>(N, MT, T, d, ctx.dev_flags);
		split_diag_kernel<<<div_up(8 * MT, 256), 256, 0, ctx.stream>>>(
			d, MT, R, reinterpret_cast<float*>(static_cast<uint8_t*>(tc) + tc_ops_bytes(8, N)));
	}
	st = cudaGetLastError() == cudaSuccess ? tc_ops_convert(ctx, d, 8, N, tc) : ERR_CUDA;
	if (cudaStreamSynchronize(ctx.stream) != cudaSuccess) st = ERR_CUDA;
	cudaFree(d);
	if (st != OK) {
		cudaFree(tc);
		ctx.last_error = "shift operators: build failed";
		return nullptr;
	}
	OpCacheEntry e;
	e.N = N; e.prec = tag; e.h = 1.0; e.bytes = bytes_tc;
	e.stamp = ++ctx.opcache_clock; e.ptr = tc;
	ctx.opcache.push_back(e);
	return static_cast<const uint4*>(tc);
}

// M2M plan of level L for the tensor-core engine: the non-leaf cells (order,
// one class; a leaf keeps its P2M expansion) and their children by octant
// (vtab[cell][8]: level-local index at L + 1, or -1).
__global__ void m2m_plan_kernel(DevTree t, int L, int32_t* __restrict__ vtab, int32_t* __restrict__ order,
                                uint32_t* __restrict__ count)
{
	const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= t.lsize[L]) return;
	const size_t g = t.loff[L] + c, cb = t.loff[L + 1];
	if (t.beg[g] >= t.end[g]) return;
	for (uint32_t k = t.beg[g]; k < t.end[g]; ++k) vtab[c * 8 + (size_t)(t.code[cb + k] & 7ull)] = (int32_t)k;
	order[atomicAdd(count, 1u)] = (int32_t)c;
}

int m2m_plan_build(Context& ctx, const DevTree& t, int L, M2LPlan& plan)
{
	const size_t m = t.lsize[L];
	plan.cells = m;
	plan.vtab = static_cast<int32_t*>(ctx.arena.take(sizeof(int32_t) * 8 * m));
	plan.order = static_cast<int32_t*>(ctx.arena.take(sizeof(int32_t) * m));
	plan.oct_count = static_cast<uint32_t*>(ctx.arena.take(sizeof(uint32_t) * 8));
	if (!plan.vtab || !plan.order || !plan.oct_count) { ctx.last_error = "m2m plan: allocation failed"; return ERR_OOM; }
	LFMM_CUDA(ctx, cudaMemsetAsync(plan.vtab, 0xff, sizeof(int32_t) * 8 * m, ctx.stream));
	LFMM_CUDA(ctx, cudaMemsetAsync(plan.oct_count, 0, sizeof(uint32_t) * 8, ctx.stream));
	m2m_plan_kernel<<<div_up(m, 256), 256, 0, ctx.stream>>>(t, L, plan.vtab, plan.order, plan.oct_count);
	LFMM_CUDA(ctx, cudaGetLastError());
	return OK;
}

template <typename real>
int solve_t(Context& ctx, const DevTree& t, int N, double* pot, double* field, SolveStats* stats,
            const int* level_N)
{
	using v2 = typename V2<real>::t;
	cudaStream_t s = ctx.stream;
	const bool timing = ctx.timing != 0;
	const int Nx2 = N * (N + 1) / 2, R = 2 * Nx2;
	const size_t n = t.n, C = t.ncells;
	const Tab<real> T = tables_of<real>(ctx.tables.d);
	const real* knm = T.knm;
	real* xr = static_cast<real*>(ctx.arena.take(sizeof(real) * n));
	real* yr = static_cast<real*>(ctx.arena.take(sizeof(real) * n));
	real* zr = static_cast<real*>(ctx.arena.take(sizeof(real) * n));
	real* qr = static_cast<real*>(ctx.arena.take(sizeof(real) * n));
	v2* outer = static_cast<v2*>(ctx.arena.take(sizeof(v2) * C * Nx2));
	v2* inner = static_cast<v2*>(ctx.arena.take(sizeof(v2) * C * Nx2));
	size_t bmax = 0;
	for (int L = 0; L < t.depth; ++L) bmax = std::max(bmax, t.lsize[L]);
	const bool coarse64 = sizeof(real) == sizeof(float);
	double* cv_in = coarse64 ? static_cast<double*>(ctx.arena.take(sizeof(double) * bmax * R)) : nullptr;
	double* cv_out = coarse64 ? static_cast<double*>(ctx.arena.take(sizeof(double) * bmax * R)) : nullptr;
	if (!xr || !yr || !zr || !qr || !outer || !inner || (coarse64 && (!cv_in || !cv_out))) {
		ctx.last_error = "scaled solve: allocation failed";
		return ERR_OOM;
	}
	const size_t n_out = t.nt ? t.nt : t.n - t.nt;
	LFMM_CUDA(ctx, cudaMemsetAsync(pot, 0, sizeof(double) * n_out, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(field, 0, sizeof(double) * 3 * n_out, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(outer, 0, sizeof(v2) * C * Nx2, s));
	LFMM_CUDA(ctx, cudaMemsetAsync(inner, 0, sizeof(v2) * C * Nx2, s));
	const unsigned nl = (unsigned)t.nleaves;
	relcoords_kernel<real><<<nl, 128, 0, s>>>(t, xr, yr, zr, qr);
	p2m_scaled_kernel<real><<<div_up(nl, WPB), WPB * 32, 0, s>>>(t, xr, yr, zr, qr, N, knm, outer);
	int st;
	// the FP32 levels' shifts on the tensor-core engine (dense scaled operators,
	// one per child octant), else the rotation-based SIMT kernels
	const bool tc_shift = sizeof(real) == sizeof(float) && ctx.m2l_engine == 3 && m2l_tc_supported(N);
	if (tc_shift) {
		const uint4* mops = shift_ops_tc(ctx, N, 0, st);
		if (!mops) return st;
		for (int L = t.depth - 2; L >= 0; --L) {
			if (t.lsize[L] == 0) continue;
			M2LPlan mp;
			if ((st = m2m_plan_build(ctx, t, L, mp))) return st;
			if ((st = shift_gemm_tc(ctx, TC_M2M, mp, mops, reinterpret_cast<const float*>(outer + t.loff[L + 1] * Nx2),
			                        reinterpret_cast<float*>(outer + t.loff[L] * Nx2), N, t.lsize[L + 1])))
				return st;
		}
	} else {
		for (int L = t.depth - 2; L >= 0; --L)
			m2m_scaled_kernel<real><<<div_up(t.lsize[L], WPB), WPB * 32, 0, s>>>(t, L, outer + t.loff[L + 1] * Nx2,
			                                                                     outer + t.loff[L] * Nx2, N, T,
			                                                                     ctx.dev_flags);
	}
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[2], s));
	std::vector<M2LPlan> plans(t.depth);
	if (t.depth > 2) {
		const real* ops = ops_of<real>(ctx, N);
		const double* opd = coarse64 ? m2l_ops_fp64(ctx, N, 1.0) : nullptr;
		if (!ops || (coarse64 && !opd)) return ERR_OOM;
		for (int L = 2; L < t.depth; ++L) {
			if (t.lsize[L] == 0) continue;
			M2LPlan& plan = plans[L];
			if ((st = m2l_plan_build(ctx, t, L, plan))) return st;
			const real* mL = reinterpret_cast<const real*>(outer + t.loff[L] * Nx2);
			real* lL = reinterpret_cast<real*>(inner + t.loff[L] * Nx2);
			if (coarse64 && L <= 3) {
				// FP64 accumulation on the coarse levels
				size_t m = t.lsize[L] * (size_t)R;
				convert_kernel<real><<<div_up(m, 256), 256, 0, s>>>(mL, cv_in, m);
				if ((st = m2l_gemm<double>(ctx, plan, opd, cv_in, cv_out, N))) return st;
				convert_back_kernel<real><<<div_up(m, 256), 256, 0, s>>>(cv_out, lL, m);
			} else if (sizeof(real) == sizeof(float) && ctx.m2l_engine == 3 && m2l_tc_supported(N)) {
				// tcgen05 hi/lo GEMM on the FP32 levels (FP16 or TF32 operands)
				float t_inv = 1.f;
				const uint4* tc = m2l_ops_tc(ctx, N, &t_inv);
				if (!tc) return ERR_OOM;
				if ((st = m2l_gemm_tc(ctx, plan, tc, reinterpret_cast<const float*>(mL), reinterpret_cast<float*>(lL), N,
				                      level_N ? level_N[L] : 0, t_inv)))
					return st;
			} else {
				if ((st = m2l_gemm<real>(ctx, plan, ops, mL, lL, N))) return st;
			}
		}
	}
	if (t.adaptive && t.n_x > 0)
		p2l_kernel<real><<<div_up(C, WPB), WPB * 32, 0, s>>>(t, N, knm, inner);
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[3], s));
	if (tc_shift && t.depth > 3) {
		const uint4* lops = shift_ops_tc(ctx, N, 1, st);
		if (!lops) return st;
		for (int L = 3; L < t.depth; ++L) {
			if (t.lsize[L] == 0) continue;
			// the level's cells grouped by octant (its M2L plan), one slot: the parent
			M2LPlan lp = plans[L];
			lp.vtab = t.parent + t.loff[L];
			if ((st = shift_gemm_tc(ctx, TC_L2L, lp, lops, reinterpret_cast<const float*>(inner + t.loff[L - 1] * Nx2),
			                        reinterpret_cast<float*>(inner + t.loff[L] * Nx2), N, t.lsize[L - 1])))
				return st;
		}
	} else {
		for (int L = 3; L < t.depth; ++L)
			if (t.lsize[L])
				l2l_scaled_kernel<real><<<div_up(t.lsize[L], WPB), WPB * 32, 0, s>>>(t, L, inner + t.loff[L - 1] * Nx2,
				                                                                     inner + t.loff[L] * Nx2, N, T,
				                                                                     ctx.dev_flags);
	}
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[4], s));
	if constexpr (sizeof(real) == sizeof(float)) {
		// the near field (a resident grid taking leaves from a counter), then
		// the expansions added onto it
		constexpr int LWP = 4, LWE = eval_warps<real>();
		unsigned* next_leaf = static_cast<unsigned*>(ctx.arena.take(sizeof(unsigned)));
		if (!next_leaf) { ctx.last_error = "scaled solve: allocation failed"; return ERR_OOM; }
		LFMM_CUDA(ctx, cudaMemsetAsync(next_leaf, 0, sizeof(unsigned), s));
		p2p_f32_kernel<LWP><<<6 * ctx.num_sms, LWP * 32, 0, s>>>(t, qr, pot, field, next_leaf);
		unsigned* next_eval = static_cast<unsigned*>(ctx.arena.take(sizeof(unsigned)));
		if (!next_eval) { ctx.last_error = "scaled solve: allocation failed"; return ERR_OOM; }
		LFMM_CUDA(ctx, cudaMemsetAsync(next_eval, 0, sizeof(unsigned), s));
		eval_scaled_kernel<real, LWE><<<8 * ctx.num_sms, LWE * 32, 0, s>>>(t, outer, inner, N, pot, field, next_eval);
	} else {
		constexpr int LW = leaf_warps<real>();
		leaves_scaled_kernel<real><<<div_up(nl, LW), LW * 32, 0, s>>>(t, qr, outer, inner, N, knm, pot, field);
	}
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[5], s));
	LFMM_CUDA(ctx, cudaGetLastError());
	(void)stats;
	return OK;
}

} // namespace

float* m2l_ops_fp32(Context& ctx, int N)
{
	for (auto& e : ctx.opcache)
		if (e.N == N && e.prec == 1) { e.stamp = ++ctx.opcache_clock; return static_cast<float*>(e.ptr); }
	double* d = m2l_ops_fp64(ctx, N, 1.0);
	if (!d) return nullptr;
	const int MT = m2l_padded(N);
	size_t cnt = (size_t)343 * MT * MT;
	OpCacheEntry e;
	e.N = N; e.prec = 1; e.h = 1.0; e.bytes = cnt * sizeof(float); e.stamp = ++ctx.opcache_clock;
	if (cudaMalloc(&e.ptr, e.bytes) != cudaSuccess) { cudaGetLastError(); ctx.last_error = "m2l operators: out of memory"; return nullptr; }
	convert_back_kernel<float><<<div_up(cnt, 256), 256, 0, ctx.stream>>>(d, static_cast<float*>(e.ptr), cnt);
	ctx.opcache.push_back(e);
	return static_cast<float*>(e.ptr);
}

int fmm3d_solve_scaled(Context& ctx, const ParticleInput& in, int N, int depth, int max_leaf, int precision,
                       double* pot, double* field, SolveStats* stats, DevTree* tree_out, const int* level_N)
{
	if (N < 1 || N > MAXN3) { ctx.last_error = "order out of range (1 <= N <= 18)"; return ERR_ARG; }
	if (!m2l_gemm_supported(N)) { ctx.last_error = "scaled / mixed / adaptive forms support N <= 18"; return ERR_UNSUPPORTED; }
	if (max_leaf < 0) { ctx.last_error = "max_leaf must be >= 0"; return ERR_ARG; }
	int st = upload_scaled_constants(ctx);
	if (st) return st;
	cudaStream_t s = ctx.stream;
	const bool timing = ctx.timing != 0;
	ctx.kev_used = 0;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[0], s));
	DevTree t;
	if ((st = tree_build_adaptive(ctx, in, depth, max_leaf, t))) return st;
	if (timing) LFMM_CUDA(ctx, cudaEventRecord(ctx.ev[1], s));
	if ((st = fmm3d_scaled_on_tree(ctx, t, N, precision, pot, field, stats, level_N))) return st;
	if (tree_out) *tree_out = t;
	return OK;
}

int fmm3d_scaled_on_tree(Context& ctx, const DevTree& t, int N, int precision, double* pot, double* field,
                         SolveStats* stats, const int* level_N)
{
	if (N < 1 || N > MAXN3 || !m2l_gemm_supported(N)) {
		ctx.last_error = "scaled / mixed / adaptive forms support N <= 18";
		return ERR_UNSUPPORTED;
	}
	int st = upload_scaled_constants(ctx);
	if (st) return st;
	cudaStream_t s = ctx.stream;
	const bool timing = ctx.timing != 0;
	st = precision == 1 ? solve_t<float>(ctx, t, N, pot, field, stats, level_N)
	                    : solve_t<double>(ctx, t, N, pot, field, stats, level_N);
	if (st) return st;
	if (stats) {
		unsigned long long h[4];
		if ((st = tree_adaptive_counts(ctx, t, h))) return st;
		stats->N = N; stats->depth = t.depth;
		stats->n_particles = t.n; stats->n_cells = t.ncells; stats->n_leaves = t.nleaves;
		stats->targets_num = t.targets_num;
		stats->n_far_pairs = h[0]; stats->n_close_pairs = h[1]; stats->n_p2p_pairs = h[2];
		stats->n_m2p = h[3]; stats->n_w = t.n_w; stats->n_x = t.n_x;
		if (timing) {
			cudaEventElapsedTime(&stats->ms_tree, ctx.ev[0], ctx.ev[1]);
			cudaEventElapsedTime(&stats->ms_upward, ctx.ev[1], ctx.ev[2]);
			cudaEventElapsedTime(&stats->ms_m2l, ctx.ev[2], ctx.ev[3]);
			cudaEventElapsedTime(&stats->ms_l2l, ctx.ev[3], ctx.ev[4]);
			cudaEventElapsedTime(&stats->ms_leaves, ctx.ev[4], ctx.ev[5]);
			cudaEventElapsedTime(&stats->ms_total, ctx.ev[0], ctx.ev[5]);
			for (int k = 0; k + 1 < ctx.kev_used; k += 2) {
				float ms = 0.f;
				cudaEventElapsedTime(&ms, ctx.kev[k], ctx.kev[k + 1]);
				stats->ms_m2l_kernel += ms;
				++stats->n_m2l_kernel;
			}
		}
	}
	return OK;
}

} // namespace lfmm
