/* orc_fmm2d.c -- TEST INFRASTRUCTURE: the 2D complex FMM of the C
 * restatement, following cpu/multipole.cpp of the reference: P2M 22-36,
 * M2M 38-53, M2L 66-84, L2L 86-97, Upward 99-177, Downward 179-231,
 * potentials 233-340, fields 342-449, constructors and Solve 451-522; pair
 * kernels common/simple_math.h:119-128. */
#include "orc_tree.h"

static void p2m2(const orc_tree* t, long long s0, long long s1, double cx, double cy, cplx* a, int N)
{
	for (int i = 1; i < N; ++i) {
		cplx acc = cmk(0.0, 0.0);
		for (long long j = s0; j < s1; ++j)
			acc = cadd(acc, cscale(cpow_u(cmk(t->x[j] - cx, t->y[j] - cy), (unsigned)i), t->q[j]));
		a[i] = cmk(-acc.re / (double)i, -acc.im / (double)i);
	}
	double s = 0.0;
	for (long long j = s0; j < s1; ++j) s += t->q[j];
	a[0] = cmk(s, 0.0);
}

/* z0 = child centre - parent centre */
static void m2m2(const cplx* a, cplx z0, cplx* b, int N)
{
	cplx w[MAXN2];
	w[0] = cmk(1.0, 0.0);
	for (int i = 1; i < N; ++i) w[i] = cmul(w[i - 1], z0);
	for (int j = 1; j < N; ++j) {
		for (int i = 1; i <= j; ++i) b[j] = cadd(b[j], cscale(cmul(a[i], w[j - i]), g_binom[j - 1][i - 1]));
		b[j] = csub(b[j], cmk((a[0].re * w[j].re - a[0].im * w[j].im) / j, (a[0].re * w[j].im + a[0].im * w[j].re) / j));
	}
	b[0] = cadd(b[0], a[0]);
}

/* z0 = source centre - target centre; b[0] takes a0 * conj(log(-z0)) */
static void m2l2(const cplx* a, cplx z0, cplx* b, int N)
{
	cplx w[MAXN2];
	w[0] = a[0];
	cplx mz = cmk(-z0.re, -z0.im);
	cplx lg = cmk(log(sqrt(mz.re * mz.re + mz.im * mz.im)), -atan2(mz.im, mz.re));
	b[0] = cadd(b[0], cmul(a[0], lg));
	for (int i = 1; i < N; ++i) {
		w[i] = cscale(cdiv(a[i], cpow_u(z0, (unsigned)i)), sgn_n(i));
		b[0] = cadd(b[0], w[i]);
	}
	for (int i = 1; i < N; ++i) {
		cplx tmp = cmk(0.0, 0.0);
		for (int j = 1; j < N; ++j) tmp = cadd(tmp, cscale(w[j], g_binom[i + j - 1][j - 1]));
		cplx num = cadd(cmk(-a[0].re / i, -a[0].im / i), tmp);
		b[i] = cadd(b[i], cdiv(num, cpow_u(z0, (unsigned)i)));
	}
}

/* b = a shifted by z0 = parent centre - child centre (overwrites b) */
static void l2l2(const cplx* a, cplx z0, cplx* b, int N)
{
	for (int i = 0; i < N; ++i) b[i] = a[i];
	for (int j = 0; j < N; ++j)
		for (int k = N - j - 1; k < N - 1; ++k) b[k] = csub(b[k], cmul(z0, b[k + 1]));
}

static int resolve_order2(int N, double eps)
{
	if (N == ORC_AUTO) { int a = (int)(-1.18 * log(1.65 * eps)); return a < MAXN2 ? a : MAXN2; }
	return N < MAXN2 ? N : MAXN2;
}
static int resolve_depth2(int depth, size_t n)
{
	if (depth == ORC_AUTO) { double d = 2 + log((double)n / 100.0) / log(4.0); if (d < 3.0) d = 3.0; return (int)d; }
	return depth;
}

static int solve2d(orc_tree* t, int N)
{
	int D = t->depth;
	t->N = N; t->ncoef = N;
	t->outer = (double**)calloc(D, sizeof(void*)); t->inner = (double**)calloc(D, sizeof(void*));
	for (int L = 0; L < D; ++L) {
		t->outer[L] = (double*)calloc(t->lsize[L] * N * 2 + 2, sizeof(double));
		t->inner[L] = (double*)calloc(t->lsize[L] * N * 2 + 2, sizeof(double));
	}
	int LL = D - 1;
#pragma omp parallel for schedule(dynamic, 16)
	for (long long c = 0; c < (long long)t->lsize[LL]; ++c)
		p2m2(t, t->sb[LL][c], t->se[LL][c], t->cx[LL][c], t->cy[LL][c], (cplx*)t->outer[LL] + c * N, N);
	for (int L = D - 2; L >= 0; --L) {
#pragma omp parallel for schedule(dynamic, 16)
		for (long long c = 0; c < (long long)t->lsize[L]; ++c)
			for (long long k = t->sb[L][c]; k < t->se[L][c]; ++k)
				m2m2((cplx*)t->outer[L + 1] + k * N, cmk(t->cx[L + 1][k] - t->cx[L][c], t->cy[L + 1][k] - t->cy[L][c]),
				     (cplx*)t->outer[L] + c * N, N);
	}
	for (int L = 2; L < D; ++L) {
#pragma omp parallel for schedule(dynamic, 16)
		for (long long c = 0; c < (long long)t->lsize[L]; ++c) {
			long long p = t->parent[L][c];
			cplx* b = (cplx*)t->inner[L] + c * N;
			l2l2((cplx*)t->inner[L - 1] + p * N, cmk(t->cx[L - 1][p] - t->cx[L][c], t->cy[L - 1][p] - t->cy[L][c]), b, N);
			for (long long e = t->far_off[L][c]; e < t->far_off[L][c + 1]; ++e) {
				long long k = t->far_idx[L][e];
				m2l2((cplx*)t->outer[L] + k * N, cmk(t->cx[L][k] - t->cx[L][c], t->cy[L][k] - t->cy[L][c]), b, N);
			}
		}
	}
	t->pot = (double*)calloc(t->n, sizeof(double));
	t->fld = (double*)calloc(2 * t->n, sizeof(double));
	int target_mode = t->targets_num != 0;
#pragma omp parallel for schedule(dynamic, 8)
	for (long long c = 0; c < (long long)t->lsize[LL]; ++c) {
		long long a0 = target_mode ? t->tb[LL][c] : t->sb[LL][c];
		long long a1 = target_mode ? t->te[LL][c] : t->se[LL][c];
		const cplx* L = (const cplx*)t->inner[LL] + c * N;
		for (long long i = a0; i < a1; ++i) {
			double xi = t->x[i], yi = t->y[i];
			double pot = 0.0, fr = 0.0, fi = 0.0;
			for (long long e = t->close_off[LL][c] - 1; e < t->close_off[LL][c + 1]; ++e) {
				long long nb = e < t->close_off[LL][c] ? c : t->close_idx[LL][e];
				for (long long j = t->sb[LL][nb]; j < t->se[LL][nb]; ++j) {
					double dx = xi - t->x[j], dy = yi - t->y[j];
					double r2 = dx * dx + dy * dy;
					if (r2 < ORC_EPS2) r2 = ORC_EPS2;
					double qj = t->q[j];
					pot += qj * 0.5 * log(r2);
					fr += qj * dx / r2; fi += qj * (-dy) / r2;
				}
			}
			/* L2P: Re sum L_k dz^k and sum k L_k dz^(k-1) */
			cplx dz = cmk(xi - t->cx[LL][c], yi - t->cy[LL][c]), pw = cmk(1.0, 0.0);
			for (int k = 0; k < N; ++k) { pot += L[k].re * pw.re - L[k].im * pw.im; pw = cmul(pw, dz); }
			pw = cmk(1.0, 0.0);
			for (int k = 1; k < N; ++k) {
				cplx term = cscale(cmul(L[k], pw), (double)k);
				fr += term.re; fi += term.im;
				pw = cmul(pw, dz);
			}
			t->pot[i] = pot; t->fld[2 * i] = fr; t->fld[2 * i + 1] = fi;
		}
	}
	return 0;
}

/* Source-only (nt == 0) or source+target 2D solve (cpu/multipole.cpp:451-471) */
void* orc_fmm2d_run(size_t ns, const double* sxy, const double* sq, size_t nt, const double* txy,
                    int N, int depth, double eps, double* pot, double* field, int* status)
{
	init_norm_tables();
	size_t n = ns + nt;
	if (n == 0) { *status = -1; return NULL; }
	double* pts = (double*)malloc(sizeof(double) * 2 * n);
	double* q = (double*)malloc(sizeof(double) * n);
	memcpy(pts, txy, sizeof(double) * 2 * nt);
	memcpy(pts + 2 * nt, sxy, sizeof(double) * 2 * ns);
	for (size_t i = 0; i < nt; ++i) q[i] = 0.0;
	memcpy(q + nt, sq, sizeof(double) * ns);
	int Nr = resolve_order2(N, eps), Dr = resolve_depth2(depth, n);
	if (Nr < 1 || Dr < 1) { free(pts); free(q); *status = -2; return NULL; }
	orc_tree* t = orc_tree_build(2, n, pts, q, Dr);
	free(pts); free(q);
	if (!t) { *status = -2; return NULL; }
	*status = solve2d(t, Nr);
	size_t nout = nt ? nt : ns;
	for (size_t i = 0; i < nout; ++i) {
		long long s = t->positions[i];
		pot[i] = t->pot[s];
		field[2 * i] = t->fld[2 * s]; field[2 * i + 1] = t->fld[2 * s + 1];
	}
	return t;
}

int orc_fmm2d(size_t ns, const double* sxy, const double* sq, size_t nt, const double* txy,
              int N, int depth, double eps, double* pot, double* field)
{
	int st = 0;
	void* h = orc_fmm2d_run(ns, sxy, sq, nt, txy, N, depth, eps, pot, field, &st);
	orc_tree_free((orc_tree*)h);
	return st;
}

void orc_run_free(void* h) { orc_tree_free((orc_tree*)h); }
