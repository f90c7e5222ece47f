/* orc_fmm3d.c -- TEST INFRASTRUCTURE: the 3D rotation-based FMM of the C
 * restatement, following cpu/multipole3d.cpp of the reference:
 * P2M 20-49, RotateZ/RotateY 51-113, M2M 115-150, M2L 152-190, L2L 192-226,
 * Upward 228-318, Downward 320-412, leaves (P2P 885-1151, L2P 1152-1208),
 * constructors and Solve 1296-1374. */
#include "orc_tree.h"

/* b += a * e^{i m phi}  (RotateZ, cpu/multipole3d.cpp:66-77) */
static void rotate_z_acc(const cplx* a, const double* e, cplx* b, int N)
{
	for (int n = 0; n < N; ++n)
		for (int m = 0; m <= n; ++m)
			b[TIX(n, m)] = cadd(b[TIX(n, m)], cmul(a[TIX(n, m)], cmk(e[2 * m], e[2 * m + 1])));
}
/* b += a * conj-table (the table for -phi holds cos(m phi), -sin(m phi)) */

/* res[n,m] = d(n,m,0) a[n,0] + sum_k (Re a[n,k](d_{m,k}+d_{m,-k}), Im a[n,k](d_{m,k}-d_{m,-k}))
 * (RotateY, cpu/multipole3d.cpp:79-113) */
static void rotate_y(const cplx* a, const double* D, cplx* res, int N)
{
	for (int n = 0; n < N; ++n)
		for (int m = 0; m <= n; ++m) {
			double vr = 0.0, vi = 0.0;
			for (int k = 1; k <= n; ++k) {
				double z1 = D[DIX(n, m, k)], z2 = D[DIX(n, m, -k)];
				cplx w = a[TIX(n, k)];
				vr = w.re * (z1 + z2) + vr;
				vi = w.im * (z1 - z2) + vi;
			}
			double d0 = D[DIX(n, m, 0)];
			vr += d0 * a[TIX(n, 0)].re;
			vi += d0 * a[TIX(n, 0)].im;
			res[TIX(n, m)] = cmk(vr, vi);
		}
}

enum { OP_M2M = 0, OP_M2L = 1, OP_L2L = 2 };

/* rotate to the z-axis of p0, translate along z, rotate back, accumulate */
static int translate(int op, const cplx* a, double px, double py, double pz, cplx* b, int N, cplx* w1, cplx* w2)
{
	int Nx2 = N * (N + 1) / 2;
	double rho, th, ph;
	dec_to_sph(px, py, pz, &rho, &th, &ph);
	const double* dm1 = dtab_for(th);
	const double* dm2 = dtab_for(-th);
	const double* e1 = etab_for(ph);
	const double* e2 = etab_for(-ph);
	if (!dm1 || !dm2 || !e1 || !e2) return -1;
	memset(w2, 0, sizeof(cplx) * Nx2);
	rotate_z_acc(a, e1, w2, N);
	rotate_y(w2, dm1, w1, N);
	memset(w2, 0, sizeof(cplx) * Nx2);
	double rn[2 * MAXN3 + 1];
	if (op == OP_M2L) {
		rn[0] = 1.0;
		for (int i = 1; i < 2 * N + 1; ++i) rn[i] = rn[i - 1] / rho;
		for (int j = 0; j < N; ++j)
			for (int k = 0; k <= j; ++k) {
				cplx acc = w2[TIX(j, k)];
				for (int n = k; n < N; ++n)
					acc = cadd(acc, cscale(w1[TIX(n, k)], m2lcoef(j, k, n) * rn[j + n + 1]));
				w2[TIX(j, k)] = acc;
			}
	} else if (op == OP_M2M) {
		rn[0] = 1.0;
		for (int i = 1; i < N; ++i) rn[i] = rn[i - 1] * rho;
		for (int j = 0; j < N; ++j)
			for (int k = 0; k <= j; ++k)
				for (int n = 0; j - n >= k; ++n) {
					int jm = j - n;
					double c = Anm(n, 0) * Anm(jm, k) * rn[n] / Anm(j, k);
					w2[TIX(j, k)] = cadd(w2[TIX(j, k)], cscale(w1[TIX(jm, k)], c));
				}
	} else {
		rn[0] = 1.0;
		for (int i = 1; i < N; ++i) rn[i] = rn[i - 1] * rho;
		for (int j = 0; j < N; ++j)
			for (int k = 0; k <= j; ++k)
				for (int n = j; n < N; ++n) {
					double c = Anm(n - j, 0) * Anm(j, k) * sgn_n(n + j) * rn[n - j] / Anm(n, k);
					w2[TIX(j, k)] = cadd(w2[TIX(j, k)], cscale(w1[TIX(n, k)], c));
				}
	}
	rotate_y(w2, dm2, w1, N);
	rotate_z_acc(w1, e2, b, N);
	return 0;
}

/* P2M for one cell (cpu/multipole3d.cpp:20-49) */
static void p2m(const orc_tree* t, long long s0, long long s1, double cx, double cy, double cz, cplx* a, int N)
{
	double P[(MAXN3 + 1) * (MAXN3 + 2) / 2];
	cplx eim[MAXN3 + 1];
	for (long long i = s0; i < s1; ++i) {
		double r, th, ph;
		dec_to_sph(t->x[i] - cx, t->y[i] - cy, t->z[i] - cz, &r, &th, &ph);
		double rn = r;
		compute_pnm(N, th, P);
		for (int m = 0; m < N; ++m) eim[m] = cmk(cos(m * ph), -sin(m * ph));
		double q = t->q[i];
		for (int n = 1; n < N; ++n) {
			for (int m = 0; m <= n; ++m)
				a[TIX(n, m)] = cadd(a[TIX(n, m)], cscale(eim[m], q * rn * Knm(n, m) * P[TIX(n, m)]));
			rn *= r;
		}
		a[0].re += q;
	}
}

/* L2P for one target (cpu/multipole3d.cpp:1152-1208) */
static void l2p(const cplx* L, double px, double py, double pz, double cx, double cy, double cz, int N,
                double* pot, double* f)
{
	double P[(MAXN3 + 2) * (MAXN3 + 3) / 2];
	cplx eim[MAXN3 + 2];
	double r, th, ph;
	dec_to_sph(px - cx, py - cy, pz - cz, &r, &th, &ph);
	compute_pnm(N + 1, th, P);
	for (int m = 0; m <= N; ++m) eim[m] = cmk(cos(m * ph), sin(m * ph));
	double x = cos(th), y = sin(th), rn = 1. / r;
	double phi = 0.0, mt0 = 0.0, mt1 = 0.0, mt2 = 0.0;
	for (int n = 0; n < N; ++n) {
		for (int m = 0; m <= n; ++m) {
			double mult = m ? 2.0 : 1.0;
			cplx Y = cscale(eim[m], P[TIX(n, m)] * Knm(n, m));
			cplx coef = cscale(L[TIX(n, m)], rn);
			cplx yc = cmul(Y, coef);
			phi += mult * (r * yc.re);
			cplx dth = cscale(eim[m], Knm(n, m) * ((1 - m + n) * P[TIX(n + 1, m)] - (n + 1) * x * P[TIX(n, m)]) / y);
			cplx dph = cmk(-m * Y.im, m * Y.re);
			mt0 -= mult * (n * yc.re);
			mt1 -= mult * cmul(coef, dth).re;
			mt2 -= mult * cmul(coef, dph).re;
		}
		rn *= r;
	}
	*pot += phi;
	double s1 = sin(th), c1 = cos(th), s2 = sin(ph), c2 = cos(ph);
	f[0] += mt0 * s1 * c2 + mt1 * c1 * c2 - mt2 * s2 / s1;
	f[1] += mt0 * s1 * s2 + mt1 * c1 * s2 + mt2 * c2 / s1;
	f[2] += mt0 * c1 - mt1 * s1;
}

/* q_j / max(r, 1e-4) and q_j (r_i - r_j) / max(r, 1e-4)^3, via 1/max(r^2, eps^2)
 * as common/avx.h:128-146 */
static inline void p2p_pair(double xi, double yi, double zi, double xj, double yj, double zj, double qj,
                            double* pot, double* f)
{
	double dx = xi - xj, dy = yi - yj, dz = zi - zj;
	double r2 = dx * dx + dy * dy + dz * dz;
	if (r2 < ORC_EPS2) r2 = ORC_EPS2;
	double inv2 = 1.0 / r2, inv = sqrt(inv2);
	double qi = qj * inv, qi3 = inv2 * qi;
	*pot += qi;
	f[0] += dx * qi3; f[1] += dy * qi3; f[2] += dz * qi3;
}

static int resolve_order3(int N, double eps)
{
	if (eps < 1.e-11) eps = 1.e-11;
	if (N == ORC_AUTO) { int a = (int)(54.2 - 10.73 * sqrt(log(2.4 * eps) + 25.5)); return a < MAXN3 ? a : MAXN3; }
	return N < MAXN3 ? N : MAXN3;
}
static int resolve_depth3(int depth, size_t n)
{
	if (depth == ORC_AUTO) { double d = 1 + log((double)n / 100.0) / log(8.0); if (d < 2.0) d = 2.0; return (int)d; }
	return depth;
}

/* full solve on a built tree; outputs in tree order (t->pot, t->fld) */
static int solve3d(orc_tree* t, int N)
{
	init_direction_tables();
	int D = t->depth, Nx2 = N * (N + 1) / 2;
	t->N = N; t->ncoef = Nx2;
	t->outer = (double**)calloc(D, sizeof(void*)); t->inner = (double**)calloc(D, sizeof(void*));
	for (int L = 0; L < D; ++L) {
		t->outer[L] = (double*)calloc(t->lsize[L] * Nx2 * 2 + 2, sizeof(double));
		t->inner[L] = (double*)calloc(t->lsize[L] * Nx2 * 2 + 2, sizeof(double));
	}
	int err = 0;
	int LL = D - 1;
	/* upward */
#pragma omp parallel for schedule(dynamic, 16)
	for (long long c = 0; c < (long long)t->lsize[LL]; ++c)
		p2m(t, t->sb[LL][c], t->se[LL][c], t->cx[LL][c], t->cy[LL][c], t->cz[LL][c], (cplx*)t->outer[LL] + c * Nx2, N);
	for (int L = D - 2; L >= 0; --L) {
#pragma omp parallel for schedule(dynamic, 16) reduction(|:err)
		for (long long c = 0; c < (long long)t->lsize[L]; ++c) {
			cplx w1[MAXN3 * (MAXN3 + 1) / 2], w2[MAXN3 * (MAXN3 + 1) / 2];
			for (long long k = t->sb[L][c]; k < t->se[L][c]; ++k)
				err |= translate(OP_M2M, (cplx*)t->outer[L + 1] + k * Nx2, t->cx[L + 1][k] - t->cx[L][c],
				                 t->cy[L + 1][k] - t->cy[L][c], t->cz[L + 1][k] - t->cz[L][c],
				                 (cplx*)t->outer[L] + c * Nx2, N, w1, w2);
		}
	}
	/* downward: M2L on levels 2..D-1, then L2L on levels 3..D-1 */
	for (int L = 2; L < D; ++L) {
#pragma omp parallel for schedule(dynamic, 16) reduction(|:err)
		for (long long c = 0; c < (long long)t->lsize[L]; ++c) {
			cplx w1[MAXN3 * (MAXN3 + 1) / 2], w2[MAXN3 * (MAXN3 + 1) / 2];
			for (long long e = t->far_off[L][c]; e < t->far_off[L][c + 1]; ++e) {
				long long k = t->far_idx[L][e];
				err |= translate(OP_M2L, (cplx*)t->outer[L] + k * Nx2, t->cx[L][k] - t->cx[L][c],
				                 t->cy[L][k] - t->cy[L][c], t->cz[L][k] - t->cz[L][c],
				                 (cplx*)t->inner[L] + c * Nx2, N, w1, w2);
			}
		}
	}
	for (int L = 3; L < D; ++L) {
#pragma omp parallel for schedule(dynamic, 16) reduction(|:err)
		for (long long c = 0; c < (long long)t->lsize[L]; ++c) {
			cplx w1[MAXN3 * (MAXN3 + 1) / 2], w2[MAXN3 * (MAXN3 + 1) / 2];
			long long p = t->parent[L][c];
			err |= translate(OP_L2L, (cplx*)t->inner[L - 1] + p * Nx2, t->cx[L - 1][p] - t->cx[L][c],
			                 t->cy[L - 1][p] - t->cy[L][c], t->cz[L - 1][p] - t->cz[L][c],
			                 (cplx*)t->inner[L] + c * Nx2, N, w1, w2);
		}
	}
	if (err) return -3;
	/* leaves: P2P over own leaf + full close list, then L2P */
	t->pot = (double*)calloc(t->n, sizeof(double));
	t->fld = (double*)calloc(3 * t->n, sizeof(double));
	int target_mode = t->targets_num != 0;
#pragma omp parallel for schedule(dynamic, 8)
	for (long long c = 0; c < (long long)t->lsize[LL]; ++c) {
		long long a0 = target_mode ? t->tb[LL][c] : t->sb[LL][c];
		long long a1 = target_mode ? t->te[LL][c] : t->se[LL][c];
		for (long long i = a0; i < a1; ++i) {
			double pot = 0.0, f[3] = { 0.0, 0.0, 0.0 };
			double xi = t->x[i], yi = t->y[i], zi = t->z[i];
			for (long long j = t->sb[LL][c]; j < t->se[LL][c]; ++j)
				p2p_pair(xi, yi, zi, t->x[j], t->y[j], t->z[j], t->q[j], &pot, f);
			for (long long e = t->close_off[LL][c]; e < t->close_off[LL][c + 1]; ++e) {
				long long nb = t->close_idx[LL][e];
				for (long long j = t->sb[LL][nb]; j < t->se[LL][nb]; ++j)
					p2p_pair(xi, yi, zi, t->x[j], t->y[j], t->z[j], t->q[j], &pot, f);
			}
			l2p((cplx*)t->inner[LL] + c * Nx2, xi, yi, zi, t->cx[LL][c], t->cy[LL][c], t->cz[LL][c], N, &pot, f);
			t->pot[i] = pot;
			t->fld[3 * i] = f[0]; t->fld[3 * i + 1] = f[1]; t->fld[3 * i + 2] = f[2];
		}
	}
	return 0;
}

/* Source-only (nt == 0) or source+target solve, the reference's
 * FastMultipole3d<double> constructors (cpu/multipole3d.cpp:1296-1319).
 * Returns a handle that keeps the tree and expansions for inspection. */
void* orc_fmm3d_run(size_t ns, const double* sxyz, const double* sq, size_t nt, const double* txyz,
                    int N, int depth, double eps, double* pot, double* field, int* status)
{
	init_norm_tables();
	size_t n = ns + nt;
	if (n == 0) { *status = -1; return NULL; }
	double* pts = (double*)malloc(sizeof(double) * 3 * n);
	double* q = (double*)malloc(sizeof(double) * n);
	memcpy(pts, txyz, sizeof(double) * 3 * nt);
	memcpy(pts + 3 * nt, sxyz, sizeof(double) * 3 * ns);
	for (size_t i = 0; i < nt; ++i) q[i] = 0.0;
	memcpy(q + nt, sq, sizeof(double) * ns);
	int Nr = resolve_order3(N, eps), Dr = resolve_depth3(depth, n);
	if (Nr < 1 || Dr < 1) { free(pts); free(q); *status = -2; return NULL; }
	orc_tree* t = orc_tree_build(3, n, pts, q, Dr);
	free(pts); free(q);
	if (!t) { *status = -2; return NULL; }
	int st = solve3d(t, Nr);
	*status = st;
	if (st) { orc_tree_free(t); return NULL; }
	size_t nout = nt ? nt : ns;
	for (size_t i = 0; i < nout; ++i) {
		long long s = t->positions[i];
		pot[i] = t->pot[s];
		field[3 * i] = t->fld[3 * s]; field[3 * i + 1] = t->fld[3 * s + 1]; field[3 * i + 2] = t->fld[3 * s + 2];
	}
	return t;
}

int orc_fmm3d(size_t ns, const double* sxyz, const double* sq, size_t nt, const double* txyz,
              int N, int depth, double eps, double* pot, double* field)
{
	int st = 0;
	void* h = orc_fmm3d_run(ns, sxyz, sq, nt, txyz, N, depth, eps, pot, field, &st);
	orc_tree_free((orc_tree*)h);
	return st;
}

/* expansions of a run handle, level L, complex interleaved (tests) */
int orc_run_expansions(void* h, int L, double* outer, double* inner)
{
	orc_tree* t = (orc_tree*)h;
	size_t m = t->lsize[L] * t->ncoef * 2;
	memcpy(outer, t->outer[L], sizeof(double) * m);
	memcpy(inner, t->inner[L], sizeof(double) * m);
	return t->ncoef;
}
int orc_run_order(void* h) { return ((orc_tree*)h)->N; }
int orc_run_depth(void* h) { return ((orc_tree*)h)->depth; }

/* single-operator entry points (per-operator tests) */
int orc_op3d(int op, int N, const double* a, double px, double py, double pz, double* b)
{
	init_norm_tables(); init_direction_tables();
	cplx w1[MAXN3 * (MAXN3 + 1) / 2], w2[MAXN3 * (MAXN3 + 1) / 2];
	return translate(op, (const cplx*)a, px, py, pz, (cplx*)b, N, w1, w2);
}
