/*
 * fmm_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A plain-C, FP64 restatement of the reference's CPU Laplace FMM (2D complex
 * and 3D rotation-based), written from the published algorithm and the
 * reference's observable behaviour, used only as the checker of the CUDA
 * library (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline leg).
 * It is pinned against the reference itself (oracle/_ref/libfmmref.so, built
 * from the reference sources by oracle/Makefile) and against the committed
 * fixtures under tests/golden/.
 *
 * Reference anchors (paths relative to the reference's src/):
 *   tree / lists ........ cpu/morton_tree.cpp:48-99 (codes), 101-145 (centres),
 *                          147-208 (close/far lists), 286-493 (build, partition,
 *                          duplicate removal)
 *   special functions ... common/special_functions.h:12-31 (Pnm), 56-138
 *                          (Knm, Anm, m2lcoef); special_functions.cpp:194-381
 *                          (Wigner-d, exponent tables keyed by int(100*angle))
 *   3D operators ........ cpu/multipole3d.cpp:20-49 (P2M), 51-113 (rotations),
 *                          115-226 (M2M, M2L, L2L), 228-412 (passes),
 *                          855-1294 (P2P + L2P), 1321-1374 (Solve heuristics)
 *   2D operators ........ cpu/multipole.cpp:22-97, 99-231, 233-449, 473-522
 *   pair kernels ........ common/simple_math.h:81-216
 *
 * Differences that are deliberate and harmless at the 1e-12 parity bar:
 *   - P2P is evaluated target-centric over the full (symmetric) close list
 *     instead of the reference's mutual Newton-3 updates over the halved
 *     list; same pairs, different summation order.
 *   - The counting sort is stable (the reference's atomic scatter makes the
 *     order inside a leaf thread-dependent; with one thread it is this order).
 */
#include "orc_internal.h"

/* ------------------------------------------------------------------ */
/* normalisation tables: special_functions.h:56-138                     */
/* ------------------------------------------------------------------ */
double g_K[MAXN3 * (MAXN3 + 1) / 2];           /* K(n,m)=sqrt((n-m)!/(n+m)!) */
double g_A[2 * MAXN3 * (2 * MAXN3 + 1) / 2];   /* A(n,m)=(-1)^n/sqrt((n-m)!(n+m)!) */
double g_binom[2 * MAXN2][2 * MAXN2];          /* Pascal triangle */
static int g_tables_ready = 0;


void init_norm_tables(void)
{
	if (g_tables_ready) return;
	g_K[0] = 1.0;
	for (int n = 1; n < MAXN3; ++n) {
		for (int m = 0; m <= n - 1; ++m) g_K[TIX(n, m)] = g_K[TIX(n - 1, m)] * (n - m) / (n + m);
		g_K[TIX(n, n)] = g_K[TIX(n, n - 1)] / (2 * n);
	}
	for (int n = 1; n < MAXN3; ++n)
		for (int m = 0; m <= n; ++m) g_K[TIX(n, m)] = sqrt(g_K[TIX(n, m)]);
	g_A[0] = 1.0;
	for (int n = 1; n < 2 * MAXN3; ++n) {
		for (int m = 0; m <= n - 1; ++m) g_A[TIX(n, m)] = g_A[TIX(n - 1, m)] * (n - m) * (n + m);
		g_A[TIX(n, n)] = g_A[TIX(n, n - 1)] * 2 * n;
	}
	for (int n = 1; n < 2 * MAXN3; ++n)
		for (int m = 0; m <= n; ++m) g_A[TIX(n, m)] = sgn_n(n) / sqrt(g_A[TIX(n, m)]);
	memset(g_binom, 0, sizeof(g_binom));
	g_binom[0][0] = 1.0;
	for (int i = 1; i < 2 * MAXN2; ++i) {
		g_binom[i][0] = 1.0; g_binom[i][i] = 1.0;
		for (int j = 1; j < i; ++j) g_binom[i][j] = g_binom[i - 1][j] + g_binom[i - 1][j - 1];
	}
	g_tables_ready = 1;
}

/* associated Legendre P(n,m)(cos theta), n<N, Condon-Shortley phase:
 * special_functions.h:12-31 */
void compute_pnm(int N, double theta, double* P)
{
	double x = cos(theta), y = sin(theta);
	P[0] = 1.0;
	for (int n = 1; n < N; ++n) {
		for (int m = 0; m <= n - 2; ++m)
			P[TIX(n, m)] = ((2 * n - 1) * x * P[TIX(n - 1, m)] - (n + m - 1) * P[TIX(n - 2, m)]) / (n - m);
		P[TIX(n, n - 1)] = P[TIX(n - 1, n - 1)] * x * (2 * n - 1);
		P[TIX(n, n)] = P[TIX(n - 1, n - 1)] * y * (1 - 2 * n);
	}
}

/* Cartesian -> (r + 1e-12, theta, phi): simple_math.h:101-117 */
void dec_to_sph(double x, double y, double z, double* r, double* th, double* ph)
{
	const double e = 1e-12;
	double rr = sqrt(x * x + y * y + z * z) + e;
	*r = rr;
	*th = acos(z / rr);
	if (fabs(x) + fabs(y) < e) *ph = 0.0;
	else if (fabs(x) < e) *ph = y / fabs(y) * PI_D * 0.5;
	else *ph = atan2(y, x);
}

/* ------------------------------------------------------------------ */
/* Wigner small-d matrices, special_functions.cpp:194-351              */
/* layout: idx(n,m,k) = n(n+1)(4n-1)/6 + m(2n+1) + (k+n), m>=0, |k|<=n */
/* ------------------------------------------------------------------ */

int orc_wignerd(int N, double theta, double* D)
{
	if (N < 1 || N > 100) return -1;
	memset(D, 0, sizeof(double) * DSIZE(N));
	int isneg = theta < 0;
	theta = fabs(theta);
	int closetopi = 0;
	if (theta > PI_D / 2) { theta = PI_D - theta; closetopi = 1; }
	if (fabs(theta) < 1e-3) {
		for (int n = 0; n < N; ++n)
			for (int m = 0; m <= n; ++m) D[DIX(n, m, m)] = 1.0;
	} else {
		double* g = (double*)malloc(sizeof(double) * N * (N + 1) / 2);
		g[0] = 1.0;
		for (int n = 1; n < N; ++n) {
			g[TIX(n, 0)] = sqrt((2 * n - 1.) / (2 * n)) * g[TIX(n - 1, 0)];
			for (int m = 1; m <= n; ++m) g[TIX(n, m)] = sqrt((n - m + 1.) / (n + m)) * g[TIX(n, m - 1)];
		}
		double s = sin(theta), c = 1.0 + cos(theta), f = s / c;
		double* sp = (double*)malloc(sizeof(double) * (N + 1));
		double* cp = (double*)malloc(sizeof(double) * (N + 1));
		sp[0] = cp[0] = 1.0;
		for (int i = 1; i <= N; ++i) { sp[i] = sp[i - 1] * s; cp[i] = cp[i - 1] * c; }
		/* stage 1: the k = n column */
		for (int n = 0; n < N; ++n)
			for (int m = 0; m <= n; ++m)
				D[DIX(n, m, n)] = sgn_n(n + m) * g[TIX(n, m)] * cp[m] * sp[n - m];
		/* stage 2: the m = n row, k descending */
		for (int n = 0; n < N; ++n)
			for (int k = n; k > -n; --k)
				D[DIX(n, n, k - 1)] = (n + k) / sqrt(n * (n + 1.) - k * (k - 1.)) * f * D[DIX(n, n, k)];
		/* stage 3: rows m < n from row m+1, k descending */
		for (int n = 0; n < N; ++n)
			for (int m = n - 1; m >= 0; --m)
				for (int k = n; k > -n; --k)
					D[DIX(n, m, k - 1)] =
						sqrt((n * (n + 1.) - m * (m + 1.)) / (n * (n + 1.) - k * (k - 1.))) * D[DIX(n, m + 1, k)] +
						(m + k) / sqrt(n * (n + 1.) - k * (k - 1.)) * f * D[DIX(n, m, k)];
		free(g); free(sp); free(cp);
	}
	if (closetopi) { /* d(pi - t)[n,m,k] = (-1)^(n+m) d(t)[n,m,-k] */
		double* cpy = (double*)malloc(sizeof(double) * DSIZE(N));
		memcpy(cpy, D, sizeof(double) * DSIZE(N));
		for (int n = 1; n < N; ++n)
			for (int m = 0; m <= n; ++m)
				for (int k = -n; k <= n; ++k) D[DIX(n, m, k)] = sgn_n(n + m) * cpy[DIX(n, m, -k)];
		free(cpy);
	}
	for (int n = 1; n < N; ++n)
		for (int m = 0; m <= n; ++m)
			for (int k = -n; k <= n; ++k) {
				if (k < 0) D[DIX(n, m, k)] *= sgn_n(k);     /* eps(k) sign convention */
				if (isneg) D[DIX(n, m, k)] *= sgn_n(m - k); /* d(-t) = (-1)^(m-k) d(t) */
			}
	return DSIZE(N);
}

/* Angle tables keyed by int(100*angle), filled in the same order as
 * special_functions.cpp:363-381 (last writer wins), over the 316 far
 * offsets of the 7x7x7 block minus its 3x3x3 core. */
#define KEYOFF 400
#define NKEY 801
static double g_theta_of_key[NKEY], g_phi_of_key[NKEY];
static int g_theta_has[NKEY], g_phi_has[NKEY];
static double* g_dtab[NKEY];      /* Wigner-d (N = 18) per theta key */
static double* g_etab[NKEY];      /* (cos(m phi), sin(m phi)), m < 18, per phi key */
static int g_dir_ready = 0;

void init_direction_tables(void)
{
	if (g_dir_ready) return;
	init_norm_tables();
	memset(g_theta_has, 0, sizeof(g_theta_has));
	memset(g_phi_has, 0, sizeof(g_phi_has));
	for (int i = -3; i < 4; ++i)
		for (int j = -3; j < 4; ++j)
			for (int k = -3; k < 4; ++k) {
				if (abs(i) <= 1 && abs(j) <= 1 && abs(k) <= 1) continue;
				double r, th, ph;
				dec_to_sph((double)i, (double)j, (double)k, &r, &th, &ph);
				int key = (int)(th * 100);
				g_theta_of_key[KEYOFF + key] = th; g_theta_has[KEYOFF + key] = 1;
				g_theta_of_key[KEYOFF - key] = -th; g_theta_has[KEYOFF - key] = 1;
				key = (int)(ph * 100);
				g_phi_of_key[KEYOFF + key] = ph; g_phi_has[KEYOFF + key] = 1;
				g_phi_of_key[KEYOFF - key] = -ph; g_phi_has[KEYOFF - key] = 1;
			}
	for (int t = 0; t < NKEY; ++t) {
		g_dtab[t] = NULL; g_etab[t] = NULL;
		if (g_theta_has[t]) {
			g_dtab[t] = (double*)malloc(sizeof(double) * DSIZE(MAXN3));
			orc_wignerd(MAXN3, g_theta_of_key[t], g_dtab[t]);
		}
		if (g_phi_has[t]) {
			g_etab[t] = (double*)malloc(sizeof(double) * 2 * MAXN3);
			for (int m = 0; m < MAXN3; ++m) {
				g_etab[t][2 * m] = cos(m * g_phi_of_key[t]);
				g_etab[t][2 * m + 1] = sin(m * g_phi_of_key[t]);
			}
		}
	}
	g_dir_ready = 1;
}

const double* dtab_for(double theta)
{
	int key = (int)(theta * 100);
	if (key < -KEYOFF || key > KEYOFF) return NULL;
	return g_dtab[KEYOFF + key];
}
const double* etab_for(double phi)
{
	int key = (int)(phi * 100);
	if (key < -KEYOFF || key > KEYOFF) return NULL;
	return g_etab[KEYOFF + key];
}

/* number of distinct keys (for tests): theta keys with theta >= 0, phi keys */
void orc_direction_key_counts(int* n_theta_pos, int* n_theta_all, int* n_phi_all)
{
	init_direction_tables();
	int a = 0, b = 0, c = 0;
	for (int t = 0; t < NKEY; ++t) {
		if (g_theta_has[t]) { b++; if (t >= KEYOFF) a++; }
		if (g_phi_has[t]) c++;
	}
	*n_theta_pos = a; *n_theta_all = b; *n_phi_all = c;
}

/* the table angle the reference would use for a runtime angle (tests) */
int orc_table_angles(double theta, double phi, double* theta_tab, double* phi_tab)
{
	init_direction_tables();
	int kt = (int)(theta * 100), kp = (int)(phi * 100);
	if (kt < -KEYOFF || kt > KEYOFF || !g_theta_has[KEYOFF + kt]) return -1;
	if (kp < -KEYOFF || kp > KEYOFF || !g_phi_has[KEYOFF + kp]) return -2;
	*theta_tab = g_theta_of_key[KEYOFF + kt];
	*phi_tab = g_phi_of_key[KEYOFF + kp];
	return 0;
}
