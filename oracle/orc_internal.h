/* orc_internal.h -- TEST INFRASTRUCTURE: shared declarations of the C
 * restatement of the reference FMM (see fmm_oracle.c for the overview). */
#pragma once
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>

#define ORC_EPS 1.0e-4
#define ORC_EPS2 (ORC_EPS * ORC_EPS)
#define ORC_AUTO INT_MAX
#define MAXN3 18
#define MAXN2 30
#define PI_D 3.14159265358979323846
#define TIX(n, m) ((n) * ((n) + 1) / 2 + (m))

/* ------------------------------------------------------------------ */
/* small complex helpers (explicit re/im, no C99 complex)              */
/* ------------------------------------------------------------------ */
typedef struct { double re, im; } cplx;
static inline cplx cmk(double r, double i) { cplx c = { r, i }; return c; }
static inline cplx cadd(cplx a, cplx b) { return cmk(a.re + b.re, a.im + b.im); }
static inline cplx csub(cplx a, cplx b) { return cmk(a.re - b.re, a.im - b.im); }
static inline cplx cmul(cplx a, cplx b) { return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cplx cscale(cplx a, double s) { return cmk(a.re * s, a.im * s); }
static inline cplx cdiv(cplx a, cplx b)
{
	double d = b.re * b.re + b.im * b.im;
	return cmk((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}
/* binary exponentiation, as simple_math.h:81-94 (MyPow) */
static cplx cpow_u(cplx b, unsigned e)
{
	cplx r = cmk(1.0, 0.0);
	while (e) { if (e & 1u) r = cmul(r, b); e >>= 1; b = cmul(b, b); }
	return r;
}
static inline double sgn_n(int n) { return (n & 1) ? -1.0 : 1.0; } /* (-1)^n */


/* shared tables and special functions (fmm_oracle.c) */
void init_norm_tables(void);
void init_direction_tables(void);
extern double g_K[];
extern double g_A[];
extern double g_binom[2 * MAXN2][2 * MAXN2];
static inline double Knm(int n, int m) { return g_K[TIX(n, m)]; }
static inline double Anm(int n, int m) { return g_A[TIX(n, m)]; }
static inline double m2lcoef(int j, int k, int n) { return Anm(n, k) * Anm(j, k) * sgn_n(n + k) / Anm(j + n, 0); }
void compute_pnm(int N, double theta, double* P);
void dec_to_sph(double x, double y, double z, double* r, double* th, double* ph);
const double* dtab_for(double theta);
const double* etab_for(double phi);
#define DSIZE(N) ((N) * ((N) + 1) * (4 * (N) - 1) / 6)
#define DIX(n, m, k) ((n) * ((n) + 1) * (4 * (n) - 1) / 6 + (m) * (2 * (n) + 1) + ((k) + (n)))
