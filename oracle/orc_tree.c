/* orc_tree.c -- TEST INFRASTRUCTURE: uniform-depth Morton tree of the C
 * restatement, following cpu/morton_tree.cpp:286-493 of the reference:
 * bounding box (218-301), Morton codes (48-99), a stable sort by code (the
 * reference's counting sort with one thread, 329-357), unique cells per level
 * with ranges, parents and centres (101-145, 371-423), the q == 0 target
 * partition (427-467) and the close/far lists (147-208). */
#include "orc_tree.h"
#include <stdio.h>

static unsigned long long spread_bits(unsigned long long v, int dim)
{
	unsigned long long out = 0;
	for (int b = 0; b < 21 && (v >> b); ++b) out |= ((v >> b) & 1ull) << (dim * b);
	return out;
}

static void center_from_code(unsigned long long v, int level, int dim, const double* shift, double scale,
                             double* cx, double* cy, double* cz)
{
	double step = 1.0 / (double)(1ull << (level + 1));
	double x = step, y = step, z = step;
	step *= 2;
	for (int i = 0; i < level; ++i) {
		if (dim == 3) { z += step * (double)(v & 1); v >>= 1; }
		y += step * (double)(v & 1); v >>= 1;
		x += step * (double)(v & 1); v >>= 1;
		step *= 2;
	}
	x *= scale; x += shift[0];
	y *= scale; y += shift[1];
	*cx = x; *cy = y;
	if (dim == 3) { z *= scale; z += shift[2]; *cz = z; }
	else *cz = 0.0;
}

/* stable LSD radix sort of indices by 64-bit key */
static void stable_sort_by_key(const unsigned long long* key, size_t n, long long* idx, int key_bits)
{
	long long* tmp = (long long*)malloc(sizeof(long long) * (n ? n : 1));
	for (size_t i = 0; i < n; ++i) idx[i] = (long long)i;
	for (int sh = 0; sh < key_bits; sh += 8) {
		size_t cnt[257];
		memset(cnt, 0, sizeof(cnt));
		for (size_t i = 0; i < n; ++i) cnt[1 + ((key[idx[i]] >> sh) & 255u)]++;
		for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
		for (size_t i = 0; i < n; ++i) tmp[cnt[(key[idx[i]] >> sh) & 255u]++] = idx[i];
		memcpy(idx, tmp, sizeof(long long) * n);
	}
	free(tmp);
}

static void* xmalloc(size_t bytes) { void* p = malloc(bytes ? bytes : 8); if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); } return p; }

orc_tree* orc_tree_build(int dim, size_t n, const double* pts, const double* q, int depth)
{
	if ((dim != 2 && dim != 3) || n == 0 || depth < 1 || dim * (depth - 1) > 60) return NULL;
	orc_tree* t = (orc_tree*)calloc(1, sizeof(orc_tree));
	t->dim = dim; t->depth = depth; t->n = n;
	double* x = (double*)xmalloc(sizeof(double) * n);
	double* y = (double*)xmalloc(sizeof(double) * n);
	double* z = (double*)xmalloc(sizeof(double) * n);
	double* qq = (double*)xmalloc(sizeof(double) * n);
	for (size_t i = 0; i < n; ++i) {
		x[i] = pts[dim * i]; y[i] = pts[dim * i + 1]; z[i] = dim == 3 ? pts[dim * i + 2] : 0.0;
		qq[i] = q[i];
	}
	/* bounding box: shift = min - 1e-7, scale = largest extent + 1e-6 */
	double mn[3] = { x[0], y[0], z[0] }, mx[3] = { x[0], y[0], z[0] };
	for (size_t i = 0; i < n; ++i) {
		double v[3] = { x[i], y[i], z[i] };
		for (int d = 0; d < dim; ++d) { if (v[d] < mn[d]) mn[d] = v[d]; if (v[d] > mx[d]) mx[d] = v[d]; }
	}
	double dw = mx[0] - mn[0];
	for (int d = 1; d < dim; ++d) if (mx[d] - mn[d] > dw) dw = mx[d] - mn[d];
	for (int d = 0; d < 3; ++d) t->shift[d] = d < dim ? mn[d] - 1.e-7 : 0.0;
	t->scale = dw + 1.e-6;
	/* Morton codes at the leaf level (depth - 1) */
	unsigned long long* code = (unsigned long long*)xmalloc(sizeof(unsigned long long) * n);
	double bit_shift = (double)(1ull << (depth - 1));
	for (size_t i = 0; i < n; ++i) {
		double v[3] = { x[i], y[i], z[i] };
		unsigned long long c = 0;
		for (int d = 0; d < dim; ++d) {
			double u = (v[d] - t->shift[d]) / t->scale;
			unsigned long long iv = (unsigned long long)(bit_shift * u);
			c |= spread_bits(iv, dim) << (dim - 1 - d);
		}
		code[i] = c;
	}
	/* stable sort; positions[i] = sorted position of input i */
	long long* order = (long long*)xmalloc(sizeof(long long) * n);
	stable_sort_by_key(code, n, order, dim * (depth - 1));
	t->x = (double*)xmalloc(sizeof(double) * n); t->y = (double*)xmalloc(sizeof(double) * n);
	t->z = (double*)xmalloc(sizeof(double) * n); t->q = (double*)xmalloc(sizeof(double) * n);
	t->pcode = (unsigned long long*)xmalloc(sizeof(unsigned long long) * n);
	t->positions = (long long*)xmalloc(sizeof(long long) * n);
	long long* inv = (long long*)xmalloc(sizeof(long long) * n); /* tree position -> input index */
	for (size_t s = 0; s < n; ++s) {
		long long i = order[s];
		t->x[s] = x[i]; t->y[s] = y[i]; t->z[s] = z[i]; t->q[s] = qq[i]; t->pcode[s] = code[i];
		inv[s] = i;
	}
	free(x); free(y); free(z); free(qq); free(code); free(order);

	/* levels */
	int D = depth;
	t->lsize = (size_t*)calloc(D, sizeof(size_t));
	t->code = (unsigned long long**)calloc(D, sizeof(void*));
	t->sb = (long long**)calloc(D, sizeof(void*)); t->se = (long long**)calloc(D, sizeof(void*));
	t->tb = (long long**)calloc(D, sizeof(void*)); t->te = (long long**)calloc(D, sizeof(void*));
	t->parent = (long long**)calloc(D, sizeof(void*));
	t->cx = (double**)calloc(D, sizeof(void*)); t->cy = (double**)calloc(D, sizeof(void*));
	t->cz = (double**)calloc(D, sizeof(void*));
	{
		size_t m = 0;
		for (size_t s = 0; s < n; ++s) if (s == 0 || t->pcode[s] != t->pcode[s - 1]) m++;
		int L = D - 1;
		t->lsize[L] = m;
		t->code[L] = (unsigned long long*)xmalloc(sizeof(unsigned long long) * m);
		t->sb[L] = (long long*)xmalloc(sizeof(long long) * m); t->se[L] = (long long*)xmalloc(sizeof(long long) * m);
		size_t c = 0;
		for (size_t s = 0; s < n; ++s) {
			if (s == 0 || t->pcode[s] != t->pcode[s - 1]) {
				if (c > 0) t->se[L][c - 1] = (long long)s;
				t->code[L][c] = t->pcode[s]; t->sb[L][c] = (long long)s; c++;
			}
		}
		t->se[L][m - 1] = (long long)n;
	}
	for (int L = D - 2; L >= 0; --L) {
		size_t mb = t->lsize[L + 1], m = 0;
		unsigned long long* cb = t->code[L + 1];
		for (size_t s = 0; s < mb; ++s) if (s == 0 || (cb[s] >> dim) != (cb[s - 1] >> dim)) m++;
		t->lsize[L] = m;
		t->code[L] = (unsigned long long*)xmalloc(sizeof(unsigned long long) * m);
		t->sb[L] = (long long*)xmalloc(sizeof(long long) * m); t->se[L] = (long long*)xmalloc(sizeof(long long) * m);
		t->parent[L + 1] = (long long*)xmalloc(sizeof(long long) * mb);
		long long c = -1;
		for (size_t s = 0; s < mb; ++s) {
			if (s == 0 || (cb[s] >> dim) != (cb[s - 1] >> dim)) {
				if (c >= 0) t->se[L][c] = (long long)s;
				c++;
				t->code[L][c] = cb[s] >> dim; t->sb[L][c] = (long long)s;
			}
			t->parent[L + 1][s] = c;
		}
		t->se[L][m - 1] = (long long)mb;
	}
	t->parent[0] = (long long*)xmalloc(sizeof(long long));
	t->parent[0][0] = -1;
	for (int L = 0; L < D; ++L) {
		size_t m = t->lsize[L];
		t->cx[L] = (double*)xmalloc(sizeof(double) * m); t->cy[L] = (double*)xmalloc(sizeof(double) * m);
		t->cz[L] = (double*)xmalloc(sizeof(double) * m);
		t->tb[L] = (long long*)xmalloc(sizeof(long long) * m); t->te[L] = (long long*)xmalloc(sizeof(long long) * m);
		for (size_t c = 0; c < m; ++c) {
			center_from_code(t->code[L][c], L, dim, t->shift, t->scale, &t->cx[L][c], &t->cy[L][c], &t->cz[L][c]);
			t->tb[L][c] = t->sb[L][c]; t->te[L][c] = t->se[L][c];
		}
	}
	/* target partition: inside each leaf, q != 0 particles move to the front
	 * by swaps; the q == 0 ones form target_range (cpu/morton_tree.cpp:427-467) */
	{
		int L = D - 1;
		size_t targets = 0;
		for (size_t c = 0; c < t->lsize[L]; ++c) {
			long long s0 = t->sb[L][c], s1 = t->se[L][c], tb = s0;
			for (long long i = s0; i < s1; ++i) {
				if (t->q[i] != 0.0) {
					double tx = t->x[tb], ty = t->y[tb], tz = t->z[tb], tq = t->q[tb];
					t->x[tb] = t->x[i]; t->y[tb] = t->y[i]; t->z[tb] = t->z[i]; t->q[tb] = t->q[i];
					t->x[i] = tx; t->y[i] = ty; t->z[i] = tz; t->q[i] = tq;
					long long ti = inv[tb]; inv[tb] = inv[i]; inv[i] = ti;
					tb++;
				}
			}
			t->tb[L][c] = tb; t->te[L][c] = s1; t->se[L][c] = tb;
			targets += (size_t)(s1 - tb);
		}
		t->targets_num = targets;
	}
	for (size_t s = 0; s < n; ++s) t->positions[inv[s]] = (long long)s;
	free(inv);

	/* close / far lists */
	t->close_off = (long long**)calloc(D, sizeof(void*)); t->close_idx = (long long**)calloc(D, sizeof(void*));
	t->far_off = (long long**)calloc(D, sizeof(void*)); t->far_idx = (long long**)calloc(D, sizeof(void*));
	for (int L = 0; L < D; ++L) {
		size_t m = t->lsize[L];
		t->close_off[L] = (long long*)calloc(m + 1, sizeof(long long));
		t->far_off[L] = (long long*)calloc(m + 1, sizeof(long long));
		if (L == 0) { t->close_idx[L] = (long long*)xmalloc(8); t->far_idx[L] = (long long*)xmalloc(8); continue; }
		if (L == 1) {
			t->close_idx[L] = (long long*)xmalloc(sizeof(long long) * m * m);
			long long a = 0;
			for (size_t c = 0; c < m; ++c) {
				for (size_t k = 0; k < m; ++k) if (k != c) t->close_idx[L][a++] = (long long)k;
				t->close_off[L][c + 1] = a;
			}
			t->far_idx[L] = (long long*)xmalloc(8);
			continue;
		}
		double h = sqrt(dim + 1.e-5) * t->scale / (double)(1ull << L);
		double dw2 = h * h;
		long long *pco = t->close_off[L - 1], *pci = t->close_idx[L - 1];
		long long *psb = t->sb[L - 1], *pse = t->se[L - 1];
		for (int pass = 0; pass < 2; ++pass) {
			long long a = 0, b = 0;
			for (size_t c = 0; c < m; ++c) {
				long long p = t->parent[L][c];
				double cx = t->cx[L][c], cy = t->cy[L][c], cz = t->cz[L][c];
				for (long long e = pco[p]; e <= pco[p + 1]; ++e) {
					long long pn = e < pco[p + 1] ? pci[e] : p; /* close list of parent, then parent itself */
					for (long long k = psb[pn]; k < pse[pn]; ++k) {
						if (pn == p && k == (long long)c) continue;
						double dx = t->cx[L][k] - cx, dy = t->cy[L][k] - cy, dz = t->cz[L][k] - cz;
						double d2 = dx * dx + dy * dy + (dim == 3 ? dz * dz : 0.0);
						if (d2 < dw2) { if (pass) t->close_idx[L][a] = k; a++; }
						else { if (pass) t->far_idx[L][b] = k; b++; }
					}
				}
				if (!pass) { t->close_off[L][c + 1] = a; t->far_off[L][c + 1] = b; }
			}
			if (!pass) {
				t->close_idx[L] = (long long*)xmalloc(sizeof(long long) * a);
				t->far_idx[L] = (long long*)xmalloc(sizeof(long long) * b);
			}
		}
	}
	return t;
}

void orc_tree_free(orc_tree* t)
{
	if (!t) return;
	for (int L = 0; L < t->depth; ++L) {
		free(t->code[L]); free(t->sb[L]); free(t->se[L]); free(t->tb[L]); free(t->te[L]); free(t->parent[L]);
		free(t->cx[L]); free(t->cy[L]); free(t->cz[L]);
		free(t->close_off[L]); free(t->close_idx[L]); free(t->far_off[L]); free(t->far_idx[L]);
		if (t->outer) free(t->outer[L]);
		if (t->inner) free(t->inner[L]);
	}
	free(t->code); free(t->sb); free(t->se); free(t->tb); free(t->te); free(t->parent);
	free(t->cx); free(t->cy); free(t->cz); free(t->close_off); free(t->close_idx); free(t->far_off); free(t->far_idx);
	free(t->outer); free(t->inner); free(t->lsize);
	free(t->x); free(t->y); free(t->z); free(t->q); free(t->pcode); free(t->positions);
	free(t->pot); free(t->fld);
	free(t);
}

/* ---- exported tree queries (tests compare these with the reference) ---- */
void* orc_tree_create(int dim, size_t n, const double* pts, const double* q, int depth)
{ return orc_tree_build(dim, n, pts, q, depth); }
void orc_tree_destroy(void* h) { orc_tree_free((orc_tree*)h); }
size_t orc_tree_level_size(void* h, int L) { return ((orc_tree*)h)->lsize[L]; }
size_t orc_tree_targets_num(void* h) { return ((orc_tree*)h)->targets_num; }
void orc_tree_geometry(void* h, double* shift, double* scale)
{ orc_tree* t = (orc_tree*)h; for (int d = 0; d < 3; ++d) shift[d] = t->shift[d]; *scale = t->scale; }
void orc_tree_cells(void* h, int L, unsigned long long* code, long long* sb, long long* se, long long* tb,
                    long long* te, long long* parent, double* center)
{
	orc_tree* t = (orc_tree*)h;
	for (size_t c = 0; c < t->lsize[L]; ++c) {
		code[c] = t->code[L][c]; sb[c] = t->sb[L][c]; se[c] = t->se[L][c]; tb[c] = t->tb[L][c]; te[c] = t->te[L][c];
		parent[c] = L > 0 ? t->parent[L][c] : -1;
		center[t->dim * c] = t->cx[L][c]; center[t->dim * c + 1] = t->cy[L][c];
		if (t->dim == 3) center[3 * c + 2] = t->cz[L][c];
	}
}
/* halved = 1 gives the leaf close lists as the reference leaves them in
 * source-only mode (each pair kept by its lower index) */
void orc_tree_list_counts(void* h, int L, int halved, long long* nclose, long long* nfar)
{
	orc_tree* t = (orc_tree*)h;
	for (size_t c = 0; c < t->lsize[L]; ++c) {
		long long k = 0;
		for (long long e = t->close_off[L][c]; e < t->close_off[L][c + 1]; ++e)
			if (!halved || t->close_idx[L][e] > (long long)c) k++;
		nclose[c] = k;
		nfar[c] = t->far_off[L][c + 1] - t->far_off[L][c];
	}
}
void orc_tree_lists(void* h, int L, int halved, long long* close, long long* far)
{
	orc_tree* t = (orc_tree*)h;
	long long a = 0, b = 0;
	for (size_t c = 0; c < t->lsize[L]; ++c) {
		for (long long e = t->close_off[L][c]; e < t->close_off[L][c + 1]; ++e)
			if (!halved || t->close_idx[L][e] > (long long)c) close[a++] = t->close_idx[L][e];
		for (long long e = t->far_off[L][c]; e < t->far_off[L][c + 1]; ++e) far[b++] = t->far_idx[L][e];
	}
}
void orc_tree_positions(void* h, long long* pos)
{ orc_tree* t = (orc_tree*)h; memcpy(pos, t->positions, sizeof(long long) * t->n); }
void orc_tree_particles(void* h, double* pts, double* q)
{
	orc_tree* t = (orc_tree*)h;
	for (size_t s = 0; s < t->n; ++s) {
		pts[t->dim * s] = t->x[s]; pts[t->dim * s + 1] = t->y[s];
		if (t->dim == 3) pts[3 * s + 2] = t->z[s];
		q[s] = t->q[s];
	}
}
