/* orc_tree.h -- TEST INFRASTRUCTURE: the uniform-depth Morton tree of the C
 * restatement (cpu/morton_tree.{h,cpp} of the reference). */
#pragma once
#include "orc_internal.h"

typedef struct {
	int dim, depth;
	size_t n;                 /* particles in the tree (targets first, then sources) */
	double shift[3], scale;
	/* particles in sorted (tree) order */
	double *x, *y, *z, *q;
	unsigned long long* pcode;
	long long* positions;     /* positions[i] = tree position of input particle i */
	size_t targets_num;       /* particles with q == 0 */
	/* per level */
	size_t* lsize;
	unsigned long long** code;
	long long **sb, **se, **tb, **te, **parent;
	double **cx, **cy, **cz;
	/* lists per level, CSR; close lists are the full symmetric lists */
	long long **close_off, **close_idx, **far_off, **far_idx;
	/* expansions per level: complex interleaved, ncoef per cell */
	int N, ncoef;
	double **outer, **inner;
	/* outputs in tree order */
	double *pot, *fld;
} orc_tree;

orc_tree* orc_tree_build(int dim, size_t n, const double* pts, const double* q, int depth);
void orc_tree_free(orc_tree* t);
