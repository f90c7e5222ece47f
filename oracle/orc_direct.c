/* orc_direct.c -- TEST INFRASTRUCTURE: FP64 direct sums with the reference's
 * clamp of r at 1e-4 and its self term (common/simple_math.h:130-216,
 * 218-281).  Used for the accuracy figures (rel-L2 against direct) and by the
 * tests; a target that coincides with a source picks up q / 1e-4. */
#include "orc_internal.h"

void orc_direct3d(size_t ns, const double* sxyz, const double* sq, size_t nt, const double* txyz,
                  double* pot, double* field)
{
#pragma omp parallel for schedule(static)
	for (long long i = 0; i < (long long)nt; ++i) {
		double xi = txyz[3 * i], yi = txyz[3 * i + 1], zi = txyz[3 * i + 2];
		double p = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
		for (size_t j = 0; j < ns; ++j) {
			double dx = xi - sxyz[3 * j], dy = yi - sxyz[3 * j + 1], dz = zi - sxyz[3 * j + 2];
			double r = sqrt(dx * dx + dy * dy + dz * dz);
			if (r < ORC_EPS) r = ORC_EPS;
			double qr = sq[j] / r, qr3 = qr / (r * r);
			p += qr; fx += dx * qr3; fy += dy * qr3; fz += dz * qr3;
		}
		pot[i] = p; field[3 * i] = fx; field[3 * i + 1] = fy; field[3 * i + 2] = fz;
	}
}

void orc_direct2d(size_t ns, const double* sxy, const double* sq, size_t nt, const double* txy,
                  double* pot, double* field)
{
#pragma omp parallel for schedule(static)
	for (long long i = 0; i < (long long)nt; ++i) {
		double xi = txy[2 * i], yi = txy[2 * i + 1];
		double p = 0.0, fr = 0.0, fi = 0.0;
		for (size_t j = 0; j < ns; ++j) {
			double dx = xi - sxy[2 * j], dy = yi - sxy[2 * j + 1];
			double r2 = dx * dx + dy * dy;
			if (r2 < ORC_EPS2) r2 = ORC_EPS2;
			p += sq[j] * 0.5 * log(r2);
			fr += sq[j] * dx / r2; fi -= sq[j] * dy / r2;
		}
		pot[i] = p; field[2 * i] = fr; field[2 * i + 1] = fi;
	}
}

void orc_set_threads(int n);
