// Test infrastructure, not product code.
//
// extern "C" wrapper around the UNMODIFIED reference CPU FMM (compiled from
// the reference's own sources by oracle/Makefile into oracle/_ref/).  Only the
// tests, the fixture generator and bench.py's reference arm load it, as the
// checker and the CPU baseline.  Entry points:
//   * ref_fmm3d / ref_fmm3d_st : fmm::FastMultipole3d<double> (cpu/multipole3d.cpp:1296-1374)
//   * ref_fmm3d_vec / ref_fmm3d_vec_st : fmm::FastMultipole3d<Vector3d> (vector charges,
//                                cpu/multipole3d.cpp:414-853, instantiated at :1397)
//   * ref_fmm2d / ref_fmm2d_st : fmm::FastMultipole            (cpu/multipole.cpp:451-522)
//   * ref_tree3d_* / ref_tree2d_* : fmm::MortonTree<dim,...>    (cpu/morton_tree.cpp:286-493)
//   * ref_wignerd              : fmm::ComputeWignerD            (common/special_functions.cpp:211-351)
#include "cpu/multipole3d.h"
#include "cpu/multipole.h"
#include "cpu/morton_tree.h"
#include "common/special_functions.h"
#include <omp.h>
#include <iostream>
#include <vector>
#include <complex>
#include <cstring>
#include <mutex>

namespace {

std::once_flag g_tables_once;

void ensure_tables()
{
	std::call_once(g_tables_once, [] { fmm::detail::InitMathConstants(fmm::detail::_3d_MAX_MULTIPOLE_NUM); });
}

struct Quiet
{
	std::streambuf* old;
	bool on;
	explicit Quiet(bool quiet) : old(std::cout.rdbuf()), on(quiet) { if (on) std::cout.rdbuf(nullptr); }
	~Quiet() { if (on) { std::cout.rdbuf(old); std::cout.clear(); } }
};

int g_verbose = 0;

std::vector<fmm::particle3d> make3d(const double* xyz, const double* q, size_t n)
{
	std::vector<fmm::particle3d> p(n);
	for (size_t i = 0; i < n; ++i)
		p[i] = { fmm::Vector3d(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]), q ? q[i] : 0.0, 0 };
	return p;
}

using vparticle = fmm::FastMultipole3d<fmm::Vector3d>::particle_t;

std::vector<vparticle> make3v(const double* xyz, const double* q3, size_t n)
{
	std::vector<vparticle> p(n);
	for (size_t i = 0; i < n; ++i)
		p[i] = { fmm::Vector3d(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]),
		         q3 ? fmm::Vector3d(q3[3 * i], q3[3 * i + 1], q3[3 * i + 2]) : fmm::Vector3d(0, 0, 0), 0 };
	return p;
}

std::vector<fmm::particle2d> make2d(const double* xy, const double* q, size_t n)
{
	std::vector<fmm::particle2d> p(n);
	for (size_t i = 0; i < n; ++i)
		p[i] = { std::complex<double>(xy[2 * i], xy[2 * i + 1]), q ? q[i] : 0.0, 0 };
	return p;
}

template <typename Tree>
struct TreeHandle
{
	Tree tree;
	template <typename P>
	TreeHandle(P&& p, size_t depth) : tree(std::move(p), depth) {}
};

} // namespace

extern "C" {

void ref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int ref_get_threads(void) { return omp_get_max_threads(); }
void ref_set_verbose(int v) { g_verbose = v; }

int ref_fmm3d(size_t n, const double* xyz, const double* q, int N, int depth, double eps,
              double* pot, double* field)
{
	ensure_tables();
	Quiet quiet(!g_verbose);
	auto p = make3d(xyz, q, n);
	fmm::FastMultipole3d<double> f(p, eps, N, depth);
	for (size_t i = 0; i < n; ++i)
	{
		pot[i] = f.potentials[i];
		for (int s = 0; s < 3; ++s) field[3 * i + s] = f.forces[i][s];
	}
	return 0;
}

int ref_fmm3d_st(size_t ns, const double* sxyz, const double* sq, size_t nt, const double* txyz,
                 int N, int depth, double eps, double* pot, double* field)
{
	ensure_tables();
	Quiet quiet(!g_verbose);
	auto s = make3d(sxyz, sq, ns);
	auto t = make3d(txyz, nullptr, nt);
	fmm::FastMultipole3d<double> f(s, t, eps, N, depth);
	for (size_t i = 0; i < nt; ++i)
	{
		pot[i] = f.potentials[i];
		for (int c = 0; c < 3; ++c) field[3 * i + c] = f.forces[i][c];
	}
	return 0;
}

int ref_fmm3d_vec(size_t n, const double* xyz, const double* q3, int N, int depth, double eps, double* field)
{
	ensure_tables();
	Quiet quiet(!g_verbose);
	auto p = make3v(xyz, q3, n);
	fmm::FastMultipole3d<fmm::Vector3d> f(p, eps, N, depth);
	for (size_t i = 0; i < n; ++i)
		for (int c = 0; c < 3; ++c) field[3 * i + c] = f.forces[i][c];
	return 0;
}

int ref_fmm3d_vec_st(size_t ns, const double* sxyz, const double* sq3, size_t nt, const double* txyz, int N,
                     int depth, double eps, double* field)
{
	ensure_tables();
	Quiet quiet(!g_verbose);
	auto s = make3v(sxyz, sq3, ns);
	auto t = make3v(txyz, nullptr, nt);
	fmm::FastMultipole3d<fmm::Vector3d> f(s, t, eps, N, depth);
	for (size_t i = 0; i < nt; ++i)
		for (int c = 0; c < 3; ++c) field[3 * i + c] = f.forces[i][c];
	return 0;
}

int ref_fmm2d(size_t n, const double* xy, const double* q, int N, int depth, double eps,
              double* pot, double* field)
{
	Quiet quiet(!g_verbose);
	auto p = make2d(xy, q, n);
	fmm::FastMultipole f(p, eps, N, depth);
	for (size_t i = 0; i < n; ++i)
	{
		pot[i] = f.potentials[i];
		field[2 * i] = f.forces[i].real();
		field[2 * i + 1] = f.forces[i].imag();
	}
	return 0;
}

int ref_fmm2d_st(size_t ns, const double* sxy, const double* sq, size_t nt, const double* txy,
                 int N, int depth, double eps, double* pot, double* field)
{
	Quiet quiet(!g_verbose);
	auto s = make2d(sxy, sq, ns);
	auto t = make2d(txy, nullptr, nt);
	fmm::FastMultipole f(s, t, eps, N, depth);
	for (size_t i = 0; i < nt; ++i)
	{
		pot[i] = f.potentials[i];
		field[2 * i] = f.forces[i].real();
		field[2 * i + 1] = f.forces[i].imag();
	}
	return 0;
}

int ref_wignerd(int N, double theta, double* out)
{
	auto d = fmm::ComputeWignerD(N, theta);
	std::memcpy(out, d.data(), d.size() * sizeof(double));
	return int(d.size());
}

// ---- tree export (dim 3 and 2) ----

void* ref_tree3d_build(size_t n, const double* xyz, const double* q, int depth)
{
	Quiet quiet(!g_verbose);
	return new TreeHandle<fmm::MortonTree3d>(make3d(xyz, q, n), size_t(depth));
}

void* ref_tree2d_build(size_t n, const double* xy, const double* q, int depth)
{
	Quiet quiet(!g_verbose);
	return new TreeHandle<fmm::MortonTree2d>(make2d(xy, q, n), size_t(depth));
}

void ref_tree3d_free(void* h) { delete static_cast<TreeHandle<fmm::MortonTree3d>*>(h); }
void ref_tree2d_free(void* h) { delete static_cast<TreeHandle<fmm::MortonTree2d>*>(h); }

#define TREE_QUERIES(DIMTAG, TREE_T, CENTER_COPY)                                                       \
size_t ref_tree##DIMTAG##_level_size(void* h, int lvl)                                                  \
{ return static_cast<TreeHandle<TREE_T>*>(h)->tree.level_sizes[lvl]; }                                   \
size_t ref_tree##DIMTAG##_targets_num(void* h)                                                          \
{ return static_cast<TreeHandle<TREE_T>*>(h)->tree.targets_num; }                                        \
void ref_tree##DIMTAG##_cells(void* h, int lvl, unsigned long long* code, long long* sb, long long* se,  \
                              long long* tb, long long* te, long long* parent, double* center)          \
{                                                                                                       \
	auto& t = static_cast<TreeHandle<TREE_T>*>(h)->tree;                                                \
	size_t m = t.level_sizes[lvl];                                                                      \
	for (size_t i = 0; i < m; ++i) {                                                                    \
		const auto& c = t.levels[lvl][i];                                                               \
		code[i] = c.morton_code;                                                                        \
		sb[i] = (long long)c.source_range.first; se[i] = (long long)c.source_range.second;              \
		tb[i] = (long long)c.target_range.first; te[i] = (long long)c.target_range.second;              \
		parent[i] = lvl > 0 ? (long long)c.parent : -1;                                                 \
		CENTER_COPY                                                                                     \
	}                                                                                                   \
}                                                                                                       \
void ref_tree##DIMTAG##_list_counts(void* h, int lvl, long long* nclose, long long* nfar)               \
{                                                                                                       \
	auto& t = static_cast<TreeHandle<TREE_T>*>(h)->tree;                                                \
	for (size_t i = 0; i < t.level_sizes[lvl]; ++i) {                                                   \
		nclose[i] = (long long)t.levels[lvl][i].closeneighbours.size();                                 \
		nfar[i] = (long long)t.levels[lvl][i].farneighbours.size();                                     \
	}                                                                                                   \
}                                                                                                       \
void ref_tree##DIMTAG##_lists(void* h, int lvl, long long* close, long long* far)                       \
{                                                                                                       \
	auto& t = static_cast<TreeHandle<TREE_T>*>(h)->tree;                                                \
	size_t a = 0, b = 0;                                                                                \
	for (size_t i = 0; i < t.level_sizes[lvl]; ++i) {                                                   \
		for (auto x : t.levels[lvl][i].closeneighbours) close[a++] = (long long)x;                      \
		for (auto x : t.levels[lvl][i].farneighbours) far[b++] = (long long)x;                          \
	}                                                                                                   \
}                                                                                                       \
void ref_tree##DIMTAG##_positions(void* h, long long* positions_map)                                    \
{                                                                                                       \
	auto& t = static_cast<TreeHandle<TREE_T>*>(h)->tree;                                                \
	for (size_t i = 0; i < t.positions_map.size(); ++i) positions_map[i] = (long long)t.positions_map[i]; \
}

TREE_QUERIES(3d, fmm::MortonTree3d,
	center[3 * i] = c.center[0]; center[3 * i + 1] = c.center[1]; center[3 * i + 2] = c.center[2];)
TREE_QUERIES(2d, fmm::MortonTree2d,
	center[2 * i] = c.center.real(); center[2 * i + 1] = c.center.imag();)

} // extern "C"
