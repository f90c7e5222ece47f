// C++ drop-in for the reference's solver classes, over the C ABI in lfmm.h.
//
// Replaces, with the same names, constructor signatures and public members:
//   fmm::gpu::FastMultipole3d<double>  (reference src/cuda/multipole3d.h:16-17)
//   fmm::gpu::FastMultipole            (reference src/cuda/multipole.h:11-12)
//   fmm::particle / Vector3d / particle3d / particle2d / FMM_AUTO
//                                      (reference src/common/utils.h:26-58, 149-151; defs.h:22)
//   InitMathConstants / cudaCopyMathConstants / cudaClearMathConstants
//                                      (reference src/common/special_functions.h:154-156)
// Results land in `potentials` and `forces`, sized to the targets and in input
// order, as in the reference.  Differences: errors throw fmm::gpu::Error (the
// reference ignores them); the math tables are built per context, so the
// three table functions are no-ops kept for source compatibility; the extra
// constructor arguments (max_leaf, precision) default to the reference's
// behaviour (uniform tree, FP64).  Link with -llfmm (laplace_fmm_b200/liblfmm.so).
#pragma once
#include "lfmm.h"

#include <array>
#include <complex>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace fmm {

const int FMM_AUTO = std::numeric_limits<int>::max();

template <typename T>
struct Vector3 : public std::array<T, 3> {
	constexpr Vector3() : std::array<T, 3>{T(), T(), T()} {}
	constexpr Vector3(T x, T y, T z) : std::array<T, 3>{x, y, z} {}
};
using Vector3d = Vector3<double>;
using point3d = Vector3d;
using point2d = std::complex<double>;

template <typename point, typename value>
struct particle {
	point center;
	value q;
	size_t morton_code;
};
using particle3d = particle<point3d, double>;
using particle2d = particle<point2d, double>;

enum class InteractionType { Potential2d, Force2d, Potential3d, Force3d };

namespace detail {
inline void InitMathConstants(int = 18) {}
} // namespace detail

namespace gpu {

inline void cudaCopyMathConstants() {}
inline void cudaClearMathConstants() {}

struct Error : std::runtime_error {
	int status;
	Error(int st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

namespace detail {

// One context per thread and device 0 (the reference solvers are blocking on
// the default device too).
struct Ctx {
	lfmm_ctx* h = nullptr;
	Ctx()
	{
		lfmm_options o{0, 0, 0};
		int st = lfmm_create(&h, &o);
		if (st != LFMM_OK) throw Error(st, "lfmm_create failed: no usable CUDA device");
	}
	~Ctx() { lfmm_destroy(h); }
	void check(int st, const char* what) const
	{
		if (st != LFMM_OK) throw Error(st, std::string(what) + ": " + lfmm_last_error(h));
	}
};

inline Ctx& ctx()
{
	thread_local Ctx c;
	return c;
}

template <int DIM, typename P>
inline void split(const std::vector<P>& ps, std::vector<double>& xyz, std::vector<double>* q)
{
	xyz.resize(ps.size() * DIM);
	if (q) q->resize(ps.size());
	for (size_t i = 0; i < ps.size(); ++i) {
		if constexpr (DIM == 3) {
			xyz[3 * i] = ps[i].center[0]; xyz[3 * i + 1] = ps[i].center[1]; xyz[3 * i + 2] = ps[i].center[2];
		} else {
			xyz[2 * i] = ps[i].center.real(); xyz[2 * i + 1] = ps[i].center.imag();
		}
		if (q) (*q)[i] = ps[i].q;
	}
}

} // namespace detail

template <typename value>
class FastMultipole3d;

// Scalar charges.
template <>
class FastMultipole3d<double> {
public:
	using particle_t = particle<point3d, double>;

	FastMultipole3d(const std::vector<particle_t>& particles, double eps = 1.e-8, int N = FMM_AUTO,
	                int tree_depth = FMM_AUTO, int max_leaf = 0, int precision = LFMM_PRECISION_FP64)
	{
		solve(particles, nullptr, eps, N, tree_depth, max_leaf, precision);
	}
	FastMultipole3d(const std::vector<particle_t>& source_particles, const std::vector<particle_t>& target_particles,
	                double eps = 1.e-8, int N = FMM_AUTO, int tree_depth = FMM_AUTO, int max_leaf = 0,
	                int precision = LFMM_PRECISION_FP64)
	{
		solve(source_particles, &target_particles, eps, N, tree_depth, max_leaf, precision);
	}

	std::vector<Vector3d> forces;
	std::vector<double> potentials;
	lfmm_stats stats{};

private:
	void solve(const std::vector<particle_t>& src, const std::vector<particle_t>* tgt, double eps, int N, int depth,
	           int max_leaf, int precision)
	{
		std::vector<double> sx, sq, tx;
		detail::split<3>(src, sx, &sq);
		if (tgt) detail::split<3>(*tgt, tx, nullptr);
		const size_t nout = tgt ? tgt->size() : src.size();
		std::vector<double> field(3 * nout);
		potentials.assign(nout, 0.0);
		lfmm_solve_opts o{N, depth, max_leaf, precision, eps};
		auto& c = detail::ctx();
		c.check(lfmm3d_solve_ex(c.h, src.size(), sx.data(), sq.data(), tgt ? tgt->size() : 0,
		                        tgt ? tx.data() : nullptr, &o, potentials.data(), field.data(), &stats),
		        "lfmm3d_solve_ex");
		forces.resize(nout);
		for (size_t i = 0; i < nout; ++i) forces[i] = Vector3d(field[3 * i], field[3 * i + 1], field[3 * i + 2]);
	}
};

// Vector charges (reference FastMultipole3d<Vector3d>): forces = sum q x d / r^3
// at every target; potentials stays empty, as in the reference.
template <>
class FastMultipole3d<Vector3d> {
public:
	using particle_t = particle<point3d, Vector3d>;

	FastMultipole3d(const std::vector<particle_t>& particles, double eps = 1.e-8, int N = FMM_AUTO,
	                int tree_depth = FMM_AUTO, int max_leaf = 0, int precision = LFMM_PRECISION_FP64)
	{
		solve(particles, nullptr, eps, N, tree_depth, max_leaf, precision);
	}
	FastMultipole3d(const std::vector<particle_t>& source_particles, const std::vector<particle_t>& target_particles,
	                double eps = 1.e-8, int N = FMM_AUTO, int tree_depth = FMM_AUTO, int max_leaf = 0,
	                int precision = LFMM_PRECISION_FP64)
	{
		solve(source_particles, &target_particles, eps, N, tree_depth, max_leaf, precision);
	}

	std::vector<Vector3d> forces;
	std::vector<double> potentials;
	lfmm_stats stats{};

private:
	void solve(const std::vector<particle_t>& src, const std::vector<particle_t>* tgt, double eps, int N, int depth,
	           int max_leaf, int precision)
	{
		std::vector<double> sx(3 * src.size()), sq(3 * src.size()), tx;
		for (size_t i = 0; i < src.size(); ++i)
			for (int c = 0; c < 3; ++c) { sx[3 * i + c] = src[i].center[c]; sq[3 * i + c] = src[i].q[c]; }
		if (tgt) {
			tx.resize(3 * tgt->size());
			for (size_t i = 0; i < tgt->size(); ++i)
				for (int c = 0; c < 3; ++c) tx[3 * i + c] = (*tgt)[i].center[c];
		}
		const size_t nout = tgt ? tgt->size() : src.size();
		std::vector<double> field(3 * nout);
		lfmm_solve_opts o{N, depth, max_leaf, precision, eps};
		auto& c = detail::ctx();
		c.check(lfmm3d_solve_vector(c.h, src.size(), sx.data(), sq.data(), tgt ? tgt->size() : 0,
		                            tgt ? tx.data() : nullptr, &o, field.data(), &stats),
		        "lfmm3d_solve_vector");
		forces.resize(nout);
		for (size_t i = 0; i < nout; ++i) forces[i] = Vector3d(field[3 * i], field[3 * i + 1], field[3 * i + 2]);
	}
};

class FastMultipole {
public:
	FastMultipole(const std::vector<particle2d>& particles, double eps = 1.e-8, int N = FMM_AUTO,
	              int tree_depth = FMM_AUTO)
	{
		solve(particles, nullptr, eps, N, tree_depth);
	}
	FastMultipole(const std::vector<particle2d>& source_particles, const std::vector<particle2d>& target_particles,
	              double eps = 1.e-8, int N = FMM_AUTO, int tree_depth = FMM_AUTO)
	{
		solve(source_particles, &target_particles, eps, N, tree_depth);
	}

	std::vector<std::complex<double>> forces;
	std::vector<double> potentials;
	lfmm_stats stats{};

private:
	void solve(const std::vector<particle2d>& src, const std::vector<particle2d>* tgt, double eps, int N, int depth)
	{
		std::vector<double> sx, sq, tx;
		detail::split<2>(src, sx, &sq);
		if (tgt) detail::split<2>(*tgt, tx, nullptr);
		const size_t nout = tgt ? tgt->size() : src.size();
		std::vector<double> field(2 * nout);
		potentials.assign(nout, 0.0);
		auto& c = detail::ctx();
		c.check(lfmm2d_solve(c.h, src.size(), sx.data(), sq.data(), tgt ? tgt->size() : 0, tgt ? tx.data() : nullptr,
		                     N, depth, eps, LFMM_PRECISION_FP64, potentials.data(), field.data(), &stats),
		        "lfmm2d_solve");
		forces.resize(nout);
		for (size_t i = 0; i < nout; ++i) forces[i] = {field[2 * i], field[2 * i + 1]};
	}
};

// FP64 direct sum (the reference's ComputeExact computes the same values and
// writes them to a file; here they are returned): potentials, or fields as
// Vector3d (3D) / complex (2D), at every target.
template <InteractionType it, typename P>
auto ComputeExact(const std::vector<P>& sources, const std::vector<P>& targets)
{
	constexpr int DIM = (it == InteractionType::Potential3d || it == InteractionType::Force3d) ? 3 : 2;
	std::vector<double> sx, sq, tx;
	detail::split<DIM>(sources, sx, &sq);
	detail::split<DIM>(targets, tx, nullptr);
	std::vector<double> pot(targets.size()), fld(DIM * targets.size());
	auto& c = detail::ctx();
	if constexpr (DIM == 3)
		c.check(lfmm3d_direct(c.h, sources.size(), sx.data(), sq.data(), targets.size(), tx.data(), pot.data(),
		                      fld.data()), "lfmm3d_direct");
	else
		c.check(lfmm2d_direct(c.h, sources.size(), sx.data(), sq.data(), targets.size(), tx.data(), pot.data(),
		                      fld.data()), "lfmm2d_direct");
	if constexpr (it == InteractionType::Potential3d || it == InteractionType::Potential2d) {
		return pot;
	} else if constexpr (DIM == 3) {
		std::vector<Vector3d> f(targets.size());
		for (size_t i = 0; i < f.size(); ++i) f[i] = Vector3d(fld[3 * i], fld[3 * i + 1], fld[3 * i + 2]);
		return f;
	} else {
		std::vector<std::complex<double>> f(targets.size());
		for (size_t i = 0; i < f.size(); ++i) f[i] = {fld[2 * i], fld[2 * i + 1]};
		return f;
	}
}

} // namespace gpu
} // namespace fmm
