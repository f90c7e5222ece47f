// A reference-style caller compiled against the drop-in header: 3D solve in
// source-only and source/target mode, vector charges, 2D solve, and the
// direct sum; prints the results as text for the test to compare.
#include "lfmm.hpp"

#include <cstdio>
#include <random>

int main()
{
	std::mt19937_64 g(12345);
	std::uniform_real_distribution<double> u(0.0, 1.0), c(-1.0, 1.0);
	std::vector<fmm::particle3d> p3(4000);
	for (auto& p : p3) { p.center = fmm::Vector3d(u(g), u(g), u(g)); p.q = c(g); }
	std::vector<fmm::particle3d> t3(300);
	for (auto& p : t3) { p.center = fmm::Vector3d(u(g), u(g), u(g)); p.q = 0.0; }
	std::vector<fmm::particle<fmm::point3d, fmm::Vector3d>> pv(2500);
	for (auto& p : pv) { p.center = fmm::Vector3d(u(g), u(g), u(g)); p.q = fmm::Vector3d(c(g), c(g), c(g)); }
	std::vector<fmm::particle2d> p2(3000);
	for (auto& p : p2) { p.center = {u(g), u(g)}; p.q = c(g); }

	fmm::detail::InitMathConstants(18);
	fmm::gpu::cudaCopyMathConstants();
	fmm::gpu::FastMultipole3d<double> a(p3, 1e-8, 9, 4);
	fmm::gpu::FastMultipole3d<double> b(p3, t3, 1e-8, 9, 4);
	fmm::gpu::FastMultipole3d<fmm::Vector3d> v(pv, 1e-8, 8, 4);
	fmm::gpu::FastMultipole f2(p2, 1e-8, 16, 5);
	auto e3 = fmm::gpu::ComputeExact<fmm::InteractionType::Potential3d>(p3, t3);
	fmm::gpu::cudaClearMathConstants();

	for (auto& p : p3) std::printf("p3 %.17g %.17g %.17g %.17g\n", p.center[0], p.center[1], p.center[2], p.q);
	for (auto& p : t3) std::printf("t3 %.17g %.17g %.17g\n", p.center[0], p.center[1], p.center[2]);
	for (auto& p : p2) std::printf("p2 %.17g %.17g %.17g\n", p.center.real(), p.center.imag(), p.q);
	for (size_t i = 0; i < p3.size(); ++i)
		std::printf("a %.17g %.17g %.17g %.17g\n", a.potentials[i], a.forces[i][0], a.forces[i][1], a.forces[i][2]);
	for (size_t i = 0; i < t3.size(); ++i)
		std::printf("b %.17g %.17g %.17g %.17g %.17g\n", b.potentials[i], b.forces[i][0], b.forces[i][1],
		            b.forces[i][2], e3[i]);
	for (size_t i = 0; i < p2.size(); ++i)
		std::printf("c %.17g %.17g %.17g\n", f2.potentials[i], f2.forces[i].real(), f2.forces[i].imag());
	for (size_t i = 0; i < pv.size(); ++i)
		std::printf("v %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", pv[i].center[0], pv[i].center[1],
		            pv[i].center[2], pv[i].q[0], pv[i].q[1], pv[i].q[2], v.forces[i][0], v.forces[i][1], v.forces[i][2]);
	if (!v.potentials.empty()) return 1;
	return 0;
}
