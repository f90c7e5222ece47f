"""Boundary-element capacitance caller (laplace_fmm_b200.bem): the exact
triangle integral on the CPU, the FMM-driven solve on the GPU."""
import numpy as np
import pytest

from laplace_fmm_b200.bem import icosphere, triangle_integral


def polar_integral(x, tri, m=400):
    """integral of 1/|x - y| over the triangle by polar coordinates about the
    projection of x into its plane (split into the three sub-triangles):
    int int r dr dtheta / sqrt(r^2 + d^2) = int (sqrt(R(theta)^2 + d^2) - |d|) dtheta,
    midpoint rule in theta."""
    n = np.cross(tri[1] - tri[0], tri[2] - tri[0])
    n /= np.linalg.norm(n)
    d = np.dot(x - tri[0], n)
    rho = x - d * n
    total = 0.0
    for k in range(3):
        a, b = tri[k], tri[(k + 1) % 3]
        sgn = np.sign(np.dot(np.cross(a - rho, b - rho), n))
        u, v = a - rho, b - rho
        ang = np.arccos(np.clip(np.dot(u, v) / np.linalg.norm(u) / np.linalg.norm(v), -1, 1))
        th = (np.arange(m) + 0.5) / m * ang
        uh = u / np.linalg.norm(u)
        w = np.cross(n, uh) * sgn
        dirs = np.cos(th)[:, None] * uh + np.sin(th)[:, None] * w
        e = (b - a) / np.linalg.norm(b - a)
        # distance along each ray to the edge line, in the plane's 2D frame (uh, n x uh)
        ex, ey = np.cross(n, uh), uh
        P = lambda z: np.stack([z @ ey, z @ ex], axis=-1)
        Md = np.stack([P(dirs), -np.broadcast_to(P(e), (m, 2))], axis=2)
        s = np.linalg.solve(Md, np.broadcast_to(P(a - rho), (m, 2))[..., None])[:, 0, 0]
        total += sgn * (np.sqrt(s * s + d * d) - abs(d)).sum() * ang / m
    return total


def test_centroids_against_quadrature():
    """The singular self case of the collocation (the centre of the source
    triangle), for arbitrary triangles in space."""
    g = np.random.default_rng(3)
    for _ in range(5):
        tri = g.random((3, 3))
        c = tri.mean(axis=0)
        assert triangle_integral(c[None], tri[None])[0] == pytest.approx(polar_integral(c, tri, m=4000), rel=1e-6)


@pytest.mark.parametrize("height", [0.05, 0.3, -0.7, 2.0])
def test_off_plane_points_against_quadrature(height):
    tri = np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.3, 0.8, 0.0]])
    for x in (np.array([0.4, 0.3, height]), np.array([1.5, -0.4, height])):
        assert triangle_integral(x[None], tri[None])[0] == pytest.approx(polar_integral(x, tri), rel=1e-5)


def test_far_point_is_the_point_charge():
    tri = np.array([[0.0, 0.0, 0.0], [0.01, 0.0, 0.0], [0.0, 0.01, 0.0]])
    x = np.array([[3.0, 4.0, 12.0]])
    area = 0.5e-4
    c = tri.mean(axis=0)
    assert triangle_integral(x, tri[None])[0] == pytest.approx(area / np.linalg.norm(x[0] - c), rel=1e-8)


def test_icosphere_is_closed_and_outward():
    V, T = icosphere(2)
    assert len(T) == 320 and np.allclose(np.linalg.norm(V, axis=1), 1.0)
    tri = V[T]
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    assert np.all(np.einsum("ij,ij->i", n, tri.mean(axis=1)) > 0)


@pytest.mark.gpu
def test_sphere_capacitance(ctx):
    """The unit sphere at unit potential carries Q = 1 (potential q / r);
    the flat-triangle discretisation converges to it, and the FMM-driven
    solve matches the dense collocation solve with exact integrals on the
    same mesh (far pairs by the 3-point rule: 2.8e-7 apart on the CPU)."""
    from laplace_fmm_b200.bem import CapacitanceSolver
    V, T = icosphere(3)
    s = CapacitanceSolver(V, T, N=14, precision="fp64", ctx=ctx)
    q_fmm = s.solve(rtol=1e-10)
    tri = V[T]
    c = tri.mean(axis=1)
    nt = len(T)
    ii, jj = np.meshgrid(np.arange(nt), np.arange(nt), indexing="ij")
    M = triangle_integral(c[ii.ravel()], tri[jj.ravel()]).reshape(nt, nt)
    area = 0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1)
    q_dense = float(np.linalg.solve(M, np.ones(nt)) @ area)
    assert q_fmm == pytest.approx(q_dense, rel=1e-6)
    s.close()
    # 20,480 triangles in the mixed form: GMRES to the operator's own accuracy
    big = CapacitanceSolver(*icosphere(5), N=12, ctx=ctx)
    q = big.solve(rtol=1e-5)
    assert q == pytest.approx(1.0, rel=2e-3) and big.matvecs < 100
    big.close()
