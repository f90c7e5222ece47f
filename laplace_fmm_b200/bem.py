"""Capacitance of a conductor by a boundary-element collocation solved
through the FMM: the application the reference's capacitance example
(examples/capacitance.cpp:148-245) computes with a dense matrix and LAPACK.

Unknown: a constant surface charge density sigma_j on each flat triangle;
collocation at the triangle centres c_i for unit potential:

    sum_j sigma_j I_j(c_i) = 1,   I_j(x) = integral over triangle j of 1 / |x - y| dA_y,

and Q = sum_j sigma_j A_j (the capacitance in units where the potential of a
charge q at distance r is q / r).  The matrix is never formed: a matvec is
the FMM potential at the centres of point charges sigma_j A_j / 3 at each
triangle's three quadrature points (the degree-2 rule at barycentric
(2/3, 1/6, 1/6) and its permutations; the centres enter the same solve
plan as zero-charge targets, so the tree and CUDA graph are built once and
each iteration changes only the charges), with the quadrature replaced by
the exact triangle integral for the near pairs (sparse correction); GMRES
(scipy) on the host drives it.

The exact integral over a flat triangle is the edge formula of D. R. Wilton,
S. M. Rao, A. W. Glisson, D. H. Schaubert, O. M. Al-Bundak and C. M. Butler,
"Potential integrals for uniform and linear source distributions on
polygonal and polyhedral domains", IEEE Trans. Antennas Propag. 32(3), 1984.
"""
from __future__ import annotations

import numpy as np

from .fmm import Plan3d

QUAD = np.array([[2 / 3, 1 / 6, 1 / 6], [1 / 6, 2 / 3, 1 / 6], [1 / 6, 1 / 6, 2 / 3]])   # barycentric, weights 1/3


def icosphere(level: int, radius: float = 1.0):
    """Vertices (nv, 3) and counter-clockwise triangles (nt, 3) of a sphere:
    the icosahedron with each face split into four ``level`` times."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(level):
        mid = {}

        def midpoint(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in mid:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                mid[key] = len(verts) - 1
            return mid[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts) * radius, np.array(faces, dtype=np.int64)


def triangle_integral(x, tri):
    """integral over the flat triangle tri[k] (3 vertices, counter-clockwise
    about its normal) of 1 / |x[k] - y| dA_y, for paired arrays x (m, 3) and
    tri (m, 3, 3): the sum over the edges of P0 ln((R+ + l+) / (R- + l-))
    minus |d| times the difference of the edge's end angles (Wilton et al.)."""
    x = np.asarray(x, dtype=np.float64)
    tri = np.asarray(tri, dtype=np.float64)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    n /= np.linalg.norm(n, axis=1)[:, None]
    d = np.einsum("ij,ij->i", x - tri[:, 0], n)          # signed height over the plane
    rho = x - d[:, None] * n                               # projection into the plane
    ad = np.abs(d)
    total = np.zeros(len(x))
    for e in range(3):
        a, b = tri[:, e], tri[:, (e + 1) % 3]
        L = np.linalg.norm(b - a, axis=1)
        lh = (b - a) / L[:, None]                          # edge direction
        uh = np.cross(lh, n)                               # outward in-plane normal
        lm = np.einsum("ij,ij->i", a - rho, lh)
        lp = np.einsum("ij,ij->i", b - rho, lh)
        p0 = np.einsum("ij,ij->i", a - rho, uh)            # signed distance to the edge's line
        r0sq = p0 * p0 + d * d
        rm = np.sqrt(r0sq + lm * lm)
        rp = np.sqrt(r0sq + lp * lp)
        on_line = np.abs(p0) < 1e-14 * np.maximum(L, 1e-300)
        with np.errstate(divide="ignore", invalid="ignore"):
            lg = np.where(on_line, 0.0, np.log((rp + lp) / (rm + lm)))
            ang = np.arctan(p0 * lp / (r0sq + ad * rp)) - np.arctan(p0 * lm / (r0sq + ad * rm))
        total += p0 * lg - ad * np.where(on_line, 0.0, ang)
    return total


class CapacitanceSolver:
    """BEM capacitance of the surface (vertices, triangles): ``solve()``
    returns Q = sum sigma_j A_j for unit potential and keeps sigma.

    near: pairs whose centres lie within ``near`` times the mean edge length
    get the exact triangle integral instead of the quadrature; N, the FMM's
    order (the plan runs the mixed form by default)."""

    def __init__(self, vertices, triangles, N: int = 12, near: float = 3.0, precision: str = "mixed",
                 tree_depth: int = 10, max_leaf: int = 32, ctx=None):
        from scipy.sparse import csr_matrix
        from scipy.spatial import cKDTree
        V = np.asarray(vertices, dtype=np.float64)
        T = np.asarray(triangles, dtype=np.int64)
        self.tri = V[T]                                               # (nt, 3, 3)
        self.centres = self.tri.mean(axis=1)
        self.areas = 0.5 * np.linalg.norm(np.cross(self.tri[:, 1] - self.tri[:, 0], self.tri[:, 2] - self.tri[:, 0]),
                                          axis=1)
        nt = len(T)
        edge = np.linalg.norm(self.tri[:, 1] - self.tri[:, 0], axis=1).mean()
        pairs = cKDTree(self.centres).query_pairs(near * edge, output_type="ndarray")
        i = np.concatenate([pairs[:, 0], pairs[:, 1], np.arange(nt)])
        j = np.concatenate([pairs[:, 1], pairs[:, 0], np.arange(nt)])
        exact = triangle_integral(self.centres[i], self.tri[j])
        self.qpts = np.einsum("qk,tkd->tqd", QUAD, self.tri).reshape(-1, 3)    # (3 nt, 3), triangle-major
        # what the FMM adds for the pair: the three quadrature charges
        quad = (self.areas[j] / 3)[:, None] / np.linalg.norm(
            self.centres[i][:, None, :] - self.qpts.reshape(nt, 3, 3)[j], axis=2)
        self.correction = csr_matrix((exact - quad.sum(axis=1), (i, j)), shape=(nt, nt))
        # sources: the quadrature points; targets: the centres (zero charge)
        pts = np.concatenate([self.qpts, self.centres])
        q0 = np.concatenate([np.repeat(self.areas / 3, 3), np.zeros(nt)])
        self.plan = Plan3d(pts, q0, N=N, tree_depth=tree_depth, max_leaf=max_leaf, precision=precision, ctx=ctx)
        self.matvecs = 0
        self.sigma = None

    def apply(self, sigma):
        """The collocation operator: sum_j sigma_j I_j(c_i) for every i."""
        sigma = np.asarray(sigma, dtype=np.float64)
        nt = len(sigma)
        q = np.concatenate([np.repeat(sigma * self.areas / 3, 3), np.zeros(nt)])
        pot, _ = self.plan.execute(q)
        self.matvecs += 1
        return pot[3 * nt:] + self.correction @ sigma

    def solve(self, rtol: float = 1e-6, maxiter: int = 200):
        """GMRES (restart 50) to the relative residual rtol; the mixed form's
        matvec is accurate to ~1e-6, so smaller rtol needs precision="fp64"."""
        from scipy.sparse.linalg import LinearOperator, gmres
        nt = len(self.areas)
        A = LinearOperator((nt, nt), matvec=self.apply, dtype=np.float64)
        rhs = np.ones(nt)
        sigma, info = gmres(A, rhs, rtol=rtol, restart=50, maxiter=maxiter)
        if info != 0:
            raise RuntimeError(f"GMRES did not converge (info {info})")
        self.sigma = sigma
        return float(sigma @ self.areas)

    def close(self):
        self.plan.close()
