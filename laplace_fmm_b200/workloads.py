"""Seeded synthetic particle sets for the benchmark and test configurations.

No public dataset is involved: every configuration is synthetic, generated
with numpy's PCG64 from a fixed seed, with the shapes, sizes and value
distributions of the configurations the solver is measured on.

* ``uniform3d``      -- uniform i.i.d. in [0,1]^3, q ~ U(-1, 1)  (3D uniform, 131,072 by default)
* ``clustered2d``    -- half uniform in the unit square, half on 64 Gaussian
                        clusters (sigma 0.005, centres uniform), rejected to the
                        open square; q ~ U(-1, 1)  (2D clustered, 4,194,304)
* ``plummer_mix3d``  -- half Plummer sphere (scale radius 0.05, centred at
                        0.5, truncated to the unit cube), half uniform;
                        q ~ U(-1, 1)  (3D clustered, 16,777,216)
* ``gaussian_mix3d`` -- 1-8 isotropic Gaussian clusters, sigma log-uniform in
                        [0.005, 0.2] (order-selection training problems)
* ``sample_targets`` -- the 4096 seeded target indices used for accuracy
"""
from __future__ import annotations

import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def uniform3d(n: int, seed: int = 12345):
    g = _rng(seed)
    pos = g.random((n, 3))
    q = g.uniform(-1.0, 1.0, n)
    return pos, q


def _in_open_cube(p, dim):
    return np.all((p > 0.0) & (p < 1.0), axis=1)


def clustered2d(n: int, seed: int = 4242, clusters: int = 64, sigma: float = 0.005):
    g = _rng(seed)
    nu = n // 2
    nc = n - nu
    uni = g.random((nu, 2))
    centres = g.random((clusters, 2))
    out = np.empty((0, 2))
    while len(out) < nc:
        k = g.integers(0, clusters, 2 * (nc - len(out)) + 16)
        p = centres[k] + sigma * g.standard_normal((len(k), 2))
        out = np.concatenate([out, p[_in_open_cube(p, 2)]])
    pos = np.concatenate([uni, out[:nc]])
    q = g.uniform(-1.0, 1.0, n)
    return pos, q


def plummer(n: int, g, a: float = 0.05, centre=0.5):
    out = np.empty((0, 3))
    while len(out) < n:
        m = 2 * (n - len(out)) + 16
        u = g.random(m)
        u = np.clip(u, 1e-12, 1.0 - 1e-12)
        r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        v = g.standard_normal((m, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        p = centre + r[:, None] * v
        out = np.concatenate([out, p[_in_open_cube(p, 3)]])
    return out[:n]


def plummer_mix3d(n: int, seed: int = 2024, a: float = 0.05):
    g = _rng(seed)
    npl = n // 2
    pos = np.concatenate([plummer(npl, g, a), g.random((n - npl, 3))])
    q = g.uniform(-1.0, 1.0, n)
    return pos, q


def gaussian_mix3d(n: int, seed: int, kmin: int = 1, kmax: int = 8, smin: float = 0.005, smax: float = 0.2):
    g = _rng(seed)
    k = int(g.integers(kmin, kmax + 1))
    centres = g.random((k, 3))
    sig = np.exp(g.uniform(np.log(smin), np.log(smax), k))
    out = np.empty((0, 3))
    while len(out) < n:
        m = 2 * (n - len(out)) + 16
        c = g.integers(0, k, m)
        p = centres[c] + sig[c, None] * g.standard_normal((m, 3))
        out = np.concatenate([out, p[_in_open_cube(p, 3)]])
    q = g.uniform(-1.0, 1.0, n)
    return out[:n], q


def sample_targets(n: int, k: int = 4096, seed: int = 777):
    """k distinct particle indices (all of them when n <= k)."""
    if n <= k:
        return np.arange(n)
    g = _rng(seed)
    return np.sort(g.choice(n, size=k, replace=False))


def rel_l2(x, ref):
    x = np.asarray(x); ref = np.asarray(ref)
    return float(np.linalg.norm((x - ref).ravel()) / np.linalg.norm(ref.ravel()))


def batch3d(count: int = 1024, seed: int = 5150, nmin: int = 2048, nmax: int = 262144, sigma: float = 0.05):
    """Uneven independent problems: sizes log-uniform in [nmin, nmax], each
    uniform in its own unit cube or one Gaussian cluster (sigma) with equal
    probability, charges uniform in [-1, 1].  Returns a list of (pos, q)."""
    g = _rng(seed)
    out = []
    for _ in range(count):
        n = int(round(np.exp(g.uniform(np.log(nmin), np.log(nmax)))))
        if g.random() < 0.5:
            pos = g.random((n, 3))
        else:
            c = g.uniform(0.2, 0.8, 3)
            pos = np.empty((0, 3))
            while len(pos) < n:
                p = c + sigma * g.standard_normal((2 * (n - len(pos)) + 16, 3))
                pos = np.concatenate([pos, p[_in_open_cube(p, 3)]])
            pos = pos[:n]
        out.append((pos, g.uniform(-1.0, 1.0, n)))
    return out
