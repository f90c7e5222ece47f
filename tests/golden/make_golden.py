"""Generate the golden fixtures from the reference's own CPU FMM.

Runs the UNMODIFIED reference CPU path (built from its sources by
``make -C oracle ref`` into ``oracle/_ref/libfmmref.so``) with one thread
(its counting sort is then deterministic) on small seeded inputs, and stores
inputs, outputs, trees and Wigner-d tables as ``tests/golden/*.npz``.  The
fixtures pin the C oracle in the CPU tests and travel with the repository.

    make -C oracle ref && python tests/golden/make_golden.py [vector]
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle.oracle import Reference  # noqa: E402


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def tree_arrays(prefix, tree):
    out = {f"{prefix}targets_num": np.int64(tree["targets_num"]), f"{prefix}positions": tree["positions"]}
    for L, lv in enumerate(tree["levels"]):
        for k in ("code", "sb", "se", "tb", "te", "parent", "close_off", "close", "far_off", "far", "center"):
            out[f"{prefix}L{L}_{k}"] = lv[k]
    out[f"{prefix}depth"] = np.int64(len(tree["levels"]))
    return out


CASES_3D = [
    # name, n_src, n_tgt, N, depth, seed
    ("c3d_src", 2000, 0, 9, 4, 11),
    ("c3d_st", 1500, 700, 7, 4, 12),
    ("c3d_n18", 1200, 0, 18, 3, 13),
    ("c3d_deep", 600, 0, 5, 6, 14),
]
CASES_VEC = [
    # vector charges (reference FastMultipole3d<Vector3d>); zero_frac: share of
    # particles with q = 0 (the reference then makes them the targets)
    # name, n_src, n_tgt, N, depth, seed, zero_frac
    ("c3d_vec", 2000, 0, 9, 4, 31, 0.0),
    ("c3d_vec_st", 1500, 600, 8, 4, 32, 0.0),
    ("c3d_vec_zero", 1200, 0, 7, 4, 33, 0.1),
]
CASES_2D = [
    ("c2d_src", 2000, 0, 21, 5, 21),
    ("c2d_st", 1500, 600, 12, 5, 22),
    ("c2d_n30", 800, 0, 30, 4, 23),
]


def vector_cases(R):
    for name, ns, nt, N, D, seed, zf in CASES_VEC:
        g = rng(seed)
        src = g.random((ns, 3)); q = g.uniform(-1, 1, (ns, 3))
        if zf:
            q[g.random(ns) < zf] = 0.0
        tgt = g.random((nt, 3)) * 1.2 - 0.1 if nt else None
        fld = R.fmm3d_vec(src, q, targets=tgt, N=N, depth=D)
        d = dict(src=src, q=q, field=fld, N=np.int64(N), depth=np.int64(D))
        if tgt is not None:
            d["tgt"] = tgt
        np.savez_compressed(HERE / f"{name}.npz", **d)


def main():
    R = Reference()
    R.set_threads(1)
    if sys.argv[1:] == ["vector"]:          # the vector-charge fixtures alone
        vector_cases(R)
        print("wrote", sorted(p.name for p in HERE.glob("c3d_vec*.npz")))
        return
    vector_cases(R)
    for name, ns, nt, N, D, seed in CASES_3D:
        g = rng(seed)
        src = g.random((ns, 3)); q = g.uniform(-1, 1, ns)
        tgt = g.random((nt, 3)) * 1.2 - 0.1 if nt else None
        pot, fld = R.fmm3d(src, q, targets=tgt, N=N, depth=D)
        allp = src if tgt is None else np.concatenate([tgt, src])
        allq = q if tgt is None else np.concatenate([np.zeros(nt), q])
        tree = R.tree(3, allp, allq, D)
        d = dict(src=src, q=q, pot=pot, field=fld, N=np.int64(N), depth=np.int64(D), **tree_arrays("tree_", tree))
        if tgt is not None:
            d["tgt"] = tgt
        np.savez_compressed(HERE / f"{name}.npz", **d)
    for name, ns, nt, N, D, seed in CASES_2D:
        g = rng(seed)
        src = g.random((ns, 2)); q = g.uniform(-1, 1, ns)
        tgt = g.random((nt, 2)) * 1.2 - 0.1 if nt else None
        pot, fld = R.fmm2d(src, q, targets=tgt, N=N, depth=D)
        allp = src if tgt is None else np.concatenate([tgt, src])
        allq = q if tgt is None else np.concatenate([np.zeros(nt), q])
        tree = R.tree(2, allp, allq, D)
        d = dict(src=src, q=q, pot=pot, field=fld, N=np.int64(N), depth=np.int64(D), **tree_arrays("tree_", tree))
        if tgt is not None:
            d["tgt"] = tgt
        np.savez_compressed(HERE / f"{name}.npz", **d)
    thetas = np.array([0.3, 0.9553166181245093, 1.1, np.pi / 2, 2.5, -0.7, -2.9, 1e-6, np.pi - 1e-6])
    wd = np.stack([R.wignerd(18, t) for t in thetas])
    np.savez_compressed(HERE / "wignerd.npz", thetas=thetas, d=wd)
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
