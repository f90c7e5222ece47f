"""The C oracle against the golden fixtures (made by the unmodified reference)
and, where it is built here, against the reference itself.  CPU only."""
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import AUTO, rel_l2

GOLD = Path(__file__).resolve().parent / "golden"
CASES3 = ["c3d_src", "c3d_st", "c3d_n18", "c3d_deep"]
CASES2 = ["c2d_src", "c2d_st", "c2d_n30"]


def load(name):
    return dict(np.load(GOLD / f"{name}.npz"))


def golden_tree(g):
    D = int(g["tree_depth"])
    levels = []
    for L in range(D):
        levels.append({k: g[f"tree_L{L}_{k}"] for k in
                       ("code", "sb", "se", "tb", "te", "parent", "close_off", "close", "far_off", "far", "center")})
    return dict(levels=levels, positions=g["tree_positions"], targets_num=int(g["tree_targets_num"]))


@pytest.mark.parametrize("name", CASES3)
def test_oracle_fmm3d_matches_golden(oracle, name):
    g = load(name)
    pot, fld = oracle.fmm3d(g["src"], g["q"], targets=g.get("tgt"), N=int(g["N"]), depth=int(g["depth"]))
    assert rel_l2(pot, g["pot"]) < 1e-13
    assert rel_l2(fld, g["field"]) < 1e-13


@pytest.mark.parametrize("name", CASES2)
def test_oracle_fmm2d_matches_golden(oracle, name):
    g = load(name)
    pot, fld = oracle.fmm2d(g["src"], g["q"], targets=g.get("tgt"), N=int(g["N"]), depth=int(g["depth"]))
    assert rel_l2(pot, g["pot"]) < 1e-13
    assert rel_l2(fld, g["field"]) < 1e-13


@pytest.mark.parametrize("name", CASES3 + CASES2)
def test_oracle_tree_matches_golden(oracle, name):
    """Codes, ranges, parents, the reference's (halved) lists in order, and
    the particle permutation: bit-exact.  Centres to the last bits (the
    reference binary fuses x*scale+shift into an FMA on some levels)."""
    g = load(name)
    dim = g["src"].shape[1]
    pts = g["src"] if "tgt" not in g else np.concatenate([g["tgt"], g["src"]])
    q = g["q"] if "tgt" not in g else np.concatenate([np.zeros(len(g["tgt"])), g["q"]])
    D = int(g["depth"])
    a = oracle.tree(dim, pts, q, D)
    b = golden_tree(g)
    assert a["targets_num"] == b["targets_num"]
    np.testing.assert_array_equal(a["positions"], b["positions"])
    for L in range(D):
        A, B = a["levels"][L], b["levels"][L]
        keys = ["code", "sb", "se", "close_off", "close", "far_off", "far"]
        keys += ["tb", "te"] if L == D - 1 else []
        keys += ["parent"] if L else []
        for k in keys:
            np.testing.assert_array_equal(A[k], B[k], err_msg=f"{name} level {L} {k}")
        np.testing.assert_allclose(A["center"], B["center"], rtol=0, atol=4e-16)


def test_oracle_wignerd_matches_golden(oracle):
    g = load("wignerd")
    for th, d in zip(g["thetas"], g["d"]):
        mine = oracle.wignerd(18, th)
        # the high-degree recurrence amplifies the reference binary's FMA rounding
        assert np.abs(mine - d).max() < 1e-11


def test_direction_tables(oracle):
    """316 far offsets collapse to 49 theta keys (97 signed) and 33 phi keys
    in the reference's int(100*angle) hashing."""
    assert oracle.direction_key_counts() == (49, 97, 33)


def test_runtime_angles_hit_table_keys(oracle):
    """Every far offset, at every level scale, hashes to the table angle of
    its canonical integer direction (so a per-direction table is exact)."""
    for dx in range(-3, 4):
        for dy in range(-3, 4):
            for dz in range(-3, 4):
                if max(abs(dx), abs(dy), abs(dz)) < 2:
                    continue
                v0 = np.array([dx, dy, dz], float)
                r0 = np.linalg.norm(v0) + 1e-12
                th0 = np.arccos(dz / r0)
                st0, t0, p0 = oracle.table_angles(th0, np.arctan2(dy, dx) if dx or dy else 0.0)
                assert st0 == 0
                for lvl in range(1, 21):
                    h = 1.000001 / 2 ** lvl
                    v = v0 * h
                    r = np.linalg.norm(v) + 1e-12
                    th = np.arccos(v[2] / r)
                    ph = 0.0 if abs(v[0]) + abs(v[1]) < 1e-12 else (
                        np.sign(v[1]) * np.pi / 2 if abs(v[0]) < 1e-12 else np.arctan2(v[1], v[0]))
                    st, t, p = oracle.table_angles(th, ph)
                    assert st == 0 and t == t0 and p == p0, (dx, dy, dz, lvl)


def test_oracle_vs_direct(oracle):
    g = np.random.Generator(np.random.PCG64(5))
    src = g.random((3000, 3)); q = g.uniform(-1, 1, 3000)
    pot, fld = oracle.fmm3d(src, q, N=13, depth=4)
    pe, fe = oracle.direct3d(src, q, src)
    self_term = q * 1e4
    assert rel_l2(pot - self_term, pe - self_term) < 5e-6
    assert rel_l2(fld, fe) < 5e-6


def test_oracle_vs_reference_live(oracle, reference):
    """Where the reference builds here: same inputs, norm-wise 1e-13."""
    g = np.random.Generator(np.random.PCG64(99))
    src = g.random((20000, 3)); q = g.uniform(-1, 1, 20000)
    p1, f1 = oracle.fmm3d(src, q, N=11, depth=5)
    p2, f2 = reference.fmm3d(src, q, N=11, depth=5)
    assert rel_l2(p1, p2) < 1e-13 and rel_l2(f1, f2) < 1e-13
    src2 = g.random((20000, 2)); q2 = g.uniform(-1, 1, 20000)
    p1, f1 = oracle.fmm2d(src2, q2, N=21, depth=6)
    p2, f2 = reference.fmm2d(src2, q2, N=21, depth=6)
    assert rel_l2(p1, p2) < 1e-13 and rel_l2(f1, f2) < 1e-13


def test_auto_order_and_depth(oracle, reference):
    g = np.random.Generator(np.random.PCG64(3))
    src = g.random((5000, 3)); q = g.uniform(-1, 1, 5000)
    p1, _ = oracle.fmm3d(src, q, N=AUTO, depth=AUTO, eps=1e-6)
    p2, _ = reference.fmm3d(src, q, N=AUTO, depth=AUTO, eps=1e-6)
    assert rel_l2(p1, p2) < 1e-13
