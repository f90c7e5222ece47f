"""Vector charges (reference FastMultipole3d<Vector3d>): the oracle's
restatement against the golden fixtures written by the reference's own
vector build, and against the direct vector sum."""
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"


def rel_l2(x, ref):
    return float(np.linalg.norm(np.asarray(x) - ref) / np.linalg.norm(ref))


@pytest.mark.parametrize("name", ["c3d_vec", "c3d_vec_st", "c3d_vec_zero"])
def test_oracle_matches_reference_fixture(oracle, name):
    g = dict(np.load(GOLD / f"{name}.npz"))
    B = oracle.fmm3d_vec(g["src"], g["q"], g.get("tgt"), N=int(g["N"]), depth=int(g["depth"]))
    assert rel_l2(B, g["field"]) < 1e-13


def test_fixture_is_the_cross_product_field():
    """B_i = sum_j q_j x (x_i - x_j) / max(r, 1e-4)^3: the FMM fixture is
    within its truncation error (N = 9) of the direct sum."""
    g = dict(np.load(GOLD / "c3d_vec.npz"))
    src, q = g["src"], g["q"]
    d = src[:, None, :] - src[None, :, :]
    r = np.maximum(np.linalg.norm(d, axis=2), 1e-4)
    B = (np.cross(q[None, :, :], d) / r[:, :, None] ** 3).sum(axis=1)
    assert rel_l2(g["field"], B) < 1e-4


def test_partial_zero_charges_are_refused(oracle):
    g = np.random.default_rng(5)
    src = g.random((50, 3)); q = g.uniform(-1, 1, (50, 3))
    q[3, 1] = 0.0
    with pytest.raises(ValueError):
        oracle.fmm3d_vec(src, q, N=5, depth=2)
