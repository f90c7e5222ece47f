"""The C++ drop-in header (include/lfmm.hpp): a reference-style caller
compiles and links against the library on the CPU; on the GPU its results
match the oracle (FP64 parity bar) and the direct sum."""
import subprocess
from collections import defaultdict

import numpy as np
import pytest

from laplace_fmm_b200.workloads import rel_l2

SRC = __import__("pathlib").Path(__file__).resolve().parent / "cpp" / "dropin.cpp"


@pytest.fixture(scope="module")
def dropin_bin(lib_path, tmp_path_factory):
    out = tmp_path_factory.mktemp("cpp") / "dropin"
    inc = lib_path.parent.parent / "include"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", str(inc), str(SRC), "-L",
                    str(lib_path.parent), "-llfmm", f"-Wl,-rpath,{lib_path.parent}", "-o", str(out)], check=True)
    return out


def test_dropin_compiles_and_links(dropin_bin):
    assert dropin_bin.exists()


@pytest.mark.gpu
def test_dropin_matches_oracle(dropin_bin, oracle):
    txt = subprocess.run([str(dropin_bin)], check=True, capture_output=True, text=True).stdout
    rows = defaultdict(list)
    for line in txt.splitlines():
        k, *v = line.split()
        rows[k].append([float(x) for x in v])
    p3, t3, p2 = (np.array(rows[k]) for k in ("p3", "t3", "p2"))
    a, b, c = (np.array(rows[k]) for k in ("a", "b", "c"))
    pot, fld = oracle.fmm3d(p3[:, :3], p3[:, 3], N=9, depth=4)
    assert rel_l2(a[:, 0], pot) < 1e-12 and rel_l2(a[:, 1:], fld) < 1e-12
    pot, fld = oracle.fmm3d(p3[:, :3], p3[:, 3], targets=t3, N=9, depth=4)
    assert rel_l2(b[:, 0], pot) < 1e-12 and rel_l2(b[:, 1:4], fld) < 1e-12
    pe, _ = oracle.direct3d(p3[:, :3], p3[:, 3], t3)
    assert rel_l2(b[:, 4], pe) < 1e-13
    pot, fld = oracle.fmm2d(p2[:, :2], p2[:, 2], N=16, depth=5)
    assert rel_l2(c[:, 0], pot) < 1e-12 and rel_l2(c[:, 1:], fld) < 1e-12
    v = np.array(rows["v"])                  # vector charges: position, q, field
    assert rel_l2(v[:, 6:], oracle.fmm3d_vec(v[:, :3], v[:, 3:6], N=8, depth=4)) < 5e-12
