"""The C-ABI library loads without a GPU and exports every symbol that
include/lfmm.h declares; the host mirror rejects bad input before any compute."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "lfmm.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lfmm\w*)\s*\(", text)))


def test_library_exports_header(lib_path):
    import ctypes
    lib = ctypes.CDLL(str(lib_path))
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/lfmm.h but not exported"


def test_exports_list_matches_header():
    from laplace_fmm_b200._lib import EXPORTS
    assert sorted(EXPORTS) == header_symbols()


def test_version_without_gpu(lib_path):
    import ctypes
    lib = ctypes.CDLL(str(lib_path))
    assert lib.lfmm_version() >= 100


def test_null_context_is_an_error(lib_path):
    import ctypes
    lib = ctypes.CDLL(str(lib_path))
    lib.lfmm3d_solve.argtypes = [ctypes.c_void_p] * 13
    assert lib.lfmm3d_solve(None, 0, None, None, 0, None, 0, 0, None, 0, None, None, None) == -1


def test_particle_layouts():
    import numpy as np
    from laplace_fmm_b200 import particle2d_dtype, particle3d_dtype
    from laplace_fmm_b200.fmm import _split
    assert particle3d_dtype.itemsize == 40 and particle2d_dtype.itemsize == 32
    a = np.zeros(4, particle3d_dtype)
    a["center"] = np.arange(12).reshape(4, 3)
    a["q"] = [1, 2, 3, 4]
    pos, q = _split(a, 3)
    assert pos.shape == (4, 3) and q.tolist() == [1, 2, 3, 4]
    b = np.zeros(3, particle2d_dtype)
    b["center"] = [1 + 2j, 3 + 4j, 5 + 6j]
    pos, q = _split(b, 2)
    assert pos.tolist() == [[1, 2], [3, 4], [5, 6]]
    with pytest.raises(ValueError):
        _split((np.zeros((3, 3)), np.zeros(2)), 3)
