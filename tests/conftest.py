"""Shared fixtures.  `gpu` marks tests that need a B200 (they call the CUDA
library through its C ABI); everything else runs on the CPU."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a); calls the library through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import ORACLE_SO, Oracle, build
    if not ORACLE_SO.exists():
        build(("oracle",))
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import REF_SO, Reference
    if not REF_SO.exists():
        pytest.skip("reference CPU build (oracle/_ref) not present")
    r = Reference()
    r.set_threads(1)
    return r


@pytest.fixture(scope="session")
def lib_path():
    from laplace_fmm_b200 import build as b
    if not b.LIB.exists():
        b.build()
    return b.LIB


@pytest.fixture(scope="session")
def ctx(lib_path):
    from laplace_fmm_b200 import default_context
    return default_context(0)
