"""Shared fixtures. Tests marked `gpu` need a B200; everything else runs on CPU."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "lib", "libbh_oracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       capture_output=True)


def _ensure_product():
    from nbodysim_b200 import build
    build.build()


@pytest.fixture(scope="session")
def oracle_mod():
    _ensure_oracle()
    import oracle
    return oracle


@pytest.fixture(scope="session")
def orc(oracle_mod):
    return oracle_mod.Oracle()


@pytest.fixture(scope="session")
def ref(oracle_mod):
    """The reference's own CPU code; skipped where oracle/_ref was not built."""
    if not os.path.exists(oracle_mod.REF_LIB):
        pytest.skip("reference harness not built (oracle/_ref)")
    return oracle_mod.Reference()


@pytest.fixture(scope="session")
def nb():
    _ensure_product()
    import nbodysim_b200
    nbodysim_b200.load_library()
    return nbodysim_b200


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    d = os.path.join(ROOT, "tests", "golden")
    return lambda name: np.load(os.path.join(d, name))
