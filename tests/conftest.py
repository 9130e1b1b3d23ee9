"""Shared test set-up: load the package (as ``fcc_b200``) and the CPU oracle
(as ``fcc_oracle``), and register the ``gpu`` marker.

Tests marked ``gpu`` need a CUDA device and the built libfcc_b200.so; the
others run on the CPU (oracle against the golden fixtures, host logic, ABI
exports)."""

import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _load(name, path, pkg_dir=None):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[pkg_dir] if pkg_dir else None)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


PKG_DIR = os.path.join(ROOT, "fouriercontourcells.jl_b200")
fcc = _load("fcc_b200", os.path.join(PKG_DIR, "__init__.py"), PKG_DIR)
oracle = _load("fcc_oracle", os.path.join(ROOT, "oracle", "oracle.py"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built libfcc_b200.so")
    config.addinivalue_line("markers", "slow: long CPU oracle runs")


@pytest.fixture(scope="session")
def ref_n64():
    z = np.load(os.path.join(GOLDEN, "reference_N64.npz"))
    return z["init"], {int(k): z[f"snap_{k}"] for k in z["steps"]}


def deformed_coef(seed=3, maxmode=6, amplitude=0.04):
    """A deformed body well inside the shape bound (test/runtests.jl:18-23)."""
    rng = np.random.default_rng(seed)
    c = np.zeros(2 * maxmode - 1)
    c[1:] = amplitude * (2 * rng.random(2 * maxmode - 2) - 1)
    c[0] = np.sqrt(1 - np.sum(c[1:] ** 2) / 2)
    return c
