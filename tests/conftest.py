"""Shared pytest setup: the `gpu` marker, the package loader and helpers.

The package directory is named ``gilaelectromagnetics.jl_b200`` (not an
importable identifier), so it is loaded here under the module name
``gila_b200``.
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "gilaelectromagnetics.jl_b200")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_pkg():
    if "gila_b200" in sys.modules:
        return sys.modules["gila_b200"]
    spec = importlib.util.spec_from_file_location(
        "gila_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gila_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def gila():
    return load_pkg()


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128).ravel(order="F")
    b = np.asarray(b, dtype=np.complex128).ravel(order="F")
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# relative-L2 tolerances against the FP64 oracle
TOL_F64 = 1e-12
TOL_F32 = 1e-5
