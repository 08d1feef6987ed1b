"""Shared test setup.

The package lives in the directory ``n-body-2d_b200`` (not an importable
name), so it is loaded here under the module name ``nbody_b200``.  Tests that
need a CUDA GPU carry ``@pytest.mark.gpu``; everything else runs on CPU.
"""
from __future__ import annotations

import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    if "nbody_b200" in sys.modules:
        return sys.modules["nbody_b200"]
    pkg = ROOT / "n-body-2d_b200"
    spec = importlib.util.spec_from_file_location(
        "nbody_b200", pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["nbody_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


@pytest.fixture(scope="session")
def nbp():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.load()
    return oracle


def rel_err(a, b, floor=0.0):
    import numpy as np

    num = np.linalg.norm(np.asarray(a) - np.asarray(b), axis=-1)
    den = np.maximum(np.linalg.norm(np.asarray(b), axis=-1), floor)
    return num / den


@pytest.fixture(scope="session")
def orc_render():
    from oracle import render_oracle

    return render_oracle
