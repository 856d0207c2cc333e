"""Shared test setup: the `gpu` marker, package loading and fixture paths."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    """Import trhepd-opt_b200/ (hyphenated directory) as `trhepd_opt_b200`."""
    name = "trhepd_opt_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = ROOT / "trhepd-opt_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def spot_errors(got, ref, floor=1e-6):
    """(max |d| / row max, max relative error over spots >= floor * row max)."""
    import numpy as np
    got = np.asarray(got)
    ref = np.asarray(ref)
    rowmax = np.maximum(np.abs(ref).max(axis=1, keepdims=True), 1e-300)
    d = np.abs(got - ref)
    big = np.abs(ref) >= floor * rowmax
    rel = np.where(big, d / np.where(big, np.abs(ref), 1.0), 0.0)
    return float((d / rowmax).max()), float(rel.max())


@pytest.fixture(scope="session")
def golden():
    return GOLDEN


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.build()
    O.set_threads()
    return O
