"""Shared fixtures.  Tests marked `gpu` need a CUDA device and the built library;
everything else runs on the CPU (oracle, golden vectors, host logic, C ABI exports)."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "static-priority-search-tree_b200"
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libpst_b200.so")


def load_package():
    if "pst_b200" in sys.modules:
        return sys.modules["pst_b200"]
    spec = importlib.util.spec_from_file_location("pst_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pst_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pst():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.Orc.lib()
    return o
