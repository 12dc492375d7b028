"""Shared test setup: the `gpu` marker, the package loader and small fixtures.

The package lives in `dg-cfl-less-maxwell-solver_b200/` (not a Python
identifier) and is loaded under the name `gdon3d_b200`.  The oracle
(`oracle/`) is imported only here in tests, as the checker.
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "dg-cfl-less-maxwell-solver_b200")


def load_package():
    if "gdon3d_b200" in sys.modules:
        return sys.modules["gdon3d_b200"]
    spec = importlib.util.spec_from_file_location(
        "gdon3d_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gdon3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def has_gpu():
    import torch
    return torch.cuda.is_available()
