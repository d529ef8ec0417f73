"""Shared fixtures. `-m "not gpu"` runs on CPU; GPU tests carry @pytest.mark.gpu."""
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "dielectricbie.jl_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def load_package():
    """Import the package directory `dielectricbie.jl_b200/` under the module name
    `dielectricbie_jl_b200` (the directory name is not a Python identifier)."""
    name = "dielectricbie_jl_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def bie():
    sys.path.insert(0, PKG_DIR)
    import build as _b  # noqa: E402  (in-tree build of libbie_b200.so)
    _b.build()
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle  # noqa: E402
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def rng():
    return np.random.default_rng(1234)
