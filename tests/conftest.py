"""Test configuration: the `gpu` marker, and loaders for the engine package and the oracle.

`-m "not gpu"` runs everything that needs no GPU (oracle pins, C-ABI exports, host logic,
gloo multi-process tests); `-m gpu` runs the parity tests through the C ABI on a B200.
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "financial-derivatives-montecarlo_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_engine():
    name = "fdmc_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def eng():
    return load_engine()


@pytest.fixture(scope="session")
def orc():
    import oracle_py
    return oracle_py


@pytest.fixture(scope="session")
def gpu(eng):
    eng.init(0)
    yield eng
