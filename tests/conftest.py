"""Shared test set-up: the `gpu` marker and loaders for the product binding
(the package directory dynamical-cloud-model_b200/ is loaded under the
module name dcm_b200) and the oracle (test infrastructure)."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "dynamical-cloud-model_b200")


def load_dcm():
    if "dcm_b200" in sys.modules:
        return sys.modules["dcm_b200"]
    spec = importlib.util.spec_from_file_location(
        "dcm_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dcm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if os.path.join(ROOT, "oracle") not in sys.path:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # noqa: E402
    return oracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libdcm_b200.so")


@pytest.fixture(scope="session")
def dcm():
    return load_dcm()


@pytest.fixture(scope="session")
def orc():
    return load_oracle()
