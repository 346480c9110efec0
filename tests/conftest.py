"""Shared fixtures: load the product package (directory name is not an identifier)
as `scphd_b200`, and the oracle (test infrastructure) as `oracle`."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "scphd-camera-calibration_b200")


def load_package():
    if "scphd_b200" in sys.modules:
        return sys.modules["scphd_b200"]
    spec = importlib.util.spec_from_file_location(
        "scphd_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["scphd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import oracle.oracle as orc  # noqa: E402
    return orc


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    o = load_oracle()
    o.lib()
    return o


@pytest.fixture(scope="session")
def ref(orc):
    try:
        return orc.RefLib()
    except FileNotFoundError:
        pytest.skip("oracle/_ref/libscphd_ref.so not built (reference sources absent)")
