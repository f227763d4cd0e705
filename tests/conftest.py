import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "anc-field_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _load_pkg():
    if "ancfield_b200" in sys.modules:
        return sys.modules["ancfield_b200"]
    spec = importlib.util.spec_from_file_location("ancfield_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ancfield_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_pkg()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def pkg():
    return _load_pkg()
