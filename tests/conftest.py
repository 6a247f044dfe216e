"""Test setup: the `gpu` marker, the product package (registered as `btd_b200`) and the oracle."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _load_package():
    if "btd_b200" in sys.modules:
        return sys.modules["btd_b200"]
    pkg = os.path.join(ROOT, "break-that-denim_b200")
    spec = importlib.util.spec_from_file_location("btd_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["btd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")
