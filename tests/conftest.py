"""Test configuration: registers the ``gpu`` marker and makes the engine
package importable as ``tf_pwa_b200`` from its ``tf-pwa_b200`` directory."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _load_pkg():
    if "tf_pwa_b200" in sys.modules:
        return
    d = os.path.join(ROOT, "tf-pwa_b200")
    spec = importlib.util.spec_from_file_location(
        "tf_pwa_b200", os.path.join(d, "__init__.py"), submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["tf_pwa_b200"] = m
    spec.loader.exec_module(m)


_load_pkg()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
