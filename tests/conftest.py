"""Shared test setup: the `gpu` marker, the product package (directory
sdf-slam_b200, imported as sdf_slam_b200) and the CPU oracle (oracle/)."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def _load_package():
    if "sdf_slam_b200" in sys.modules:
        return sys.modules["sdf_slam_b200"]
    pkg_dir = os.path.join(ROOT, "sdf-slam_b200")
    spec = importlib.util.spec_from_file_location(
        "sdf_slam_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sdf_slam_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the GPU path")
