"""Shared fixtures: the CPU checker (oracle), the golden fixtures of the
reference, and the B200 platform package loaded from its in-tree directory."""
import importlib.util
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU and the CUDA library")


def _ensure_oracle():
    so = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    return so


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    from pyoracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "lmp_golden.npz")))


def load_platform():
    """Import hiflow3_2.0_b200 (its directory name is not a Python identifier)."""
    name = "hiflow3_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "hiflow3_2.0_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path,
                                                  submodule_search_locations=[os.path.dirname(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def b200():
    return load_platform()
