"""Shared pytest set-up: the ``gpu`` marker and the package loader."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and the built CUDA library")


def load_package():
    """Import the ``abacus-develop_b200`` directory as module ``abacus_develop_b200``."""
    name = "abacus_develop_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = ROOT / "abacus-develop_b200"
    spec = importlib.util.spec_from_file_location(name, pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def _load(name):
        return np.load(ROOT / "tests" / "golden" / f"{name}.npz")
    return _load
