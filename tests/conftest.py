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


@pytest.fixture(scope="session")
def diamond8_dense_h(pkg):
    """8-atom cell (config 0): workload, the oracle's H assembled column by column (npw 2945), its spectrum
    and the oracle's basis (for the preconditioners)."""
    import numpy as np
    from oracle import hamilt_ref as H
    from oracle.pw_basis_ref import PWBasisKRef
    spec = pkg.synth.config(0)
    wl = pkg.pwdft.build_workload(spec)
    ld = wl.basis.npwk_max
    npw = int(wl.basis.npwk[0])
    ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, np.zeros((1, 3)))
    ref = H.HamiltPWRef(ref_b, 0, wl.veff_h, wl.vkb_h[0][:, :ld], wl.deeq_h, [8], [wl.cell.nat])
    eye = np.zeros((npw, ld), complex)
    eye[np.arange(npw), np.arange(npw)] = 1.0
    hm = np.zeros((npw, npw), complex)
    for i in range(0, npw, 256):
        nb = min(256, npw - i)
        hm[:, i:i + nb] = ref.hpsi(eye[i:i + nb].reshape(-1), nb, ld).reshape(nb, ld)[:, :npw].T
    return wl, hm, np.linalg.eigvalsh(hm), ref_b
