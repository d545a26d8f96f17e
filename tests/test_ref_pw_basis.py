"""This library's plane-wave basis (csrc/pw_basis.cpp, through the C-ABI) against the reference's own
PW_Basis_K set-up compiled from its sources (oracle/_ref; skipped where it was not built), set up as
ESolver_KS_PW sets up the wavefunction basis: the FFT grid, the plane waves of every k-point in the same
order (ig2ixyz) and their |k+G|^2, bit for bit, on every cell of the benchmark and test workloads."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import ref_david

pytestmark = pytest.mark.skipif(not ref_david.available(), reason="oracle/_ref/libref_david.so not built")

HEX = np.array([[1.0, 0.0, 0.0], [0.5, 0.8660254037844386, 0.0], [0.0, 0.0, 1.6]])
FCC = np.array([[-0.5, 0.0, 0.5], [0.0, 0.5, 0.5], [-0.5, 0.5, 0.0]])


def _cases(pkg):
    S = pkg.synth
    out = []
    for spec in [S.config(0), S.config(1), S.config(2), S.config(4)] + S.serving_cells():
        lv = np.diag(np.asarray(spec.latvec, dtype=np.float64))
        kd = np.zeros((1, 3)) if spec.kpts is None else np.asarray(spec.kpts)
        out.append((spec.name, spec.a, lv, spec.ecut, kd, spec.grid))
    out.append(("hexagonal_k", 7.0, HEX, 20.0, np.array([[0.1, 0.2, 0.3], [0.0, 0.5, 0.25]]), None))
    out.append(("fcc_k", 5.3233, FCC, 20.0, np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.0], [0.5, 0.0, 0.5]]), None))
    return out


def test_basis_matches_the_reference_setup(pkg):
    for name, lat0, lv, ecut, kd, grid in _cases(pkg):
        (nx, ny, nz), npwk, ig, g2 = ref_david.pw_basis_k(lat0, lv, ecut, kd, grid=grid)
        b = pkg.pwdft.PWBasisK(lat0, lv, ecut, kd, grid=grid)
        assert (b.nx, b.ny, b.nz) == (nx, ny, nz), name
        assert np.array_equal(b.npwk, npwk), name
        for ik in range(len(kd)):
            assert np.array_equal(b.ig2ixyz(ik), ig[ik]), (name, ik)
            assert np.array_equal(b.gk2_k(ik), g2[ik]), (name, ik)
