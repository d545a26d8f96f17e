"""The oracle's plane-wave transforms (oracle/hamilt_ref.py: sphere <-> box with a 3-D FFT) against the
reference's own PW_Basis_K::recip2real / real2recip <double> (pw_transform_k.cpp: stick scatter, z FFTs,
stick-to-plane transposition, x and y FFTs over the occupied columns, gather), compiled from its sources with
its FFT class; FFTW's lines evaluated by the oracle build's mixed-radix stand-in.  Skipped where oracle/_ref
was not built."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import hamilt_ref as H
from oracle import ref_david
from oracle.pw_basis_ref import PWBasisKRef

pytestmark = pytest.mark.skipif(not ref_david.available(), reason="oracle/_ref/libref_david.so not built")

HEX = np.array([[1.0, 0.0, 0.0], [0.5, 0.8660254037844386, 0.0], [0.0, 0.0, 1.6]])
CELLS = [
    (5.13, np.eye(3), 30.0, np.zeros((1, 3))),                                  # 18^3, Gamma
    (10.26, np.eye(3), 30.0, np.array([[0.0, 0.0, 0.0], [0.125, -0.375, 0.375]])),  # 36^3, second k-point
    (7.0, HEX, 20.0, np.array([[0.1, 0.2, 0.3]])),                               # 20 x 20 x 32, hexagonal
]


@pytest.mark.parametrize("case", range(len(CELLS)))
def test_transforms_match_the_reference(case):
    lat0, lv, ecut, kd = CELLS[case]
    ik = len(kd) - 1
    b = PWBasisKRef(lat0, lv, ecut, kd)
    npw, N = int(b.npwk[ik]), b.nx * b.ny * b.nz
    rng = np.random.default_rng(case)
    g = rng.standard_normal(npw) + 1j * rng.standard_normal(npw)
    r_ref = ref_david.pw_transform(lat0, lv, ecut, kd, ik, g, True)
    r_o = H.recip_to_real(b, g, ik)
    assert np.max(np.abs(r_ref - r_o)) < 1e-13 * np.max(np.abs(r_o))
    box = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    g_ref = ref_david.pw_transform(lat0, lv, ecut, kd, ik, box, False, factor=0.7)
    g_o = H.real_to_recip(b, box, ik, factor=0.7)
    assert np.max(np.abs(g_ref - g_o)) < 1e-13 * np.max(np.abs(g_o))
    # add = true accumulates (the form Veff::act uses)
    acc = rng.standard_normal(npw) + 1j * rng.standard_normal(npw)
    a_ref, a_o = acc.copy(), acc.copy()
    ref_david.pw_transform(lat0, lv, ecut, kd, ik, box, False, add=True, factor=1.3, out=a_ref)
    H.real_to_recip(b, box, ik, out=a_o, add=True, factor=1.3)
    assert np.max(np.abs(a_ref - a_o)) < 1e-13 * np.max(np.abs(a_o))
    r_acc = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    ra_ref, ra_o = r_acc.copy(), r_acc.copy()
    ref_david.pw_transform(lat0, lv, ecut, kd, ik, g, True, add=True, factor=0.5, out=ra_ref)
    H.recip_to_real(b, g, ik, out=ra_o, add=True, factor=0.5)
    assert np.max(np.abs(ra_ref - ra_o)) < 1e-13 * np.max(np.abs(ra_o))
