"""The oracle's kinetic + local H|psi> (oracle/hamilt_ref.py, which the device H|psi> is tested against) against
the reference's own operators Ekinetic and Veff (operator_pw/ekinetic_pw.cpp, veff_pw.cpp with their CPU
kernels and PW_Basis_K's transforms), compiled from its sources and chained as Operator::hPsi chains them.
Skipped where oracle/_ref was not built."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import hamilt_ref as H
from oracle import ref_david
from oracle.pw_basis_ref import PWBasisKRef

pytestmark = pytest.mark.skipif(not ref_david.available(), reason="oracle/_ref/libref_david.so not built")


@pytest.mark.parametrize("cell", ["serve0", "config0", "config1"])
def test_local_hpsi_matches_the_reference_operators(pkg, cell):
    """18^3, 36^3 and the headline 64-atom cell (96^3, npw 51627)."""
    spec = {"serve0": pkg.synth.serving_cells()[0], "config0": pkg.synth.config(0),
            "config1": pkg.synth.config(1)}[cell]
    wl = pkg.pwdft.build_workload(spec)
    ld = wl.basis.npwk_max
    lv = np.diag(np.asarray(spec.latvec, dtype=np.float64))
    rb = PWBasisKRef(spec.a, lv, spec.ecut, np.zeros((1, 3)))
    ham = H.HamiltPWRef(rb, 0, wl.veff_h, wl.vkb_h[0][:, :ld], wl.deeq_h, [8], [wl.cell.nat])
    nb = 4 if cell != "config1" else 2
    psi = wl.psi0_h[0][:nb].copy()
    h_ref = ref_david.hpsi_local(spec.a, lv, spec.ecut, np.zeros((1, 3)), 0, wl.veff_h, psi, nb)
    h_o = ham.hpsi_local(psi.reshape(-1), nb, ld).reshape(nb, ld)
    assert np.max(np.abs(h_ref - h_o)) < 1e-13 * np.max(np.abs(h_o))
