"""The oracle's nonlocal H|psi> (oracle/hamilt_ref.py HamiltPWRef.nonlocal_act, which the device H|psi> is tested
against) against the reference's own Nonlocal operator (operator_pw/nonlocal_pw.cpp: init, act and
add_nonlocal_pp with the nonlocal_pw_op, gemm_op and gemv_op CPU functors), compiled from its source against
stand-ins for UnitCell and pseudopot_cell_vnl that hold the atom counts, projector counts, projectors and D.
Skipped where oracle/_ref was not built."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import hamilt_ref as H
from oracle import ref_david
from oracle.pw_basis_ref import PWBasisKRef

pytestmark = pytest.mark.skipif(not ref_david.available(), reason="oracle/_ref/libref_david.so not built")


def _ref_basis(spec):
    lv = np.diag(np.asarray(spec.latvec, dtype=np.float64))
    return PWBasisKRef(spec.a, lv, spec.ecut, np.zeros((1, 3)))


@pytest.mark.parametrize("cell,nb", [("config0", 1), ("config0", 5), ("config1", 2)])
def test_nonlocal_matches_the_reference_operator(pkg, cell, nb):
    """The 8-atom cell (one band: act's gemv branch; five: its gemm branch) and the headline 64-atom cell
    (npw 51 627, 512 projectors), the workloads' own projectors and D."""
    spec = pkg.synth.config(0 if cell == "config0" else 1)
    wl = pkg.pwdft.build_workload(spec)
    ld = wl.basis.npwk_max
    rb = _ref_basis(spec)
    vkb = wl.vkb_h[0][:, :ld]
    ham = H.HamiltPWRef(rb, 0, wl.veff_h, vkb, wl.deeq_h, [8], [wl.cell.nat])
    psi = wl.psi0_h[0][:nb].copy()
    h_o = np.zeros(nb * ld, dtype=np.complex128)
    ham.nonlocal_act(nb, ld, psi.reshape(-1), h_o)
    h_ref = ref_david.nonlocal_act([wl.cell.nat], [8], vkb, wl.deeq_h, psi, int(rb.npwk[0]))
    assert np.max(np.abs(h_ref.reshape(-1) - h_o)) <= 1e-14 * np.max(np.abs(h_o))


def test_nonlocal_two_atom_types_and_accumulation(pkg):
    """Two atom types with different projector counts (3 atoms of 4 projectors, 5 of 8: the sum / iat offsets
    of add_nonlocal_pp), a D that differs per atom and is not symmetric, and H psi accumulated onto a nonzero
    input (act adds to it)."""
    spec = pkg.synth.config(0)
    wl = pkg.pwdft.build_workload(spec)
    ld = wl.basis.npwk_max
    rb = _ref_basis(spec)
    npw = int(rb.npwk[0])
    rng = np.random.default_rng(21)
    na, nh = [3, 5], [4, 8]
    nkb = sum(a * h for a, h in zip(na, nh))
    vkb = rng.standard_normal((nkb, ld)) + 1j * rng.standard_normal((nkb, ld))
    vkb[:, npw:] = 0.0
    deeq = rng.uniform(-3.0, 3.0, size=(1, sum(na), 8, 8))
    nb = 3
    psi = rng.standard_normal((nb, ld)) + 1j * rng.standard_normal((nb, ld))
    h0 = rng.standard_normal((nb, ld)) + 1j * rng.standard_normal((nb, ld))
    ham = H.HamiltPWRef(rb, 0, wl.veff_h, vkb, deeq, nh, na)
    h_o = h0.reshape(-1).copy()
    ham.nonlocal_act(nb, ld, psi.reshape(-1), h_o)
    h_ref = ref_david.nonlocal_act(na, nh, vkb, deeq, psi, npw, hpsi=h0)
    assert np.max(np.abs(h_ref.reshape(-1) - h_o)) <= 1e-13 * np.max(np.abs(h_o))
