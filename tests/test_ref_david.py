"""The Davidson oracle against the reference's own DiagoDavid, compiled from the reference sources
(oracle/build_ref.py -> oracle/_ref/libref_david.so; skipped where that library was not built).

Same matrix, same start vectors, same preconditioner: the restatement must take the same number of
iterations and reach the same eigenvalues.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse

from oracle import ref_david
from oracle.david_ref import DiagoDavidRef, copy_spsi

pytestmark = pytest.mark.skipif(not ref_david.available(), reason="oracle/_ref/libref_david.so not built")


def test_reference_david_pins_the_oracle_on_si2(golden):
    d = golden("pyabacus_si2")
    A = scipy.sparse.csc_matrix((d["data"], d["indices"], d["indptr"]), shape=tuple(d["shape"])).toarray()
    A = A.astype(np.complex128)
    n, nband = A.shape[0], 16
    diag = np.abs(np.diag(A)).real
    diag = np.where(diag < 1e-8, 1e-8, diag)
    psi0 = np.random.default_rng(12).random(n * nband).astype(np.complex128)
    psi_r, e_r = psi0.copy(), np.zeros(nband)
    it_r = ref_david.diag(lambda x, nv, dim, i0, i1: (A @ x[i0:i1 + 1].T).T, diag, nband, n, 8, n, psi_r, e_r,
                          1e-12, 5000)
    psi_o, e_o = psi0.copy(), np.zeros(nband)
    it_o = DiagoDavidRef(diag, nband, n, 8).diag(lambda x, nv: (A @ x.reshape(nv, n).T).T.reshape(-1), copy_spsi, n,
                                                  psi_o, e_o, 1e-12, 5000)
    assert it_o == it_r
    assert np.max(np.abs(e_o - e_r)) < 1e-12
    ref = np.sort(np.linalg.eigvalsh(A))[:nband]
    assert np.max(np.abs(e_r - ref)) < 1e-8


def test_reference_david_pins_the_oracle_on_a_plane_wave_hamiltonian(pkg):
    """The 2-atom serving cell (npw 365, 8 bands) with the oracle's H|psi>: the reference's Davidson and the
    restatement agree in iterations and eigenvalues."""
    from oracle import hamilt_ref as H
    from oracle.pw_basis_ref import PWBasisKRef
    spec = pkg.synth.serving_cells()[0]
    cell = pkg.synth.make_cell(spec)
    b = PWBasisKRef(spec.a, cell.latvec, spec.ecut, np.zeros((1, 3)))
    ld = int(b.npwk_max)
    ham = H.HamiltPWRef(b, 0, cell.veff(b.nx, b.ny, b.nz), cell.vkb(b.gplusk_cart(0), ld, b.omega), cell.deeq(), [8],
                        [cell.nat])
    nband = spec.nbands
    pc = H.precondition(b, 0)
    psi0 = cell.psi0(b.gplusk_cart(0), nband, ld).reshape(-1)
    psi_r, e_r = psi0.copy(), np.zeros(nband)
    it_r = ref_david.diag(lambda x, nv, dim, i0, i1: ham.hpsi(x[i0:i1 + 1].reshape(-1), i1 - i0 + 1, dim)
                          .reshape(i1 - i0 + 1, dim), pc, nband, ld, 4, ld, psi_r, e_r, 1e-10, 200)
    psi_o, e_o = psi0.copy(), np.zeros(nband)
    it_o = DiagoDavidRef(pc, nband, ld, 4).diag(lambda x, nv: ham.hpsi(x, nv, ld), copy_spsi, ld, psi_o, e_o, 1e-10, 200)
    assert it_o == it_r
    assert np.max(np.abs(e_o - e_r)) < 1e-11
