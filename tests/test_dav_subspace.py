"""The Davidson-subspace oracle (oracle/dav_subspace_ref.py) against the reference's own CPU
Diago_DavSubspace, compiled from the reference sources (oracle/build_ref.py -> oracle/_ref; skipped where that
library was not built).  Same matrix, start vectors and preconditioner: the same iteration counts and the same
eigenvalues.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse

from oracle import ref_david
from oracle.dav_subspace_ref import DavSubspaceRef

pytestmark = pytest.mark.skipif(not ref_david.available(), reason="oracle/_ref/libref_david.so not built")


def _si2(golden):
    d = golden("pyabacus_si2")
    A = scipy.sparse.csc_matrix((d["data"], d["indices"], d["indptr"]), shape=tuple(d["shape"])).toarray()
    return A.astype(np.complex128)


@pytest.mark.parametrize("need_subspace,scf", [(False, False), (True, True)])
def test_reference_dav_subspace_pins_the_oracle_on_si2(golden, need_subspace, scf):
    A = _si2(golden)
    n, nband = A.shape[0], 8
    pc = np.abs(np.diag(A)).real  # a kinetic-like diagonal, as g2kin is for HSolverPW
    q, _ = np.linalg.qr(np.random.default_rng(5).standard_normal((n, nband)) + 0j)
    psi0 = np.ascontiguousarray(q.T)
    thr = 1e-10
    psi_r, e_r = psi0.copy(), np.zeros(nband)
    it_r = ref_david.dav_subspace(lambda x, nv, d, i0, i1: (A @ x[i0:i1 + 1].T).T, pc, nband, n, 4, n, psi_r, e_r,
                                  thr, 300, need_subspace, scf)
    psi_o, e_o = psi0.copy(), np.zeros(nband)
    it_o = DavSubspaceRef(pc, nband, n, 4, thr, 300, need_subspace).diag(lambda x: (A @ x.T).T, psi_o, e_o, scf)
    assert it_o == it_r
    assert np.max(np.abs(e_o - e_r)) < 1e-12
    w = np.linalg.eigvalsh(A)[:nband]
    assert np.max(np.abs(e_o - w)) < 1e-8


def test_reference_dav_subspace_pins_the_oracle_on_a_plane_wave_cell():
    """A 2-atom plane-wave cell (Si2 serving cell: 18^3 grid, 365 plane waves, 8 bands) through the oracle's
    H|psi>: the preconditioner is g2kin as HSolverPW gives this method."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from conftest import load_package
    from oracle import hamilt_ref as H
    from oracle.pw_basis_ref import PWBasisKRef
    pkg = load_package()
    spec = pkg.synth.serve_configs()[0] if hasattr(pkg.synth, "serve_configs") else pkg.synth.config(0)
    wl = pkg.pwdft.build_workload(spec)
    ld = wl.basis.npwk_max
    npw = int(wl.basis.npwk[0])
    ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, np.zeros((1, 3)), grid=spec.grid)
    ham = H.HamiltPWRef(ref_b, 0, wl.veff_h, wl.vkb_h[0][:, :ld], wl.deeq_h, [8], [wl.cell.nat])
    pc = H.precondition_dav_subspace(ref_b, 0)
    nb = min(spec.nbands, 16)
    psi0 = wl.psi0_h[0][:nb].copy()
    q, _ = np.linalg.qr(psi0[:, :npw].T)
    psi0[:, :npw] = q.T

    def hp(x):
        m = x.shape[0]
        y = np.zeros((m, ld), complex)
        y[:, :npw] = x
        return ham.hpsi(y.reshape(-1), m, ld).reshape(m, ld)[:, :npw]

    e_r, p_r = np.zeros(nb), np.ascontiguousarray(psi0.copy())
    it_r = ref_david.dav_subspace(lambda x, nv, d, i0, i1: hp(x[i0:i1 + 1, :npw]), pc, nb, npw, 4, ld, p_r, e_r, 1e-9,
                                  100)
    e_o, p_o = np.zeros(nb), psi0.copy()
    it_o = DavSubspaceRef(pc, nb, npw, 4, 1e-9, 100).diag(hp, p_o, e_o)
    assert it_o == it_r
    assert np.max(np.abs(e_o - e_r)) < 1e-11


@pytest.mark.parametrize("scf", [False, True])
def test_reference_dav_subspace_pins_the_empty_band_rule(scf):
    """Empty bands converge at max(5 thr, 1e-5) (diago_dav_subspace.cpp:186-194): the oracle and the compiled
    reference with the same occupation flags on a seeded Hermitian matrix."""
    rng = np.random.default_rng(21)
    n, nband = 240, 6
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    A = 0.05 * (a + a.conj().T) + np.diag(np.linspace(0.0, 20.0, n))
    pc = np.real(np.diag(A)).copy()
    q, _ = np.linalg.qr(rng.standard_normal((n, nband)) + 0j)
    psi0 = np.ascontiguousarray(q.T)
    occ = [True, True, True, False, False, False]
    thr = 1e-10
    psi_r, e_r = psi0.copy(), np.zeros(nband)
    it_r = ref_david.dav_subspace(lambda x, nv, d, i0, i1: (A @ x[i0:i1 + 1].T).T, pc, nband, n, 4, n, psi_r, e_r,
                                  thr, 300, False, scf, occupied=occ)
    psi_o, e_o = psi0.copy(), np.zeros(nband)
    it_o = DavSubspaceRef(pc, nband, n, 4, thr, 300).diag(lambda x: (A @ x.T).T, psi_o, e_o, scf, occ)
    assert it_o == it_r
    assert np.max(np.abs(e_o - e_r)) < 1e-12
    w = np.linalg.eigvalsh(A)[:nband]
    assert np.max(np.abs(e_o[:3] - w[:3])) < 1e-8
    e_all = np.zeros(nband)
    it_all = DavSubspaceRef(pc, nband, n, 4, thr, 300).diag(lambda x: (A @ x.T).T, psi0.copy(), e_all, scf)
    assert it_o < it_all  # the empty bands' looser threshold ends the solve earlier (21 against 31 iterations)
