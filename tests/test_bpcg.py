"""The BPCG oracle (oracle/bpcg_ref.py) against the reference's own CPU DiagoBPCG, compiled from the
reference sources (oracle/build_ref.py -> oracle/_ref; the pins are skipped where that library was not
built).  Same matrix, start vectors and preconditioner: the same eigenvalues and vectors after a diag call.

BPCG's later calls are sensitive to rounding once the bands have converged (the normalised gradients are
then rounding noise): the reference itself, restarted from a start perturbed by 1e-14, differs by 1e-2 Ry
after its second call on Si2.mat.  So the pins compare one call at a time from the same start; convergence
over many calls is checked against the dense spectrum.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse

from oracle import ref_david
from oracle.bpcg_ref import DiagoBPCGRef

need_ref = pytest.mark.skipif(not ref_david.available(), reason="oracle/_ref/libref_david.so not built")


def _si2(golden):
    d = golden("pyabacus_si2")
    A = scipy.sparse.csc_matrix((d["data"], d["indices"], d["indptr"]), shape=tuple(d["shape"])).toarray()
    return A.astype(np.complex128)


def _start(n, nband, seed):
    q, _ = np.linalg.qr(np.random.default_rng(seed).standard_normal((n, nband))
                        + 1j * np.random.default_rng(seed + 1).standard_normal((n, nband)))
    return np.ascontiguousarray(q.T)


def _prec(A):
    g = np.abs(np.diag(A)).real
    return 1.0 + g + np.sqrt(1.0 + (g - 1.0) ** 2)


@need_ref
@pytest.mark.parametrize("scf_iter", [1, 2])
def test_reference_bpcg_pins_the_oracle_on_si2(golden, scf_iter):
    A = _si2(golden)
    n, nb = A.shape[0], 8
    pc = _prec(A)
    o = DiagoBPCGRef(pc, nb, n)
    p_o = _start(n, nb, 5)
    e_o = np.zeros(nb)
    for call in range(3):
        start = p_o.copy()
        o.diag(lambda x: (A @ x.T).T, p_o, e_o, scf_iter)
        p_r, e_r = start.copy(), np.zeros(nb)
        ref_david.bpcg(lambda x, nv, d, i0, i1: (A @ x[i0:i1 + 1].T).T, pc, nb, n, p_r, e_r, scf_iter, 1)
        assert np.max(np.abs(e_o - e_r)) < 1e-11, (call, e_o - e_r)
        ov = np.abs(np.sum(np.conj(p_o) * p_r, axis=1))  # the same vectors up to the eigensolver's phases
        assert np.max(np.abs(ov - 1.0)) < 1e-9, (call, ov)


def test_bpcg_oracle_converges_to_the_dense_spectrum(golden):
    A = _si2(golden)
    n, nb = A.shape[0], 8
    o = DiagoBPCGRef(_prec(A), nb, n)
    p, e = _start(n, nb, 7), np.zeros(nb)
    for _ in range(16):  # converged (every residual below 1e-5) after 14 calls from this start
        o.diag(lambda x: (A @ x.T).T, p, e, 1)
    w = np.linalg.eigvalsh(A)[:nb]
    assert np.max(np.abs(e - w)) < 1e-8, e - w
    assert np.max(o.err) < 1e-5


@need_ref
def test_reference_bpcg_pins_the_oracle_on_a_plane_wave_cell():
    """The 2-atom plane-wave cell (18^3 grid, 365 plane waves) through the oracle's H|psi>, 8 bands, the
    first-SCF-step schedule (24 iterations, Rayleigh-Ritz every 4)."""
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
    pc = H.precondition(ref_b, 0)[:npw]
    nb = 8
    q, _ = np.linalg.qr(wl.psi0_h[0][:nb, :npw].T)
    psi0 = np.ascontiguousarray(q.T)

    def hp(x):
        m = x.shape[0]
        y = np.zeros((m, ld), complex)
        y[:, :npw] = x
        return ham.hpsi(y.reshape(-1), m, ld).reshape(m, ld)[:, :npw]

    p_r, e_r = psi0.copy(), np.zeros(nb)
    ref_david.bpcg(lambda x, nv, d, i0, i1: hp(x[i0:i1 + 1]), pc, nb, npw, p_r, e_r, 1, 1)
    p_o, e_o = psi0.copy(), np.zeros(nb)
    DiagoBPCGRef(pc, nb, npw).diag(hp, p_o, e_o, 1)
    assert np.max(np.abs(e_o - e_r)) < 1e-11
    assert np.max(np.abs(np.abs(np.sum(np.conj(p_o) * p_r, axis=1)) - 1.0)) < 1e-9
