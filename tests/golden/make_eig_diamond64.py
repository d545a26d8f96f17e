"""Eigenvalue fixture of the 64-atom cell (eig_diamond64.npz), made on the host by the oracle.

The workload is the 64-atom diamond supercell (a = 20.52 bohr, ecut 50 Ry, 96^3 grid, npw 51 627, 512
projectors, Gamma point) from this package's seeded synthetic generators (V_eff, beta, D, start vectors).
H|psi> is the oracle's restatement of Operator::hPsi (oracle/hamilt_ref.py: Ekinetic, Veff through the
reference's stick transforms, Nonlocal), which agrees with the reference's own Ekinetic and Veff operators
to 1e-16 on this cell.  The Davidson iteration is the reference's own DiagoDavid<complex<double>, CPU>
compiled from its sources (oracle/_ref/libref_david.so, built by oracle/build_ref.py), driven through the
oracle's H|psi>: pw_diag_ndim 4, the reference's preconditioner, thr 1e-11, the package's start vectors.
Where that library is absent the numpy restatement of DiagoDavid (oracle/david_ref.py, pinned to it
iteration for iteration) runs instead; the fixture records which ran.

Stored: the 160 eigenvalues (Ry), the iteration count, thr, the solver that ran, and the largest residual
norm |H x - e x| of the returned vectors (a-posteriori bound on each eigenvalue's error).

Run from the repository root:  python tests/golden/make_eig_diamond64.py   (about 10 minutes on 8 cores)
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import hamilt_ref as H  # noqa: E402
from oracle import ref_david  # noqa: E402
from oracle.david_ref import DiagoDavidRef, copy_spsi  # noqa: E402
from oracle.pw_basis_ref import PWBasisKRef  # noqa: E402
from tests.conftest import load_package  # noqa: E402

THR = 1e-11
OUT = Path(__file__).resolve().parent / "eig_diamond64.npz"


def main():
    pkg = load_package()
    spec = pkg.synth.config(1)
    wl = pkg.pwdft.build_workload(spec)
    k = np.zeros((1, 3))
    basis = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, k, grid=spec.grid)
    ld = wl.basis.npwk_max
    npw = int(basis.npwk[0])
    assert npw == ld
    ref = H.HamiltPWRef(basis, 0, wl.veff_h, wl.vkb_h[0][:, :ld], wl.deeq_h, [8], [wl.cell.nat])
    nband = spec.nbands
    psi = wl.psi0_h[0][:nband].reshape(-1).copy()
    eig = np.zeros(nband)
    pc = H.precondition(basis, 0)
    t0 = time.time()
    if ref_david.available():
        solver = "reference DiagoDavid (compiled from its sources)"
        it = ref_david.diag(lambda x, nv, dim, i0, i1: ref.hpsi(x[i0:i1 + 1].reshape(-1), i1 - i0 + 1, ld)
                            .reshape(i1 - i0 + 1, ld), pc, nband, ld, 4, ld, psi, eig, THR, 200)
    else:
        solver = "oracle DiagoDavid restatement"
        it = DiagoDavidRef(pc, nband, ld, 4).diag(lambda x, nv: ref.hpsi(x, nv, ld), copy_spsi, ld, psi, eig, THR, 200)
    dt = time.time() - t0
    X = psi.reshape(nband, ld)
    HX = ref.hpsi(psi, nband, ld).reshape(nband, ld)
    rq = np.real(np.sum(X.conj() * HX, axis=1))
    res = np.linalg.norm(HX - rq[:, None] * X, axis=1)
    print(f"{solver}: {it} iterations in {dt:.0f} s; max |e - <x|H|x>| {np.max(np.abs(eig - rq)):.2e}; "
          f"max residual {res.max():.2e}")
    np.savez(OUT, eig=eig, iterations=it, thr=THR, solver=np.array(solver), max_residual=res.max(),
             workload=np.array(f"64-atom diamond a={spec.a} ecut {spec.ecut} Ry grid {basis.nx}^3 npw {npw} "
                               f"nbands {nband} nkb {wl.nkb}"))


if __name__ == "__main__":
    main()
