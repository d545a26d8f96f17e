"""Eigenvalue fixture of the 216-atom cell (eig_diamond216.npz), made on the host by the oracle.

The workload is the 216-atom diamond supercell (a = 30.78 bohr, ecut 40 Ry, 128^3 grid, npw 124 289, 1728
projectors, Gamma point, 480 bands) from this package's seeded synthetic generators (V_eff, D, start
vectors), with the projectors of the oracle's getvnl restatement (oracle/vnl_ref.getvnl: the reference's
cal_ylm_real_op, polynomial interpolation of the radial tables, structure factors and (-i)^l), which the
device getvnl matches to 1e-12 on this cell.  H|psi> is the oracle's restatement of Operator::hPsi
(oracle/hamilt_ref.py: Ekinetic, Veff through the reference's stick transforms, Nonlocal).  The Davidson
iteration is the reference's own DiagoDavid<complex<double>, CPU> compiled from its sources
(oracle/_ref/libref_david.so, built by oracle/build_ref.py), driven through the oracle's H|psi>:
pw_diag_ndim 4, the reference's preconditioner, thr 1e-10, the package's start vectors.  Where that library
is absent the numpy restatement of DiagoDavid (oracle/david_ref.py, pinned to it iteration for iteration)
runs instead; the fixture records which ran.

Stored: the 480 eigenvalues (Ry), the iteration count, thr, the solver that ran, and the largest residual
norm |H x - e x| of the returned vectors (a-posteriori bound on each eigenvalue's error).

Run from the repository root:  python tests/golden/make_eig_diamond216.py   (about 30 minutes on 8 cores,
about 20 GB of host memory)
"""
from __future__ import annotations

import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import hamilt_ref as H  # noqa: E402
from oracle import ref_david  # noqa: E402
from oracle import vnl_ref as V  # noqa: E402
from oracle.david_ref import DiagoDavidRef, copy_spsi  # noqa: E402
from oracle.pw_basis_ref import PWBasisKRef  # noqa: E402
from tests.conftest import load_package  # noqa: E402

THR = 1e-10
OUT = Path(__file__).resolve().parent / "eig_diamond216.npz"
CHUNK = 24  # bands per oracle H|psi> call (a 128^3 box per band in flight)


def main():
    H.FFT_WORKERS = os.cpu_count() or 1
    pkg = load_package()
    P = pkg.pwdft
    spec = pkg.synth.config(4)
    cell = pkg.synth.make_cell(spec)
    k = np.zeros((1, 3))
    basis = P.PWBasisK(spec.a, cell.latvec, spec.ecut, k, grid=spec.grid)
    ref_b = PWBasisKRef(spec.a, cell.latvec, spec.ecut, k, grid=spec.grid)
    ld = basis.npwk_max
    npw = int(ref_b.npwk[0])
    assert npw == ld
    proj = cell.projector_tables(basis.omega, spec.ecut)
    vkb = V.getvnl(ref_b, 0, proj, cell.tau / spec.a)
    ref = H.HamiltPWRef(ref_b, 0, cell.veff(basis.nx, basis.ny, basis.nz), vkb, cell.deeq(), [8], [cell.nat])
    nband = spec.nbands
    psi = cell.psi0(basis.gplusk_cart(0), nband, ld).reshape(-1).copy()
    eig = np.zeros(nband)
    pc = H.precondition(ref_b, 0)
    calls = [0, 0, time.time()]

    def hpsi_rows(x, nv):
        """H applied to the nv vectors of x (nv x ld), CHUNK bands per oracle call."""
        x = np.asarray(x).reshape(nv, ld)
        out = np.empty((nv, ld), dtype=np.complex128)
        for b0 in range(0, nv, CHUNK):
            b1 = min(nv, b0 + CHUNK)
            out[b0:b1] = ref.hpsi(x[b0:b1].reshape(-1), b1 - b0, ld).reshape(b1 - b0, ld)
        calls[0] += 1
        calls[1] += nv
        print(f"H|psi> call {calls[0]}: {nv} bands ({calls[1]} in all), {time.time() - calls[2]:.0f} s", flush=True)
        return out

    t0 = time.time()
    if ref_david.available():
        solver = "reference DiagoDavid (compiled from its sources)"
        it = ref_david.diag(lambda x, nv, dim, i0, i1: hpsi_rows(x[i0:i1 + 1], i1 - i0 + 1), pc, nband, ld, 4, ld,
                            psi, eig, THR, 200)
    else:
        solver = "oracle DiagoDavid restatement"
        it = DiagoDavidRef(pc, nband, ld, 4).diag(lambda x, nv: hpsi_rows(x, nv).reshape(-1), copy_spsi, ld, psi, eig,
                                                  THR, 200)
    dt = time.time() - t0
    X = psi.reshape(nband, ld)
    HX = hpsi_rows(X, nband)
    rq = np.real(np.sum(X.conj() * HX, axis=1))
    res = np.linalg.norm(HX - rq[:, None] * X, axis=1)
    print(f"{solver}: {it} iterations in {dt:.0f} s; max |e - <x|H|x>| {np.max(np.abs(eig - rq)):.2e}; "
          f"max residual {res.max():.2e}")
    np.savez(OUT, eig=eig, iterations=it, thr=THR, solver=np.array(solver), max_residual=res.max(),
             workload=np.array(f"216-atom diamond a={spec.a} ecut {spec.ecut} Ry grid {basis.nx}^3 npw {npw} "
                               f"nbands {nband} nkb {proj.nkb} (oracle getvnl)"))


if __name__ == "__main__":
    main()
