"""The NSCF driver (abacus-develop_b200/nscf.py) end to end on the 8-atom cell: V_eff through a cube file and
start vectors through a wavefunction file, the device band solve of the k-point, occupations, the band file
and the written eigenvectors, against the dense spectrum of the oracle's H."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_nscf_from_files(pkg, diamond8_dense_h, tmp_path, prec):
    wl, hm, w, _ = diamond8_dense_h
    P, io, N = pkg.pwdft, pkg.nscf_io, pkg.nscf
    b, spec = wl.basis, wl.spec
    nb = spec.nbands
    atoms = [io.CubeAtom(z=6, zv=4.0, tau=tuple(t)) for t in wl.cell.tau]
    io.write_cube(tmp_path / "SPIN1_POT.cube", wl.veff_h, b.nx, b.ny, b.nz, spec.a, wl.cell.latvec, atoms,
                  precision=16, out_fermi=0)
    veff = N.load_veff_cube(tmp_path / "SPIN1_POT.cube", b)
    assert np.allclose(veff, wl.veff_h, rtol=1e-15, atol=1e-300)
    npw = int(b.npwk[0])
    io.write_wfc_pw(str(tmp_path / "START"), b, [wl.psi0_h[0][:nb, :npw]], np.zeros((1, 3)), [2.0], spec.ecut,
                    wl.cell.latvec, fmt=2)
    start = N.read_start_wavefunctions(str(tmp_path / "START"), b, nb, 1, wl.cell.latvec)
    assert np.array_equal(start[0], wl.psi0_h[0][:nb, :npw])

    h = P.device_hamilt(dataclasses.replace(wl, veff_h=veff), P.PREC_FP64 if prec == "fp64" else P.PREC_MIXED)
    res = N.run_nscf(h, nb, start, wk=[2.0], nelec=4.0 * wl.cell.nat, latvec=wl.cell.latvec, ecutwfc=spec.ecut,
                     pw_diag_thr=1e-10, precision=P.PREC_FP64 if prec == "fp64" else P.PREC_MIXED,
                     out_dir=tmp_path / "OUT", out_wfc_pw=2)
    assert res.diag_thr == 1e-10
    assert np.max(np.abs(res.ekb[0] - w[:nb])) < 1e-8, res.ekb[0] - w[:nb]
    nocc = int(2 * wl.cell.nat)
    assert res.ef == res.ekb[0, nocc - 1] and np.all(res.wg[0, :nocc] == 2.0) and np.all(res.wg[0, nocc:] == 0.0)
    band = (tmp_path / "OUT" / "BANDS_1.dat").read_text().split("\n")
    vals = np.array(band[0].split()[2:], dtype=float)
    assert band[0].startswith("   1 0.00000000 ") and np.allclose(vals, (res.ekb[0] - res.ef) * io.RY_TO_EV, atol=1e-8)
    # the written eigenvectors read back bit for bit and diagonalise the dense H
    back = io.read_wfc_pw(res.files["wfc"][0], b, 0, 1, nb, wl.cell.latvec)
    assert np.array_equal(back, res.psis[0])
    r = back @ hm.T - res.ekb[0][:, None] * back
    assert np.max(np.linalg.norm(r, axis=1)) < 1e-3
    assert "spin1_final_band 1 " in (tmp_path / "OUT" / "running_nscf.log").read_text()
