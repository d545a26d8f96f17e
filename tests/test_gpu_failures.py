"""Failure detection on the GPU, with the failures made on the host (no fault, trap or hang of the GPU).

* NaN / Inf in the start vectors, in V_eff or in D: the device Davidson (FP64 and mixed) stops with
  B200_STATUS_NUMERICAL_ERROR instead of returning NaN eigenvalues; the subspace eigensolver is never
  given a non-finite matrix; the same handles solve correctly once the inputs are repaired.
* The serving loop: a resident cell whose V_eff holds a NaN reports that status per request, and the
  requests on the other cells are served correctly meanwhile (the server keeps running).

The reference has no counterpart: its Davidson goes on with NaN and SchmidtOrth calls exit(0) on a
breakdown (diago_david.cpp:1055-1060)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

NUMERICAL_ERROR = 5


@pytest.fixture(scope="module")
def cell8(pkg):
    P = pkg.pwdft
    spec = pkg.synth.config(0)
    wl = P.build_workload(spec)
    return P, wl


def _solve(P, h, wl, prec, psi0=None, nb=16):
    ld = wl.basis.npwk_max
    pc = P.precondition_d(wl.basis, 0)
    dav = P.DiagoDavid(pc, nb, ld, 4, prec)
    x0 = wl.psi0_h[0][:nb].reshape(-1).copy() if psi0 is None else psi0
    x = torch.from_numpy(x0).to("cuda:0")
    e = np.zeros(nb)
    dav.diag_hamilt(h, 0, ld, x, e, 1e-9, 80)
    return e


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_nan_in_start_vectors(pkg, cell8, prec):
    P, wl = cell8
    p = P.PREC_FP64 if prec == "fp64" else P.PREC_MIXED
    h = P.device_hamilt(wl, p)
    good = _solve(P, h, wl, p)
    bad = wl.psi0_h[0][:16].reshape(-1).copy()
    bad[123] = np.nan
    with pytest.raises(pkg._lib.B200Error) as ei:
        _solve(P, h, wl, p, psi0=bad)
    assert ei.value.code == NUMERICAL_ERROR
    np.testing.assert_allclose(_solve(P, h, wl, p), good, atol=1e-8)


@pytest.mark.parametrize("what", ["veff_inf", "deeq_nan"])
def test_non_finite_potential_or_d(pkg, cell8, what):
    P, wl = cell8
    h = P.device_hamilt(wl, P.PREC_FP64)
    good = _solve(P, h, wl, P.PREC_FP64)
    if what == "veff_inf":
        v = np.array(wl.veff_h, copy=True)
        v.reshape(-1)[777] = np.inf
        vd = torch.from_numpy(v).cuda()
        h.set_veff(vd)
    else:
        d = np.array(wl.deeq_h, copy=True)
        d.reshape(-1)[3] = np.nan
        dd = torch.from_numpy(d).cuda()
        h.set_deeq([wl.cell.nat], [pkg.synth.NH], dd)
    with pytest.raises(pkg._lib.B200Error) as ei:
        _solve(P, h, wl, P.PREC_FP64)
    assert ei.value.code == NUMERICAL_ERROR
    # repaired inputs: the same handle solves as before
    fixed = torch.from_numpy(np.array(wl.veff_h if what == "veff_inf" else wl.deeq_h, copy=True)).cuda()
    if what == "veff_inf":
        h.set_veff(fixed)
    else:
        h.set_deeq([wl.cell.nat], [pkg.synth.NH], fixed)
    torch.cuda.synchronize()
    np.testing.assert_allclose(_solve(P, h, wl, P.PREC_FP64), good, atol=1e-8)


def test_server_reports_bad_cell_and_keeps_serving(pkg):
    S = pkg.serve
    spec = pkg.synth.serving_cells()[0]  # 2-atom cell
    good_cell, bad_cell = S.build_serving_cells([spec, spec], npath=2)
    v = np.array(bad_cell.cell.veff(bad_cell.basis.nx, bad_cell.basis.ny, bad_cell.basis.nz), copy=True)
    v.reshape(-1)[5] = np.nan
    vd = torch.from_numpy(v).cuda()
    bad_cell.hamilt.set_veff(vd)
    torch.cuda.synchronize()
    srv = S.Server(hbm_budget_bytes=2 << 30, nworkers=2)
    try:
        gid = srv.add_cell(good_cell.hamilt)
        bid = srv.add_cell(bad_cell.hamilt)
        for prec in (S.PREC_MIXED, S.PREC_FP64):
            for i in range(4):
                srv.submit(bid if i % 2 else gid, i % 2, spec.nbands, thr=1e-9, precision=prec, tag=("r", prec, i))
        res = srv.drain()
        assert len(res) == 8
        for r in res:
            expect = NUMERICAL_ERROR if r.tag[2] % 2 else 0
            assert r.status == expect, (r.tag, r.status)
        # the good cell after the failures: same eigenvalues as alone in a fresh server
        srv.submit(gid, 1, spec.nbands, thr=1e-9, precision=S.PREC_FP64, tag="after")
        after = srv.drain()
        assert after[0].status == 0
        ref = S.Server(hbm_budget_bytes=1 << 30, nworkers=1)
        try:
            rid = ref.add_cell(good_cell.hamilt)
            ref.submit(rid, 1, spec.nbands, thr=1e-9, precision=S.PREC_FP64)
            alone = ref.drain()
        finally:
            ref.close()
        assert np.max(np.abs(after[0].eig - alone[0].eig)) <= 1e-10
    finally:
        srv.close()
