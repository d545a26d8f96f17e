"""Serving loop on the GPU: continuous admission, results independent of the mix, and parity of a served
result with the oracle.

Cells: the 2-atom (a = 5.13 bohr, ecut 30 Ry, 8 bands) and 8-atom (a = 10.26, ecut 30, 32 bands) cells
of the serving workload, each with a 4-point high-symmetry path whose projectors are built on the device.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import hamilt_ref as H
from oracle.pw_basis_ref import PWBasisKRef

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def served(pkg):
    S = pkg.serve
    specs = pkg.synth.serving_cells()[:2]
    cells = S.build_serving_cells(specs, npath=4)
    srv = S.Server(hbm_budget_bytes=8 << 30, nworkers=4)
    ids = [srv.add_cell(c.hamilt) for c in cells]
    yield S, srv, cells, ids
    srv.close()


def test_result_same_alone_and_in_the_mix(served):
    """A request gives the same eigenvalues alone and among others in flight (tolerance 1e-10 Ry, ten
    times below the solve threshold; pooled solvers start from a zeroed subspace, so it is bitwise)."""
    S, srv, cells, ids = served
    probe = (ids[1], 2, cells[1].nbands)
    srv.submit(*probe, thr=1e-9)
    alone = srv.drain()
    assert len(alone) == 1 and alone[0].status == 0
    for i in range(12):
        c = i % 2
        srv.submit(ids[c], i % 4, cells[c].nbands, thr=1e-9, tag=("other", i))
    srv.submit(*probe, thr=1e-9, tag="probe")
    for i in range(6):
        srv.submit(ids[i % 2], (i + 1) % 4, cells[i % 2].nbands, thr=1e-9, tag=("other2", i))
    mix = srv.drain()
    assert all(r.status == 0 for r in mix)
    got = [r for r in mix if r.tag == "probe"][0]
    assert np.max(np.abs(got.eig - alone[0].eig)) <= 1e-10
    st = srv.stats()
    assert st["peak_in_flight"] >= 2  # requests really overlapped
    assert st["peak_pool_bytes"] <= 8 << 30


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_served_eigenvalues_match_oracle(served, prec):
    """The 2-atom cell at a path k-point: served eigenvalues within 1e-8 Ry of the oracle's dense spectrum
    of the same Hamiltonian (V_eff, D and the device-built projectors)."""
    S, srv, cells, ids = served
    c = cells[0]
    ik = 1
    p = S.PREC_MIXED if prec == "mixed" else S.PREC_FP64
    srv.submit(ids[0], ik, c.nbands, thr=1e-11, precision=p)
    r = srv.drain()[0]
    assert r.status == 0
    npwx = c.basis.npwk_max
    vkb = torch.zeros(c.cell.nkb * npwx, dtype=torch.complex128, device="cuda")
    c.hamilt.copy_vkb(ik, vkb)
    torch.cuda.synchronize()
    ref_b = PWBasisKRef(c.spec.a, c.cell.latvec, c.spec.ecut, c.kpath[ik:ik + 1], grid=c.spec.grid)
    npw = int(ref_b.npwk[0])
    veff = c.cell.veff(c.basis.nx, c.basis.ny, c.basis.nz)
    ref = H.HamiltPWRef(ref_b, 0, veff, vkb.cpu().numpy().reshape(c.cell.nkb, npwx)[:, :npw], c.cell.deeq(), [8],
                        [c.cell.nat])
    e_exact = np.linalg.eigvalsh(ref.dense())[:c.nbands]
    assert np.max(np.abs(r.eig - e_exact)) < 1e-8, r.eig - e_exact


def test_budget_too_small_is_rejected(served):
    S, _, cells, _ = served
    tiny = S.Server(hbm_budget_bytes=1 << 20, nworkers=1)
    cid = tiny.add_cell(cells[1].hamilt)
    tiny.submit(cid, 0, cells[1].nbands)
    r = tiny.drain()
    assert len(r) == 1 and r[0].status == 6  # B200_STATUS_CAPACITY_ERROR
    tiny.close()


def test_admission_policy_and_shedding(served):
    """The response-ratio policy serves every request of a burst with the same eigenvalues as first come, first
    served; with shedding on, requests that waited past the bound come back as STATUS_SHED, the others are
    served correctly and the server keeps serving afterwards; with express workers (reserved for cells of
    short service) every request is still served, with the results it has alone."""
    S, srv, cells, ids = served
    c = 1
    probe = (ids[c], 2, cells[c].nbands)
    srv.set_policy(0, 0.0)
    srv.submit(*probe, thr=1e-9)
    ref = srv.drain()[0]
    assert ref.status == 0
    try:
        srv.set_policy(1, 0.0)
        for i in range(10):
            srv.submit(ids[i % 2], i % 4, cells[i % 2].nbands, thr=1e-9, tag=("rr", i))
        srv.submit(*probe, thr=1e-9, tag="probe")
        res = srv.drain()
        assert len(res) == 11 and all(r.status == 0 for r in res)
        got = [r for r in res if r.tag == "probe"][0]
        assert np.max(np.abs(got.eig - ref.eig)) <= 1e-10
        # a bound of 1 % of the mean service time: a burst larger than the workers' slots must shed some
        srv.set_policy(1, 0.01)
        for i in range(24):
            srv.submit(ids[c], i % 4, cells[c].nbands, thr=1e-9, tag=("shed", i))
        res = srv.drain()
        assert len(res) == 24
        st = [r.status for r in res]
        assert S.STATUS_SHED in st and 0 in st
        assert set(st) <= {0, S.STATUS_SHED}
        for r in res:
            if r.status == 0 and r.tag[1] % 4 == 2:
                assert np.max(np.abs(r.eig - ref.eig)) <= 1e-10
        # express workers: one that takes no timed cell (bound 1 ns), then two that take every cell; every
        # request is served with the results it has alone
        srv.set_policy(1, 0.0)
        for nexp, bound in ((1, 1e-9), (2, 10.0)):
            srv.set_express(nexp, bound)
            for i in range(8):
                srv.submit(ids[i % 2], i % 4, cells[i % 2].nbands, thr=1e-9, tag=("x", i))
            srv.submit(*probe, thr=1e-9, tag="probe")
            res = srv.drain()
            assert len(res) == 9 and all(r.status == 0 for r in res)
            got = [r for r in res if r.tag == "probe"][0]
            assert np.max(np.abs(got.eig - ref.eig)) <= 1e-10
    finally:
        srv.set_express(0, 0.0)
        srv.set_policy(0, 0.0)
    srv.submit(*probe, thr=1e-9)
    after = srv.drain()
    assert after[0].status == 0 and np.max(np.abs(after[0].eig - ref.eig)) <= 1e-10
