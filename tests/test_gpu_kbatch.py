"""k-point batches on the GPU: batched H|psi>, its CUDA-graph replay, the band-chunk autotuner and
concurrent Davidson solves, each against the per-k-point path (itself checked against the oracle).

Workload: the 8-atom diamond cell with a shifted 4x4x4 Monkhorst-Pack grid (36^3 FFT box, npwk
between about 2900 and 2960 per k-point, 32 bands).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from oracle import hamilt_ref as H
from oracle.pw_basis_ref import PWBasisKRef

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def mp444(pkg):
    spec = pkg.synth.config(2)
    kpts = spec.kpts[:8]
    return spec, pkg.pwdft.build_workload(spec, kpts=kpts)


def _psis(wl, nb, dtype):
    return [torch.from_numpy(wl.psi0_h[ik][:nb].reshape(-1).astype(dtype)).cuda() for ik in range(wl.basis.nks)]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_hpsi_kbatch_equals_per_k(pkg, mp444, prec):
    spec, wl = mp444
    P = pkg.pwdft
    p = P.PREC_FP64 if prec == "fp64" else P.PREC_MIXED
    dt = np.complex128 if prec == "fp64" else np.complex64
    h = P.device_hamilt(wl, p)
    nb, ld = 32, wl.basis.npwk_max
    iks = list(range(wl.basis.nks))
    psis = _psis(wl, nb, dt)
    outs = [torch.full_like(x, complex(5.0, 1.0)) for x in psis]
    h.hpsi_kbatch(iks, psis, outs, nb, ld)
    torch.cuda.synchronize()
    for ik in iks:
        one = torch.zeros_like(psis[ik])
        h.hpsi(ik, psis[ik], one, nb, ld)
        torch.cuda.synchronize()
        # the batched passes run the same arithmetic per band: identical up to FP32 rounding order
        tol = 1e-14 if prec == "fp64" else 1e-6
        assert rel(outs[ik].cpu().numpy(), one.cpu().numpy()) < tol, ik
    # two k-points against the oracle
    for ik in (0, 5):
        k = spec.kpts[ik:ik + 1]
        ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, k, grid=spec.grid)
        ref = H.HamiltPWRef(ref_b, 0, wl.veff_h, wl.vkb_h[ik][:, :ref_b.npwk_max], wl.deeq_h, [8], [wl.cell.nat])
        npw = ref_b.npwk[0]
        psi = wl.psi0_h[ik][:nb, :npw].reshape(-1)
        href = ref.hpsi(psi, nb, npw).reshape(nb, npw)
        got = outs[ik].cpu().numpy().reshape(nb, ld)[:, :npw].astype(np.complex128)
        assert rel(got, href) < (1e-12 if prec == "fp64" else 2e-5), ik


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_hpsi_kbatch_register_transforms(pkg, prec):
    """A 96^3 grid takes the register/shuffle transforms in both the batched and the per-k-point calls;
    they give the same H|psi>, and one k-point agrees with the oracle."""
    spec = dataclasses.replace(pkg.synth.config(0), grid=(96, 96, 96))
    kpts = pkg.synth.mp_grid(2, True)[:3]
    P = pkg.pwdft
    wl = P.build_workload(spec, kpts=kpts)
    p = P.PREC_FP64 if prec == "fp64" else P.PREC_MIXED
    dt = np.complex128 if prec == "fp64" else np.complex64
    h = P.device_hamilt(wl, p)
    nb, ld = 5, wl.basis.npwk_max
    psis = _psis(wl, nb, dt)
    outs = [torch.zeros_like(x) for x in psis]
    h.hpsi_kbatch([0, 1, 2], psis, outs, nb, ld)
    for ik in range(3):
        one = torch.zeros_like(psis[ik])
        h.hpsi(ik, psis[ik], one, nb, ld)
        torch.cuda.synchronize()
        assert rel(outs[ik].cpu().numpy(), one.cpu().numpy()) < (1e-14 if prec == "fp64" else 1e-6)
    ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, kpts[1:2], grid=spec.grid)
    ref = H.HamiltPWRef(ref_b, 0, wl.veff_h, wl.vkb_h[1][:, :ref_b.npwk_max], wl.deeq_h, [8], [wl.cell.nat])
    npw = ref_b.npwk[0]
    href = ref.hpsi(wl.psi0_h[1][:nb, :npw].reshape(-1), nb, npw).reshape(nb, npw)
    got = outs[1].cpu().numpy().reshape(nb, ld)[:, :npw].astype(np.complex128)
    assert rel(got, href) < (1e-12 if prec == "fp64" else 2e-5)


def test_hpsi_kbatch_generic_grid_falls_back(pkg):
    """A grid outside the compiled warp-transform sizes takes the per-k path inside the batch call."""
    spec = dataclasses.replace(pkg.synth.config(0), grid=(40, 40, 40))
    kpts = pkg.synth.mp_grid(2, True)[:3]
    P = pkg.pwdft
    wl = P.build_workload(spec, kpts=kpts)
    h = P.device_hamilt(wl, P.PREC_FP64)
    nb, ld = 6, wl.basis.npwk_max
    psis = _psis(wl, nb, np.complex128)
    outs = [torch.zeros_like(x) for x in psis]
    h.hpsi_kbatch([0, 1, 2], psis, outs, nb, ld)
    for ik in range(3):
        one = torch.zeros_like(psis[ik])
        h.hpsi(ik, psis[ik], one, nb, ld)
        torch.cuda.synchronize()
        assert rel(outs[ik].cpu().numpy(), one.cpu().numpy()) < 1e-14


def test_graph_replay_equals_direct(pkg, mp444):
    spec, wl = mp444
    P = pkg.pwdft
    h = P.device_hamilt(wl, P.PREC_FP64)
    nb, ld = 16, wl.basis.npwk_max
    iks = [1, 2, 3, 6]
    psis = [_psis(wl, nb, np.complex128)[ik] for ik in iks]
    outs = [torch.zeros_like(x) for x in psis]
    s = torch.cuda.Stream()
    g = h.capture_hpsi_kbatch(iks, psis, outs, nb, ld, stream=s)
    # new input in the captured buffers, replay, compare with a direct call on the same input
    rng = np.random.default_rng(3)
    for x in psis:
        v = rng.standard_normal(x.numel()) + 1j * rng.standard_normal(x.numel())
        x.copy_(torch.from_numpy(v))
    torch.cuda.synchronize()
    g.launch(s)
    s.synchronize()
    for q, ik in enumerate(iks):
        one = torch.zeros_like(psis[q])
        h.hpsi(ik, psis[q], one, nb, ld)
        torch.cuda.synchronize()
        # replayed results use the new input; the padding of psi is not zero, H|psi> ignores it
        assert rel(outs[q].cpu().numpy(), one.cpu().numpy()) < 1e-14, ik
    del g


def test_autotune_keeps_result(pkg, mp444):
    spec, wl = mp444
    P = pkg.pwdft
    h = P.device_hamilt(wl, P.PREC_FP64)
    nb, ld = 32, wl.basis.npwk_max
    psi = _psis(wl, nb, np.complex128)[0]
    before = torch.zeros_like(psi)
    h.hpsi(0, psi, before, nb, ld)
    scratch = torch.zeros_like(psi)
    best = h.autotune(0, psi, scratch, nb, ld)
    assert best in (1, 2, 4, 8, 16, 32)
    after = torch.zeros_like(psi)
    h.hpsi(0, psi, after, nb, ld)
    torch.cuda.synchronize()
    assert rel(after.cpu().numpy(), before.cpu().numpy()) < 1e-14


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_concurrent_solves_equal_alone(pkg, mp444, prec):
    """Each k-point's eigenvalues from the concurrent solve equal its solve alone."""
    spec, wl = mp444
    P = pkg.pwdft
    p = P.PREC_FP64 if prec == "fp64" else P.PREC_MIXED
    h = P.device_hamilt(wl, P.PREC_FP64)
    nband, ld = 32, wl.basis.npwk_max
    iks = [0, 1, 2, 3, 4, 5]
    pcs = [P.precondition_d(wl.basis, ik) for ik in iks]
    psis = [torch.from_numpy(wl.psi0_h[ik].reshape(-1).copy()).cuda() for ik in iks]
    eig, its = h.solve_kpoints(iks, pcs, psis, ld, nband, 1e-10, 100, precision=p, nworkers=3)
    for q, ik in enumerate(iks):
        npw = int(wl.basis.npwk[ik])
        dav = P.DiagoDavid(pcs[q], nband, npw, 4, p)
        psi = torch.from_numpy(wl.psi0_h[ik].reshape(-1).copy()).cuda()
        e = np.zeros(nband)
        it = dav.diag_hamilt(h, ik, ld, psi, e, 1e-10, 100)
        assert np.max(np.abs(eig[q] - e)) < 1e-10, (ik, eig[q] - e)
        assert its[q] == it
        # eigenvectors: residual |H psi - e psi| small
        hp = torch.zeros_like(psis[q])
        h.hpsi(ik, psis[q], hp, nband, ld)
        torch.cuda.synchronize()
        X = psis[q].cpu().numpy().reshape(nband, ld)
        HX = hp.cpu().numpy().reshape(nband, ld)
        assert np.max(np.linalg.norm(HX - eig[q][:, None] * X, axis=1)) < 1e-3


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batched_solve_equals_per_k_and_oracle(pkg, mp444, prec):
    """The lock-step batched Davidson of 8 k-points (uneven npw), FP64 and mixed (FP32 stage + FP64 refinement),
    gives each k-point's eigenvalues of its own FP64 solve within 1e-8 Ry, and, at two k-points, the dense
    spectrum of the oracle's Hamiltonian within 1e-8 Ry; the returned vectors are orthonormal eigenvectors (small
    residuals)."""
    spec, wl = mp444
    P = pkg.pwdft
    h = P.device_hamilt(wl, P.PREC_FP64)
    nband, ld = 32, wl.basis.npwk_max
    iks = list(range(wl.basis.nks))
    pcs = [P.precondition_d(wl.basis, ik) for ik in iks]
    psis = [torch.from_numpy(wl.psi0_h[ik].reshape(-1).copy()).cuda() for ik in iks]
    p = P.PREC_FP64 if prec == "fp64" else P.PREC_MIXED
    eig, its = h.solve_kpoints_batched(iks, pcs, psis, ld, nband, 1e-10, 200, precision=p)
    assert np.all(its > 0)
    for q, ik in enumerate(iks):
        npw = int(wl.basis.npwk[ik])
        dav = P.DiagoDavid(pcs[q], nband, npw, 4, P.PREC_FP64)
        psi = torch.from_numpy(wl.psi0_h[ik].reshape(-1).copy()).cuda()
        e = np.zeros(nband)
        dav.diag_hamilt(h, ik, ld, psi, e, 1e-10, 200)
        assert np.max(np.abs(eig[q] - e)) < 1e-8, (ik, np.max(np.abs(eig[q] - e)))
        hp = torch.zeros_like(psis[q])
        h.hpsi(ik, psis[q], hp, nband, ld)
        torch.cuda.synchronize()
        X = psis[q].cpu().numpy().reshape(nband, ld)
        HX = hp.cpu().numpy().reshape(nband, ld)
        if npw < ld:
            assert np.max(np.abs(X[:, npw:])) == 0.0
        assert np.max(np.abs(X.conj() @ X.T - np.eye(nband))) < 1e-10
        assert np.max(np.linalg.norm(HX - eig[q][:, None] * X, axis=1)) < 1e-3
    for ik in (0, 5):
        k = spec.kpts[ik:ik + 1]
        ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, k, grid=spec.grid)
        ref = H.HamiltPWRef(ref_b, 0, wl.veff_h, wl.vkb_h[ik][:, :ref_b.npwk_max], wl.deeq_h, [8], [wl.cell.nat])
        dense = np.linalg.eigvalsh(ref.dense())[:nband]
        assert np.max(np.abs(eig[ik] - dense)) < 1e-8, ik
