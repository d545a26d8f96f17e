"""H|psi> with npol = 2 (non-collinear spinors) against the oracle.

The oracle chain (oracle/hamilt_ref.py HamiltPWRefNC) composes the reference's spinor branches from the
oracle's functors: Ekinetic on every column, Veff::act's npol = 2 branch (veff_pw_op's 2x2 form), Nonlocal::act
with the deeq_nc overload of nonlocal_pw_op.  FP64 must match within 1e-12 relative, mixed within 2e-5.
A CPU check pins the oracle itself: with the magnetic components zero and deeq_nc = (D, 0, 0, D) the
spinor chain is the collinear chain on each component.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from oracle import hamilt_ref as H
from oracle.pw_basis_ref import PWBasisKRef


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def _nc_inputs(wl, magnetic=True, seed=5):
    """V_eff's four components and deeq_nc(4, dx, dy, dz) built from the workload's collinear ones."""
    rng = np.random.default_rng(seed)
    v0 = np.asarray(wl.veff_h, dtype=np.float64)
    scale = 0.05 * np.max(np.abs(v0)) if magnetic else 0.0
    v4 = [v0] + [scale * rng.standard_normal(v0.shape) for _ in range(3)]
    d = np.asarray(wl.deeq_h)[0]  # (dx, dy, dz) real, D(iat, ip, ip2) of the collinear form
    dt = np.transpose(d, (0, 2, 1)).astype(np.complex128)  # the spinor form indexes D(iat, kk, xx)
    dnc = np.zeros((4,) + d.shape, dtype=np.complex128)
    dnc[0] = dt
    if magnetic:
        off = 0.1 * np.max(np.abs(d)) * (rng.standard_normal(d.shape) + 1j * rng.standard_normal(d.shape))
        dnc[3] = 0.8 * dt
        dnc[1] = off
        dnc[2] = np.conj(np.transpose(off, (0, 2, 1)))
    else:
        dnc[3] = dt
    return v4, dnc


def _setup(pkg, spec, kpt, nb):
    P = pkg.pwdft
    k = np.zeros((1, 3)) if kpt is None else np.atleast_2d(kpt)
    wl = P.build_workload(spec, kpts=k)
    ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, k, grid=spec.grid)
    ld = wl.basis.npwk_max
    psi = np.asarray(wl.psi0_h[0][:2 * nb]).reshape(-1)  # 2 nb spinor columns
    return wl, ref_b, psi, ld


def test_oracle_nc_reduces_to_collinear(pkg):
    spec = pkg.synth.config(0)
    wl, ref_b, psi, ld = _setup(pkg, spec, None, 3)
    vkb = wl.vkb_h[0][:, :ld]
    v4, dnc = _nc_inputs(wl, magnetic=False)
    nc = H.HamiltPWRefNC(ref_b, 0, v4, vkb, dnc, [8], [wl.cell.nat]).hpsi(psi, 3, ld)
    col = H.HamiltPWRef(ref_b, 0, wl.veff_h, vkb, wl.deeq_h, [8], [wl.cell.nat]).hpsi(psi, 6, ld)
    assert rel(nc, col) < 1e-13


def _device_nc(pkg, wl, prec, v4, dnc):
    import torch
    P = pkg.pwdft
    h = P.device_hamilt(wl, prec)
    h.set_veff_nc(torch.from_numpy(np.stack(v4)).cuda())
    h.set_deeq_nc([wl.cell.nat], [8], torch.from_numpy(dnc).cuda())
    return h


@pytest.mark.gpu
@pytest.mark.parametrize("gemm", [0, 2])
@pytest.mark.parametrize("cfg", ["diamond8", "diamond8_k", "diamond8_grid96"])
def test_hpsi_nc_fp64_matches_oracle(pkg, cfg, gemm):
    torch = pytest.importorskip("torch")
    spec, kpt, nb = pkg.synth.config(0), None, 6
    if cfg == "diamond8_k":
        kpt = np.array([0.125, -0.375, 0.375])
    elif cfg == "diamond8_grid96":
        spec, nb = dataclasses.replace(spec, grid=(96, 96, 96)), 3
    wl, ref_b, psi, ld = _setup(pkg, spec, kpt, nb)
    v4, dnc = _nc_inputs(wl)
    href = H.HamiltPWRefNC(ref_b, 0, v4, wl.vkb_h[0][:, :ld], dnc, [8], [wl.cell.nat]).hpsi(psi, nb, ld)
    h = _device_nc(pkg, wl, pkg.pwdft.PREC_FP64, v4, dnc)
    h.set_fp64_gemm(gemm)
    pd = torch.from_numpy(psi).cuda()
    hd = torch.full_like(pd, complex(7.0, -3.0))  # garbage: overwritten, padding included
    h.hpsi_nc(0, pd, hd, nb, ld)
    torch.cuda.synchronize()
    assert rel(hd.cpu().numpy(), href) < 1e-12


@pytest.mark.gpu
def test_hpsi_nc_mixed_matches_oracle(pkg):
    torch = pytest.importorskip("torch")
    spec, nb = pkg.synth.config(0), 6
    wl, ref_b, psi, ld = _setup(pkg, spec, None, nb)
    v4, dnc = _nc_inputs(wl)
    href = H.HamiltPWRefNC(ref_b, 0, v4, wl.vkb_h[0][:, :ld], dnc, [8], [wl.cell.nat]).hpsi(psi, nb, ld)
    h = _device_nc(pkg, wl, pkg.pwdft.PREC_MIXED, v4, dnc)
    pd = torch.from_numpy(psi.astype(np.complex64)).cuda()
    hd = torch.zeros_like(pd)
    h.hpsi_nc(0, pd, hd, nb, ld)
    torch.cuda.synchronize()
    assert rel(hd.cpu().numpy().astype(np.complex128), href) < 2e-5


@pytest.mark.gpu
def test_hpsi_nc_without_magnetism_is_collinear_per_component(pkg):
    """V1 = V2 = V3 = 0 and deeq_nc = (D, 0, 0, D): the spinor H|psi> is the collinear one on each component."""
    torch = pytest.importorskip("torch")
    spec, nb = pkg.synth.config(0), 6
    wl, ref_b, psi, ld = _setup(pkg, spec, None, nb)
    v4, dnc = _nc_inputs(wl, magnetic=False)
    h = _device_nc(pkg, wl, pkg.pwdft.PREC_FP64, v4, dnc)
    pd = torch.from_numpy(psi).cuda()
    hnc = torch.zeros_like(pd)
    hcol = torch.zeros_like(pd)
    h.hpsi_nc(0, pd, hnc, nb, ld)
    h.hpsi(0, pd, hcol, 2 * nb, ld)
    torch.cuda.synchronize()
    assert rel(hnc.cpu().numpy(), hcol.cpu().numpy()) < 1e-13
