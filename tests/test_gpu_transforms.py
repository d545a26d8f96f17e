"""GPU parity of the G-sphere <-> r-box transforms (PW_Basis_K::recip_to_real /
real_to_recip on the device) against the oracle (numpy's FFT with ABACUS's
sign and normalisation), at the grid sizes of the workloads.

Tolerances: FP64 1e-12 relative to the largest entry; FP32 2e-6 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import hamilt_ref as H
from oracle.pw_basis_ref import PWBasisKRef

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = {
    "18^3": (5.13, np.eye(3), 30.0, np.zeros((1, 3)), None),
    "36^3_k": (10.26, np.eye(3), 30.0, np.array([[0.125, -0.375, 0.375]]), None),
    "45x45x90": (10.26, np.diag([1.0, 1.0, 2.0]), 40.0, np.zeros((1, 3)), None),
    "96^3": (20.52, np.eye(3), 50.0, np.zeros((1, 3)), None),
    "40^3_explicit": (10.26, np.eye(3), 30.0, np.zeros((1, 3)), (40, 40, 40)),
}


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("name", list(CASES))
def test_transforms_fp64(pkg, name):
    lat0, lv, ec, kd, grid = CASES[name]
    ref = PWBasisKRef(lat0, lv, ec, kd, grid=grid)
    b = pkg.pwdft.PWBasisK(lat0, lv, ec, kd, grid=grid)
    rng = np.random.default_rng(11)
    npw = int(ref.npwk[0])
    N = ref.nxyz
    c = rng.standard_normal(npw) + 1j * rng.standard_normal(npw)
    r_ref = H.recip_to_real(ref, c, 0)
    out = torch.zeros(N, dtype=torch.complex128, device="cuda")
    b.recip_to_real(torch.from_numpy(c).cuda(), out, 0)
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), r_ref) < 1e-12
    # add mode: out += factor * r
    base = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    out = torch.from_numpy(base.copy()).cuda()
    b.recip_to_real(torch.from_numpy(c).cuda(), out, 0, add=True, factor=0.7)
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), base + 0.7 * r_ref) < 1e-12
    # real_to_recip of a random box
    box = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    g_ref = H.real_to_recip(ref, box, 0)
    g = torch.zeros(npw, dtype=torch.complex128, device="cuda")
    b.real_to_recip(torch.from_numpy(box).cuda(), g, 0)
    torch.cuda.synchronize()
    assert rel(g.cpu().numpy(), g_ref) < 1e-12
    acc0 = rng.standard_normal(npw) + 1j * rng.standard_normal(npw)
    g = torch.from_numpy(acc0.copy()).cuda()
    b.real_to_recip(torch.from_numpy(box).cuda(), g, 0, add=True, factor=2.5)
    torch.cuda.synchronize()
    gr = acc0.copy()
    H.real_to_recip(ref, box, 0, out=gr, add=True, factor=2.5)
    assert rel(g.cpu().numpy(), gr) < 1e-12
    # round trip is the identity on the sphere
    rr = torch.zeros(N, dtype=torch.complex128, device="cuda")
    b.recip_to_real(torch.from_numpy(c).cuda(), rr, 0)
    back = torch.zeros(npw, dtype=torch.complex128, device="cuda")
    b.real_to_recip(rr, back, 0)
    torch.cuda.synchronize()
    assert rel(back.cpu().numpy(), c) < 1e-13


@pytest.mark.parametrize("name", ["36^3_k", "96^3"])
def test_transforms_fp32(pkg, name):
    lat0, lv, ec, kd, grid = CASES[name]
    ref = PWBasisKRef(lat0, lv, ec, kd, grid=grid)
    b = pkg.pwdft.PWBasisK(lat0, lv, ec, kd, grid=grid)
    rng = np.random.default_rng(12)
    npw = int(ref.npwk[0])
    N = ref.nxyz
    c = (rng.standard_normal(npw) + 1j * rng.standard_normal(npw)).astype(np.complex64)
    r_ref = H.recip_to_real(ref, c.astype(np.complex128), 0)
    out = torch.zeros(N, dtype=torch.complex64, device="cuda")
    b.recip_to_real(torch.from_numpy(c).cuda(), out, 0)
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy().astype(np.complex128), r_ref) < 2e-6
    g = torch.zeros(npw, dtype=torch.complex64, device="cuda")
    b.real_to_recip(out, g, 0)
    torch.cuda.synchronize()
    assert rel(g.cpu().numpy().astype(np.complex128), c.astype(np.complex128)) < 2e-6
