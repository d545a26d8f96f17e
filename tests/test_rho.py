"""psi -> rho: the oracle against the reference's literals (elecstate_op_test.cpp) on the CPU; the device
functors and the device psiToRho band loop against the oracle, and the sum rule at a full-size grid, on the GPU.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import rho_ref as R


def test_oracle_elecstate_matches_golden(golden):
    d = golden("elecstate_op")
    n = int(d["nrxx"])
    rho = [np.zeros(n)]
    R.elecstate_pw_op(int(d["spin"]), n, float(d["w1"]), rho, d["wfcr"])
    assert np.max(np.abs(rho[0] - d["expected_rho"])) < 6e-5  # literals carry 6 digits; the reference's bound
    assert np.max(np.abs(rho[0] - d["expected_rho"]) / np.abs(d["expected_rho"])) < 1e-5
    # the nspin = 4 case: the reference's test calls the functor with w1 and bounds the error by 5e-4 absolute,
    # which its values (about 1e-4) always meet; its literals are the functor's output for w2 = w1/2, to
    # their 6 printed digits.  Both checks:
    rho4 = [np.zeros(n) for _ in range(4)]
    R.elecstate_pw_op_nc(int(d["DOMAG"]), int(d["DOMAG_Z"]), n, float(d["w1"]), rho4, d["wfcr_2"],
                         d["wfcr_another_spin_2"])
    assert np.max(np.abs(np.concatenate(rho4) - d["expected_rho_2"])) < 5e-4
    rho4 = [np.zeros(n) for _ in range(4)]
    R.elecstate_pw_op_nc(int(d["DOMAG"]), int(d["DOMAG_Z"]), n, float(d["w2"]), rho4, d["wfcr_2"],
                         d["wfcr_another_spin_2"])
    for i in (0, 3):
        ex = d["expected_rho_2"][i * n:(i + 1) * n]
        assert np.max(np.abs(rho4[i] - ex) / np.abs(ex)) < 2e-5
    assert not np.any(rho4[1]) and not np.any(rho4[2])  # DOMAG_Z: the in-plane components are set to zero


# ------------------------------------------------------------------ GPU
torch = pytest.importorskip("torch")


@pytest.mark.gpu
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_gpu_elecstate_matches_oracle(pkg, golden, dt):
    P = pkg.pwdft
    rt, ct = (torch.float64, torch.complex128) if dt == "f64" else (torch.float32, torch.complex64)
    tol = 1e-13 if dt == "f64" else 1e-6
    d = golden("elecstate_op")
    n = int(d["nrxx"])
    ref = [np.full(n, 0.5)]
    R.elecstate_pw_op(0, n, float(d["w1"]), ref, d["wfcr"])
    rho = torch.full((n,), 0.5, dtype=rt, device="cuda")
    P.elecstate_pw_op(0, n, float(d["w1"]), [rho], torch.tensor(d["wfcr"], dtype=ct, device="cuda"))
    torch.cuda.synchronize()
    assert np.max(np.abs(rho.cpu().numpy() - ref[0]) / np.abs(ref[0])) < tol
    for domag, domag_z in ((0, 1), (1, 0), (0, 0)):
        ref4 = [np.full(n, 0.25 * (i + 1)) for i in range(4)]
        R.elecstate_pw_op_nc(domag, domag_z, n, float(d["w1"]), ref4, d["wfcr_2"], d["wfcr_another_spin_2"])
        rho4 = [torch.full((n,), 0.25 * (i + 1), dtype=rt, device="cuda") for i in range(4)]
        P.elecstate_pw_op_nc(domag, domag_z, n, float(d["w1"]), rho4, torch.tensor(d["wfcr_2"], dtype=ct, device="cuda"),
                             torch.tensor(d["wfcr_another_spin_2"], dtype=ct, device="cuda"))
        torch.cuda.synchronize()
        for i in range(4):
            assert np.max(np.abs(rho4[i].cpu().numpy() - ref4[i])) < tol * max(1.0, np.max(np.abs(ref4[i])))


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_gpu_psi_to_rho_matches_oracle(pkg, prec):
    """8-atom cell at a k-point: 12 bands with weights (two of them zero) against the oracle's band loop."""
    P = pkg.pwdft
    from oracle.pw_basis_ref import PWBasisKRef
    spec = pkg.synth.config(0)
    k = np.array([[0.125, -0.25, 0.375]])
    wl = P.build_workload(spec, kpts=k)
    b = wl.basis
    nb, ld = 12, b.npwk_max
    w1 = np.linspace(2.0, 0.1, nb) / b.omega
    w1[[3, 7]] = 0.0
    psi = wl.psi0_h[0][:nb].reshape(-1)
    ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, k, grid=spec.grid)
    ref = R.psi_to_rho(ref_b, 0, psi, nb, ld, w1, np.full(ref_b.nxyz, 0.01))
    f64 = prec == "f64"
    pd = torch.from_numpy(psi.astype(np.complex128 if f64 else np.complex64)).cuda()
    rho = torch.full((b.nx * b.ny * b.nz,), 0.01, dtype=torch.float64 if f64 else torch.float32, device="cuda")
    b.psi_to_rho(0, pd, nb, ld, w1, rho)
    torch.cuda.synchronize()
    got = rho.cpu().numpy().astype(np.float64)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < (1e-12 if f64 else 2e-6)


@pytest.mark.gpu
def test_gpu_psi_to_rho_sum_rule_64_atoms(pkg):
    """Size-independent property at the 64-atom size (96^3, 160 bands): sum_r rho(r) = N sum_b w1_b |c_b|^2
    (Parseval for the un-normalised backward transform)."""
    P = pkg.pwdft
    spec = pkg.synth.config(1)
    wl = P.build_workload(spec)
    b = wl.basis
    nb, ld = spec.nbands, b.npwk_max
    w1 = np.full(nb, 2.0 / b.omega)
    psi = wl.psi0_h[0][:nb]
    N = b.nx * b.ny * b.nz
    rho = torch.zeros(N, dtype=torch.float64, device="cuda")
    b.psi_to_rho(0, torch.from_numpy(psi.reshape(-1)).cuda(), nb, ld, w1, rho)
    torch.cuda.synchronize()
    expect = N * np.sum(w1[:, None] * np.abs(psi) ** 2)
    assert abs(rho.sum().item() - expect) / expect < 1e-12
    assert rho.min().item() >= 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n", [64, 96, 128])
def test_gpu_psi_to_rho_register_transforms_match_oracle(pkg, prec, n):
    """The fused path (grids with register transforms: inverse z pass, then per z plane the inverse y and x
    transforms with w|psi|^2 summed in registers, partial planes reduced in a fixed order) against the
    oracle's band loop, at a k-point, with zero-weight bands splitting the occupied runs."""
    import dataclasses
    P = pkg.pwdft
    from oracle.pw_basis_ref import PWBasisKRef
    spec = dataclasses.replace(pkg.synth.config(0), grid=(n, n, n))
    k = np.array([[0.125, -0.25, 0.375]])
    wl = P.build_workload(spec, kpts=k)
    b = wl.basis
    nb, ld = 10, b.npwk_max
    w1 = np.linspace(1.5, 0.2, nb) / b.omega
    w1[[0, 4, 5]] = 0.0
    psi = wl.psi0_h[0][:nb].reshape(-1)
    ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, k, grid=spec.grid)
    ref = R.psi_to_rho(ref_b, 0, psi, nb, ld, w1, np.full(ref_b.nxyz, 0.02))
    f64 = prec == "f64"
    pd = torch.from_numpy(psi.astype(np.complex128 if f64 else np.complex64)).cuda()
    rho = torch.full((n * n * n,), 0.02, dtype=torch.float64 if f64 else torch.float32, device="cuda")
    b.psi_to_rho(0, pd, nb, ld, w1, rho)
    torch.cuda.synchronize()
    got = rho.cpu().numpy().astype(np.float64)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < (1e-12 if f64 else 2e-6)
