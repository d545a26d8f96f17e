"""Projector generation (getvnl and its functors): the oracle against the reference's literals on the CPU,
the device functors and the fused getvnl against the oracle on the GPU.

Golden literals: cal_ylm_real_op (math_op_test.cpp, printed to 6 significant digits there), cal_sk_op
(wf_op_test.cpp), cal_vnl_op (vnl_op_test.cpp).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import vnl_ref as V


def _sk_args(w):
    return (int(w["ik"]), int(w["ntype"]), int(w["nx"]), int(w["ny"]), int(w["nz"]), int(w["rho_nx"]),
            int(w["rho_ny"]), int(w["rho_nz"]), int(w["npw"]), int(w["npwx"]), int(w["fftny"]), int(w["eigts1_nc"]),
            int(w["eigts2_nc"]), int(w["eigts3_nc"]))


def _vnl_counts(v):
    return (int(v["ntype"]), int(v["npw"]), int(v["npwx"]), int(v["nhm"]), int(v["tab_2"]), int(v["tab_3"]),
            [int(v["atom_na"])], [int(v["atom_nb"])], [int(v["atom_nh"])], float(v["DQ"]), float(v["tpiba"]))


def test_oracle_ylm_matches_golden(golden):
    d = golden("ylm_op")
    y = V.ylm_real(int(d["lmax"]), d["g"])
    assert np.max(np.abs(y.reshape(-1) - d["expected_ylm"])) < 1e-6  # literals carry 6 digits


def test_oracle_ylm_orthonormal_lmax3():
    """Size-independent property: the real Y_lm are orthonormal on the sphere (Gauss-Legendre in cos theta
    times a uniform grid in phi integrates these polynomials exactly)."""
    xs, ws = np.polynomial.legendre.leggauss(24)
    ph = np.linspace(0, 2 * np.pi, 48, endpoint=False)
    ct, pp = np.meshgrid(xs, ph, indexing="ij")
    st = np.sqrt(1 - ct ** 2)
    g = np.stack([st * np.cos(pp), st * np.sin(pp), ct], axis=-1).reshape(-1, 3)
    w = (ws[:, None] * np.full(len(ph), 2 * np.pi / len(ph))[None, :]).reshape(-1)
    y = V.ylm_real(3, g)
    gram = (y * w[None, :]) @ y.T
    assert np.max(np.abs(gram - np.eye(16))) < 1e-12


def test_oracle_sk_matches_golden(golden):
    w = golden("wf_op")
    sk = V.cal_sk(*_sk_args(w), [int(w["atom_na"])], w["igl2isz"], w["is2fftixy"], float(w["TWO_PI"]), w["kvec_c"],
                  w["atom_tau"], w["eigts1"], w["eigts2"], w["eigts3"])
    assert np.max(np.abs(sk.reshape(-1) - w["expected_sk"])) < 1e-12


def test_oracle_vnl_matches_golden(golden):
    v = golden("vnl_op")
    vkb = V.cal_vnl(*_vnl_counts(v), v["gk"], v["ylm"], v["indv"], v["nhtol"], v["nhtolm"], v["tab"], v["sk"])
    assert np.max(np.abs(vkb.reshape(-1) - v["expected_vkb"])) < 1e-11


def test_synthetic_tables_reproduce_analytic_projectors(pkg):
    """getvnl on the synthetic tables gives the analytic generator's projectors up to the sign of the
    l = 1, m = +-1 channels, within the 4-point interpolation error of a dq = 0.01 table (about 1e-8 of the
    largest value for these Gaussians)."""
    spec = pkg.synth.serving_cells()[1]
    cell = pkg.synth.make_cell(spec)
    from oracle.pw_basis_ref import PWBasisKRef
    k = np.array([[0.1, -0.2, 0.3]])
    b = PWBasisKRef(spec.a, cell.latvec, spec.ecut, k)
    proj = cell.projector_tables(b.omega, spec.ecut)
    vk = V.getvnl(b, 0, proj, cell.tau / spec.a)
    va = cell.vkb(b.gplusk_cart(0), b.npwk_max, b.omega)
    sign = np.array([1, 1, -1, -1, 1, 1, -1, -1] * cell.nat)[:, None]
    assert np.max(np.abs(vk - sign * va)) / np.max(np.abs(va)) < 1e-7


# ------------------------------------------------------------------ GPU
torch = pytest.importorskip("torch")


@pytest.mark.gpu
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_gpu_functors_match_golden(pkg, golden, dt):
    P = pkg.pwdft
    rt, ct = (torch.float64, torch.complex128) if dt == "f64" else (torch.float32, torch.complex64)
    tol = 1e-11 if dt == "f64" else 2e-5

    def cu(x, t):
        return torch.tensor(np.asarray(x), dtype=t, device="cuda")

    d = golden("ylm_op")
    ng, lmax = int(d["ng"]), int(d["lmax"])
    y = torch.zeros((lmax + 1) ** 2 * ng, dtype=rt, device="cuda")
    P.cal_ylm_real_op(ng, lmax, cu(d["g"], rt), y)
    ref = V.ylm_real(lmax, d["g"]).reshape(-1)
    assert np.max(np.abs(y.cpu().numpy() - ref)) < tol
    w = golden("wf_op")
    a = _sk_args(w)
    sk = torch.zeros(int(w["atom_na"]) * a[8], dtype=ct, device="cuda")
    P.cal_sk_op(*a, [int(w["atom_na"])], cu(w["igl2isz"], torch.int32), cu(w["is2fftixy"], torch.int32),
                float(w["TWO_PI"]), cu(w["kvec_c"], rt), cu(w["atom_tau"], rt), cu(w["eigts1"], ct), cu(w["eigts2"], ct),
                cu(w["eigts3"], ct), sk)
    assert np.max(np.abs(sk.cpu().numpy() - w["expected_sk"])) < tol
    v = golden("vnl_op")
    c = _vnl_counts(v)
    vkb = torch.zeros(v["expected_vkb"].size, dtype=ct, device="cuda")
    P.cal_vnl_op(*c, cu(v["gk"], rt), cu(v["ylm"], rt), cu(v["indv"], rt), cu(v["nhtol"], rt), cu(v["nhtolm"], rt),
                 cu(v["tab"], rt), None, cu(v["sk"], ct), vkb)
    ref = V.cal_vnl(*c, v["gk"], v["ylm"], v["indv"], v["nhtol"], v["nhtolm"], v["tab"], v["sk"]).reshape(-1)
    assert np.max(np.abs(vkb.cpu().numpy() - ref)) < tol
    assert np.max(np.abs(vkb.cpu().numpy() - v["expected_vkb"])) < 6e-5  # the reference test's own bound


@pytest.mark.gpu
def test_gpu_getvnl_matches_oracle(pkg):
    """Fused on-device getvnl against the oracle composition, at several k-points of the 16-atom cell."""
    P = pkg.pwdft
    spec = pkg.synth.serving_cells()[2]
    kpts = np.array([[0.0, 0.0, 0.0], [0.25, 0.0, 0.0], [0.5, 0.5, 0.0], [0.1, -0.3, 0.45]])
    wl = P.build_workload(spec, kpts=kpts)
    h = P.HamiltPW(wl.basis, P.PREC_FP64)
    proj = wl.cell.projector_tables(wl.basis.omega, spec.ecut)
    h.set_projectors(proj, wl.cell.tau / spec.a)
    from oracle.pw_basis_ref import PWBasisKRef
    ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, kpts, grid=spec.grid)
    for ik in range(len(kpts)):
        h.build_vkb(ik)
        out = torch.zeros(proj.nkb * wl.basis.npwk_max, dtype=torch.complex128, device="cuda")
        h.copy_vkb(ik, out)
        torch.cuda.synchronize()
        ref = V.getvnl(ref_b, ik, proj, wl.cell.tau / spec.a)
        got = out.cpu().numpy().reshape(proj.nkb, -1)
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-12, ik
