"""GPU parity of the full H|psi> (Operator::hPsi: Ekinetic -> Veff -> Nonlocal) against the oracle.

FP64 must match within 1e-12 relative; the mixed path
(FP32 FFTs and FP32 products) within 2e-5 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import hamilt_ref as H
from oracle.pw_basis_ref import PWBasisKRef

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def _setup(pkg, spec, kpt=None, nb=None):
    P = pkg.pwdft
    k = np.zeros((1, 3)) if kpt is None else np.atleast_2d(kpt)
    wl = P.build_workload(spec, kpts=k)
    b = wl.basis
    ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, k, grid=spec.grid)
    npwx = b.npwk_max
    ref = H.HamiltPWRef(ref_b, 0, wl.veff_h, wl.vkb_h[0][:, :npwx], wl.deeq_h, [8], [wl.cell.nat])
    nb = nb or spec.nbands
    psi = wl.psi0_h[0][:nb].reshape(-1)
    return wl, ref, psi, nb, npwx


@pytest.mark.parametrize("gemm", [0, 2])  # FP64 projector products: cuBLAS ZGEMM / int8 tensor cores
@pytest.mark.parametrize("cfg", ["si2", "diamond8", "diamond8_k", "diamond16", "diamond8_grid40", "diamond8_grid96_k",
                                 "diamond8_grid128"])
def test_hpsi_fp64_matches_oracle(pkg, cfg, gemm):
    S = pkg.synth
    if cfg == "si2":
        spec, kpt, nb = S.serving_cells()[0], None, 8
    elif cfg == "diamond8":
        spec, kpt, nb = S.config(0), None, 32
    elif cfg == "diamond8_k":
        spec, kpt, nb = S.config(0), np.array([0.125, -0.375, 0.375]), 12
    elif cfg == "diamond16":
        spec, kpt, nb = S.serving_cells()[2], None, 6
    elif cfg == "diamond8_grid40":  # a grid outside the compiled warp-transform sizes: the generic kernels
        import dataclasses
        spec, kpt, nb = dataclasses.replace(S.config(0), grid=(40, 40, 40)), None, 10
    else:  # square planes of 32*m points: the register/shuffle plane transforms
        import dataclasses
        n = 96 if "96" in cfg else 128
        kpt = np.array([0.25, -0.125, 0.375]) if cfg.endswith("_k") else None
        spec, nb = dataclasses.replace(S.config(0), grid=(n, n, n)), 6
    wl, ref, psi, nb, ld = _setup(pkg, spec, kpt, nb)
    href = ref.hpsi(psi, nb, ld)
    h = pkg.pwdft.device_hamilt(wl, pkg.pwdft.PREC_FP64)
    h.set_fp64_gemm(gemm)
    pd = torch.from_numpy(psi).cuda()
    hd = torch.full_like(pd, complex(7.0, -3.0))  # garbage: hPsi must overwrite, padding included
    h.hpsi(0, pd, hd, nb, ld)
    torch.cuda.synchronize()
    out = hd.cpu().numpy()
    assert rel(out, href) < 1e-12
    # local and nonlocal parts separately
    hl = torch.zeros_like(pd)
    h.hpsi_part(0, pd, hl, nb, ld, mode=1)
    torch.cuda.synchronize()
    assert rel(hl.cpu().numpy(), ref.hpsi_local(psi, nb, ld)) < 1e-12


@pytest.mark.parametrize("grid", [None, (96, 96, 96)])
def test_hpsi_mixed_matches_oracle(pkg, grid):
    import dataclasses
    spec = pkg.synth.config(0) if grid is None else dataclasses.replace(pkg.synth.config(0), grid=grid)
    wl, ref, psi, nb, ld = _setup(pkg, spec, None, 32 if grid is None else 6)
    href = ref.hpsi(psi, nb, ld)
    h = pkg.pwdft.device_hamilt(wl, pkg.pwdft.PREC_MIXED)
    pd = torch.from_numpy(psi.astype(np.complex64)).cuda()
    hd = torch.zeros_like(pd)
    h.hpsi(0, pd, hd, nb, ld)
    torch.cuda.synchronize()
    assert rel(hd.cpu().numpy().astype(np.complex128), href) < 2e-5


def test_hpsi_is_hermitian_and_linear(pkg):
    """Size-independent properties at the 64-atom size: <a|H b> = <H a|b>, H(a + 2b) = Ha + 2Hb."""
    spec = pkg.synth.config(1)
    P = pkg.pwdft
    wl = P.build_workload(spec)
    h = P.device_hamilt(wl, P.PREC_FP64)
    ld = wl.basis.npwk_max
    rng = np.random.default_rng(5)
    npw = int(wl.basis.npwk[0])
    a = np.zeros(ld, complex)
    b = np.zeros(ld, complex)
    a[:npw] = rng.standard_normal(npw) + 1j * rng.standard_normal(npw)
    b[:npw] = rng.standard_normal(npw) + 1j * rng.standard_normal(npw)
    x = torch.from_numpy(np.concatenate([a, b, a + 2 * b])).cuda()
    hx = torch.zeros_like(x)
    h.hpsi(0, x, hx, 3, ld)
    torch.cuda.synchronize()
    ha, hb, hab = hx.cpu().numpy().reshape(3, ld)
    assert abs(np.vdot(a, hb) - np.vdot(ha, b)) < 1e-11 * abs(np.vdot(a, hb)) + 1e-9
    assert rel(hab, ha + 2 * hb) < 1e-13


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("pieces,pinned", [(1, True), (3, True), (4, True), (5, False)])
def test_hpsi_host_pipeline_equals_device_hpsi(pkg, prec, pieces, pinned):
    """b200_hamilt_hpsi_host (host buffers, uploads / H|psi> pieces / downloads overlapped on three streams)
    gives the device H|psi> of the same pieces bit for bit (the projector GEMM of a smaller piece may round
    differently from the whole block's: within 1e-13 of it), for uneven pieces and for pinned and pageable
    host buffers."""
    P = pkg.pwdft
    wl, _, psi, nb, ld = _setup(pkg, pkg.synth.config(0), None, 13)
    p = P.PREC_FP64 if prec == "fp64" else P.PREC_MIXED
    ct = torch.complex128 if prec == "fp64" else torch.complex64
    h = P.device_hamilt(wl, p)
    ph = torch.from_numpy(psi.copy()).to(ct)
    ref_d = torch.zeros(nb * ld, dtype=ct, device="cuda")
    whole = torch.zeros(nb * ld, dtype=ct, device="cuda")
    pdev = ph.cuda()
    h.hpsi(0, pdev, whole, nb, ld)
    P_ = min(pieces, nb)

    # the pipeline's pieces weigh 1, 2, ..., 2, 1 (two pieces: 1, 1), at least one band each
    bnd = [0] * (P_ + 1)
    total = 2 * (P_ - 1)
    for q in range(1, P_):
        bnd[q] = nb * (2 * q - 1) // total
    bnd[P_] = nb
    for q in range(1, P_):
        bnd[q] = max(bnd[q], bnd[q - 1] + 1)
    for q in range(P_ - 1, 0, -1):
        bnd[q] = min(bnd[q], bnd[q + 1] - 1)

    for q in range(P_):
        b0, b1 = bnd[q], bnd[q + 1]
        h.hpsi(0, pdev[b0 * ld:], ref_d[b0 * ld:], b1 - b0, ld)
    if pinned:
        ph = ph.pin_memory()
    out_h = torch.full((nb * ld,), 7.0, dtype=ct)
    if pinned:
        out_h = out_h.pin_memory()
    pd = torch.zeros(nb * ld, dtype=ct, device="cuda")
    hd = torch.zeros(nb * ld, dtype=ct, device="cuda")
    h.hpsi_host(0, ph, out_h, pd, hd, nb, ld, pieces=pieces)
    torch.cuda.synchronize()
    assert torch.equal(out_h, ref_d.cpu())
    tol = 1e-13 if prec == "fp64" else 1e-6
    assert rel(out_h.numpy(), whole.cpu().numpy()) < tol


@pytest.mark.parametrize("cfg", [1, 4])
def test_headline_cells_match_oracle(pkg, cfg):
    """The benchmarked cells at full size: the 64-atom cell (96^3, npw 51 627, 512 projectors) and the
    216-atom cell (128^3, npw 124 289, 1728 projectors), as the bench builds them (projectors by the fused
    device getvnl).  Against the oracle (oracle/vnl_ref.getvnl, oracle/hamilt_ref: Ekinetic, Veff, and
    Nonlocal::act as gemm('C','N') -> nonlocal_pw_op -> gemm('N','T'), nonlocal_pw.cpp:211-304):
    the projectors and the FP64 H|psi> of 6 bands within 1e-12 relative, the local and nonlocal parts each
    within 1e-12 of their own size; the mixed path within 2e-5."""
    from oracle import vnl_ref as V
    P = pkg.pwdft
    spec = pkg.synth.config(cfg)
    cell = pkg.synth.make_cell(spec)
    k = np.zeros((1, 3))
    basis = P.PWBasisK(spec.a, cell.latvec, spec.ecut, k, grid=spec.grid)
    ref_b = PWBasisKRef(spec.a, cell.latvec, spec.ecut, k, grid=spec.grid)
    ld = basis.npwk_max
    assert ld == int(ref_b.npwk[0])
    nb = 6
    veff = cell.veff(basis.nx, basis.ny, basis.nz)
    deeq = cell.deeq()
    proj = cell.projector_tables(basis.omega, spec.ecut)
    tau = cell.tau / spec.a
    vkb_o = V.getvnl(ref_b, 0, proj, tau)
    psi = cell.psi0(basis.gplusk_cart(0), nb, ld).reshape(-1)
    ref = H.HamiltPWRef(ref_b, 0, veff, vkb_o, deeq, [8], [cell.nat])
    href = ref.hpsi(psi, nb, ld)
    hloc = ref.hpsi_local(psi, nb, ld)
    hnl = href - hloc
    vd = torch.from_numpy(veff).cuda()
    dd = torch.from_numpy(deeq).cuda()
    pd = torch.from_numpy(psi).cuda()
    for prec in (P.PREC_FP64, P.PREC_MIXED):
        h = P.HamiltPW(basis, prec)
        h.set_veff(vd)
        h.set_deeq([cell.nat], [pkg.synth.NH], dd)
        h.set_projectors(proj, tau)
        h.build_vkb(0)
        if prec == P.PREC_FP64:
            out = torch.zeros(proj.nkb * ld, dtype=torch.complex128, device="cuda")
            h.copy_vkb(0, out)
            torch.cuda.synchronize()
            assert rel(out.cpu().numpy().reshape(proj.nkb, ld), vkb_o) < 1e-12
            del out
            hd = torch.full_like(pd, complex(7.0, -3.0))
            h.hpsi(0, pd, hd, nb, ld)
            hl = torch.zeros_like(pd)
            h.hpsi_part(0, pd, hl, nb, ld, mode=1)
            hn = torch.zeros_like(pd)
            h.hpsi_part(0, pd, hn, nb, ld, mode=2)
            torch.cuda.synchronize()
            assert rel(hd.cpu().numpy(), href) < 1e-12
            assert rel(hl.cpu().numpy(), hloc) < 1e-12
            assert rel(hn.cpu().numpy(), hnl) < 1e-12
        else:
            p32 = pd.to(torch.complex64)
            hd = torch.zeros_like(p32)
            h.hpsi(0, p32, hd, nb, ld)
            torch.cuda.synchronize()
            assert rel(hd.cpu().numpy().astype(np.complex128), href) < 2e-5
        del h
        torch.cuda.empty_cache()


@pytest.mark.parametrize("n", [64, 96, 128])
@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5])
def test_plane_variants_match_oracle(pkg, n, variant):
    """Every plane-pass variant of the register transforms (1: warp-shuffle lane stages; 2-5: two-pass
    transforms through shared memory in four launch shapes) gives the oracle's local H|psi> (kinetic +
    V_eff) on square planes of 64, 96 and 128 points, at k != 0: FP64 within 1e-12, mixed within 2e-5."""
    import dataclasses
    spec = dataclasses.replace(pkg.synth.config(0), grid=(n, n, n))
    wl, ref, psi, nb, ld = _setup(pkg, spec, np.array([0.25, -0.125, 0.375]), 6)
    href = ref.hpsi_local(psi, nb, ld)
    P = pkg.pwdft
    for prec in (P.PREC_FP64, P.PREC_MIXED):
        h = P.device_hamilt(wl, prec)
        h.set_plane_variant(variant)
        ct = torch.complex128 if prec == P.PREC_FP64 else torch.complex64
        pd = torch.from_numpy(psi).to(ct).cuda()
        hd = torch.full_like(pd, complex(7.0, -3.0))
        h.hpsi_part(0, pd, hd, nb, ld, mode=1)
        torch.cuda.synchronize()
        err = rel(hd.cpu().numpy().astype(np.complex128), href)
        assert err < (1e-12 if prec == P.PREC_FP64 else 2e-5), (prec, err)
        h.set_plane_variant(0)
