"""Python face of the plane-wave H|psi> / Davidson C-ABI.

Names, argument order and meaning follow the reference's op functors,
PW_Basis_K and DiagoDavid (abacus-develop v3.8.0) so that tests read like the
reference's own.  Device buffers are torch CUDA tensors (torch is used for
device memory and streams only; every computation runs in libabacus_b200.so).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import call, ptr, stream_ptr

PREC_FP64 = 0
PREC_MIXED = 1


def _torch():
    import torch
    return torch


def _f64p(a: np.ndarray):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_lib.pf64)


# ------------------------------------------------------------------ op functors
def ekinetic_pw_op(nband, npw, max_npw, tpiba2, gk2_ik, tmhpsi, tmpsi_in, stream=None):
    """ekinetic_pw_op<FP, DEVICE_GPU> (ekinetic_op.h:38-48); FP from the tensors' dtype."""
    torch = _torch()
    f = "b200_ekinetic_pw_op_f64" if tmhpsi.dtype == torch.complex128 else "b200_ekinetic_pw_op_f32"
    call(f, nband, npw, max_npw, tpiba2, ptr(gk2_ik), ptr(tmhpsi), ptr(tmpsi_in), stream_ptr(stream))


def veff_pw_op(size, out, vin, stream=None):
    """veff_pw_op<FP, DEVICE_GPU>(dev, size, out, in) (veff_op.h:57-66)."""
    torch = _torch()
    f = "b200_veff_pw_op_f64" if out.dtype == torch.complex128 else "b200_veff_pw_op_f32"
    call(f, size, ptr(out), ptr(vin), stream_ptr(stream))


def veff_pw_op_npol2(size, out, out1, vin4, stream=None):
    """veff_pw_op<FP, DEVICE_GPU>(dev, size, out, out1, in[4]) (veff_op.h:57-66)."""
    torch = _torch()
    f = "b200_veff_pw_op_npol2_f64" if out.dtype == torch.complex128 else "b200_veff_pw_op_npol2_f32"
    call(f, size, ptr(out), ptr(out1), *(ptr(v) for v in vin4), stream_ptr(stream))


def nonlocal_pw_op(l1, l2, l3, sum_, iat, spin, nkb, deeq_x, deeq_y, deeq_z, deeq, ps, becp, stream=None):
    """nonlocal_pw_op<FP, DEVICE_GPU> (nonlocal_op.h:82-113). Returns the updated (sum, iat)."""
    torch = _torch()
    s, i = C.c_int(sum_), C.c_int(iat)
    f = "b200_nonlocal_pw_op_f64" if ps.dtype == torch.complex128 else "b200_nonlocal_pw_op_f32"
    call(f, l1, l2, l3, C.byref(s), C.byref(i), spin, nkb, deeq_x, deeq_y, deeq_z, ptr(deeq), ptr(ps), ptr(becp),
         stream_ptr(stream))
    return s.value, i.value


def nonlocal_pw_op_nc(l1, l2, l3, sum_, iat, nkb, deeq_x, deeq_y, deeq_z, deeq_nc, ps, becp, stream=None):
    torch = _torch()
    s, i = C.c_int(sum_), C.c_int(iat)
    f = "b200_nonlocal_pw_op_nc_f64" if ps.dtype == torch.complex128 else "b200_nonlocal_pw_op_nc_f32"
    call(f, l1, l2, l3, C.byref(s), C.byref(i), nkb, deeq_x, deeq_y, deeq_z, ptr(deeq_nc), ptr(ps), ptr(becp),
         stream_ptr(stream))
    return s.value, i.value


def set_3d_fft_box_op(npwk, box_index, inp, out, stream=None):
    torch = _torch()
    f = "b200_set_3d_fft_box_op_f64" if out.dtype == torch.complex128 else "b200_set_3d_fft_box_op_f32"
    call(f, npwk, ptr(box_index), ptr(inp), ptr(out), stream_ptr(stream))


def set_recip_to_real_output_op(nrxx, add, factor, inp, out, stream=None):
    torch = _torch()
    f = "b200_set_recip_to_real_output_op_f64" if out.dtype == torch.complex128 else "b200_set_recip_to_real_output_op_f32"
    call(f, nrxx, int(add), factor, ptr(inp), ptr(out), stream_ptr(stream))


def set_real_to_recip_output_op(npw_k, nxyz, add, factor, box_index, inp, out, stream=None):
    torch = _torch()
    f = "b200_set_real_to_recip_output_op_f64" if out.dtype == torch.complex128 else "b200_set_real_to_recip_output_op_f32"
    call(f, npw_k, nxyz, int(add), factor, ptr(box_index), ptr(inp), ptr(out), stream_ptr(stream))


def tc_cgemm(transa, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=None):
    """gemm_op<complex<float>, DEVICE_GPU> on the tensor cores (3xTF32 split precision):
    C = alpha*op(A)*B + beta*C, column-major complex64, transa 'N' or 'C', transb 'N'."""
    alpha = complex(alpha)
    beta = complex(beta)
    call("b200_tc_cgemm", transa.encode(), b"N", m, n, k, alpha.real, alpha.imag, ptr(a), lda, ptr(b), ldb,
         beta.real, beta.imag, ptr(c), ldc, stream_ptr(stream))


def zgemm_i8(transa, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, nmods=16, stream=None):
    """gemm_op<complex<double>, DEVICE_GPU> on the int8 tensor cores (exact modular emulation of the FP64
    product): C = alpha*op(A)*B + beta*C, column-major complex128, transa 'N' or 'C', transb 'N'."""
    al = (C.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    be = (C.c_double * 2)(complex(beta).real, complex(beta).imag)
    call("b200_zgemm_i8", transa.encode(), b"N", m, n, k, al, ptr(a), lda, ptr(b), ldb, be, ptr(c), ldc, int(nmods),
         stream_ptr(stream))


def zgemm_i8_error():
    """Error word of this thread's int8 GEMMs (nonzero: a bounded wait ran out); the read clears it."""
    code = C.c_int()
    call("b200_zgemm_i8_error", C.byref(code))
    return code.value


def zgemm_i8_constants(nmods, kr):
    """Recombination constants of the int8 GEMM for nmods moduli and real rows of length kr: the moduli,
    the weights w_l / M as (wa, wb), M as a double and the scale exponent q.  No GPU needed."""
    mods = (C.c_int * nmods)()
    wa = (C.c_double * nmods)()
    wb = (C.c_double * nmods)()
    mp = C.c_double()
    q = C.c_int()
    call("b200_zgemm_i8_constants", int(nmods), int(kr), mods, wa, wb, C.byref(mp), C.byref(q))
    return list(mods), list(wa), list(wb), mp.value, q.value


def tc_cgemm_error():
    """Error word of this thread's tensor-core GEMMs (nonzero: a bounded wait ran out); the read clears it."""
    code = C.c_int()
    call("b200_tc_cgemm_error", C.byref(code))
    return code.value


def measure_peaks():
    """Measured FP64 / FP32 CUDA-core FMA and FP64 tensor-core MMA peaks of the current device, TFLOP/s."""
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    call("b200_measure_peaks", C.byref(a), C.byref(b), C.byref(c))
    return {"fp64_tflops": a.value, "fp32_tflops": b.value, "dmma_fp64_tflops": c.value}


def tc_set_wait_limit_ns(ns):
    """Limit of each pipeline wait inside the tensor-core GEMMs launched afterwards (0: the default, 2 s)."""
    call("b200_tc_set_wait_limit_ns", int(ns))


def _ints(v):
    v = [int(x) for x in v]
    return (C.c_int * max(1, len(v)))(*v)


def _check_block(t, complex128: bool, nbands: int, ld: int, what: str):
    """The C-ABI takes device pointers without types or sizes: refuse a tensor whose element type is not the
    one the call will read or that holds fewer than nbands*ld elements (an out-of-bounds device access)."""
    torch = _torch()
    want = torch.complex128 if complex128 else torch.complex64
    if t.dtype != want:
        raise TypeError(f"{what}: expected {want}, got {t.dtype}")
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError(f"{what}: expected a contiguous CUDA tensor")
    if t.numel() < int(nbands) * int(ld):
        raise ValueError(f"{what}: {t.numel()} elements, the call reads or writes {int(nbands) * int(ld)}")


def elecstate_pw_op(spin, nrxx, w1, rho, wfcr, stream=None):
    """elecstate_pw_op<FP, DEVICE_GPU>: rho[spin] += w1*|wfcr|^2; rho is a sequence of nspin device tensors."""
    torch = _torch()
    f = "b200_elecstate_pw_op_f64" if wfcr.dtype == torch.complex128 else "b200_elecstate_pw_op_f32"
    arr = (_lib.vp * len(rho))(*[ptr(r) for r in rho])
    call(f, spin, nrxx, w1, arr, ptr(wfcr), stream_ptr(stream))


def elecstate_pw_op_nc(domag, domag_z, nrxx, w1, rho, wfcr, wfcr_another_spin, stream=None):
    """The nspin = 4 overload of elecstate_pw_op; rho is a sequence of 4 device tensors."""
    torch = _torch()
    f = "b200_elecstate_pw_op_nc_f64" if wfcr.dtype == torch.complex128 else "b200_elecstate_pw_op_nc_f32"
    arr = (_lib.vp * 4)(*[ptr(r) for r in rho])
    call(f, int(domag), int(domag_z), nrxx, w1, arr, ptr(wfcr), ptr(wfcr_another_spin), stream_ptr(stream))


def cal_ylm_real_op(ng, lmax, g, ylm, stream=None):
    """ModuleBase::cal_ylm_real_op<FP, DEVICE_GPU>: g (ng x 3) -> ylm ((lmax+1)^2 x ng)."""
    torch = _torch()
    f = "b200_cal_ylm_real_op_f64" if ylm.dtype == torch.float64 else "b200_cal_ylm_real_op_f32"
    call(f, ng, lmax, ptr(g), ptr(ylm), stream_ptr(stream))


def cal_sk_op(ik, ntype, nx, ny, nz, rho_nx, rho_ny, rho_nz, npw, npwx, fftny, eigts1_nc, eigts2_nc, eigts3_nc,
              atom_na, igl2isz, is2fftixy, two_pi, kvec_c, atom_tau, eigts1, eigts2, eigts3, sk, stream=None):
    """hamilt::cal_sk_op<FP, DEVICE_GPU> (wf_op.h); atom_na is a host sequence, the rest device tensors."""
    torch = _torch()
    f = "b200_cal_sk_op_f64" if sk.dtype == torch.complex128 else "b200_cal_sk_op_f32"
    call(f, ik, ntype, nx, ny, nz, rho_nx, rho_ny, rho_nz, npw, npwx, fftny, eigts1_nc, eigts2_nc, eigts3_nc,
         _ints(atom_na), ptr(igl2isz), ptr(is2fftixy), two_pi, ptr(kvec_c), ptr(atom_tau), ptr(eigts1), ptr(eigts2),
         ptr(eigts3), ptr(sk), stream_ptr(stream))


def cal_vnl_op(ntype, npw, npwx, nhm, tab_2, tab_3, atom_na, atom_nb, atom_nh, dq, tpiba, gk, ylm, indv, nhtol,
               nhtolm, tab, vkb1, sk, vkb, stream=None):
    """hamilt::cal_vnl_op<FP, DEVICE_GPU> (vnl_op.h:58-100); per-type counts are host sequences."""
    torch = _torch()
    f = "b200_cal_vnl_op_f64" if vkb.dtype == torch.complex128 else "b200_cal_vnl_op_f32"
    call(f, ntype, npw, npwx, nhm, tab_2, tab_3, _ints(atom_na), _ints(atom_nb), _ints(atom_nh), dq, tpiba, ptr(gk),
         ptr(ylm), ptr(indv), ptr(nhtol), ptr(nhtolm), ptr(tab), ptr(vkb1), ptr(sk), ptr(vkb), stream_ptr(stream))


@dataclass
class ProjectorSet:
    """The projector tables getvnl reads (pseudopot_cell_vnl after init_vnl): per type na / nbeta / nh, the
    (ih -> beta, l, lm) maps indv / nhtol / nhtolm (ntype x nhm), the radial table tab (ntype x tab_2 x tab_3,
    step dq in bohr^-1) and lmax."""
    ntype: int
    na: list
    nbeta: list
    nh: list
    nhm: int
    lmax: int
    indv: np.ndarray
    nhtol: np.ndarray
    nhtolm: np.ndarray
    tab: np.ndarray
    dq: float

    @property
    def tab_2(self):
        return int(self.tab.shape[1])

    @property
    def tab_3(self):
        return int(self.tab.shape[2])

    @property
    def nkb(self):
        return int(sum(a * h for a, h in zip(self.na, self.nh)))


# ------------------------------------------------------------------ basis
class PWBasisK:
    """ModulePW::PW_Basis_K for one pool: grid, G sphere, index maps, device transforms."""

    def __init__(self, lat0, latvec, ecutwfc, kvec_d, ecutrho=None, grid=None):
        lib = _lib.load()
        lv, lvp = _f64p(np.asarray(latvec, dtype=np.float64).reshape(9))
        kd, kdp = _f64p(np.atleast_2d(np.asarray(kvec_d, dtype=np.float64)).reshape(-1))
        nks = kd.size // 3
        gx, gy, gz = grid if grid is not None else (0, 0, 0)
        h = _lib.vp()
        call("b200_pw_basis_create", float(lat0), lvp, float(ecutwfc), float(ecutrho or 0.0), gx, gy, gz, nks, kdp,
             C.byref(h))
        self._h = h
        self._lib = lib
        dims = (C.c_int * 8)()
        call("b200_pw_basis_dims", h, dims)
        self.nx, self.ny, self.nz, self.nst, self.npw, self.npwk_max, self.nks, self.nxc = list(dims)
        sc = (C.c_double * 3)()
        call("b200_pw_basis_scalars", h, sc)
        self.tpiba2, self.omega, self.gk_ecut = list(sc)
        self.lat0 = float(lat0)
        self.npwk = np.zeros(self.nks, dtype=np.int64)
        self._kcache = {}
        for ik in range(self.nks):
            n = C.c_int()
            call("b200_pw_basis_kpoint", h, ik, C.byref(n), None, None, None)
            self.npwk[ik] = n.value

    @property
    def handle(self):
        return self._h

    @property
    def nxyz(self):
        return self.nx * self.ny * self.nz

    def _k(self, ik):
        if ik not in self._kcache:
            n = int(self.npwk[ik])
            idx = np.zeros(n, dtype=np.int32)
            gk2 = np.zeros(n)
            gcar = np.zeros((n, 3))
            call("b200_pw_basis_kpoint", self._h, ik, None, idx.ctypes.data_as(_lib.vp), gk2.ctypes.data_as(_lib.vp),
                 gcar.ctypes.data_as(_lib.vp))
            kc = (C.c_double * 3)()
            call("b200_pw_basis_kvec_c", self._h, ik, kc)
            self._kcache[ik] = (idx, gk2, gcar, np.array(list(kc)))
        return self._kcache[ik]

    def ig2ixyz(self, ik):
        return self._k(ik)[0].astype(np.int64)

    def kvec_c(self, ik):
        """k-point ik in cartesian units of 2 pi / lat0 (PW_Basis_K::kvec_c)."""
        return self._k(ik)[3].copy()

    def gk2_k(self, ik):
        return self._k(ik)[1]

    def gplusk_cart(self, ik):
        """k+G cartesian in bohr^-1."""
        _, _, gcar, kc = self._k(ik)
        return (gcar + kc[None, :]) * np.sqrt(self.tpiba2)

    def device_maps(self, ik):
        g, gf, ix = _lib.vp(), _lib.vp(), _lib.vp()
        call("b200_pw_basis_device_maps", self._h, ik, C.byref(g), C.byref(gf), C.byref(ix))
        return g.value, gf.value, ix.value

    def recip_to_real(self, inp, out, ik, add=False, factor=1.0, stream=None):
        """PW_Basis_K::recip_to_real<FP, DEVICE_GPU> (pw_basis_k.h:140-153)."""
        torch = _torch()
        f = "b200_recip_to_real_f64" if out.dtype == torch.complex128 else "b200_recip_to_real_f32"
        call(f, self._h, ptr(inp), ptr(out), ik, int(add), factor, stream_ptr(stream))

    def real_to_recip(self, inp, out, ik, add=False, factor=1.0, stream=None):
        """PW_Basis_K::real_to_recip<FP, DEVICE_GPU> (pw_basis_k.h:140-153)."""
        torch = _torch()
        f = "b200_real_to_recip_f64" if out.dtype == torch.complex128 else "b200_real_to_recip_f32"
        call(f, self._h, ptr(inp), ptr(out), ik, int(add), factor, stream_ptr(stream))

    def psi_to_rho(self, ik, psi, nbands, ld, w1, rho, stream=None):
        """psiToRho's band loop for k-point ik: rho[r] += w1[ib]*|psi_ib(r)|^2 (rho in ABACUS's r order)."""
        torch = _torch()
        f64 = psi.dtype == torch.complex128
        _check_block(psi, f64, nbands, ld, "psi")
        if rho.dtype != (torch.float64 if f64 else torch.float32) or rho.numel() < self.nx * self.ny * self.nz:
            raise ValueError("rho: need a real tensor of the psi precision with nx*ny*nz entries")
        w = np.ascontiguousarray(np.asarray(w1, dtype=np.float64))
        if len(w) < nbands:
            raise ValueError("w1: need nbands weights")
        call("b200_pw_basis_psi_to_rho_f64" if f64 else "b200_pw_basis_psi_to_rho_f32", self._h, ik, nbands, ld,
             ptr(psi), w.ctypes.data_as(_lib.pf64), ptr(rho), stream_ptr(stream))

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.b200_pw_basis_destroy(self._h)
                self._h = None
        except Exception:
            pass


# ------------------------------------------------------------------ Hamiltonian
class HamiltPW:
    """Ekinetic -> Veff -> Nonlocal on the device (HamiltPW, hamilt_pw.cpp:21-114)."""

    def __init__(self, basis: PWBasisK, precision=PREC_FP64):
        self.basis = basis
        self.precision = precision
        h = _lib.vp()
        call("b200_hamilt_create", basis.handle, precision, C.byref(h))
        self._h = h
        self._lib = _lib.load()
        self._keep = []

    @property
    def handle(self):
        return self._h

    def set_veff(self, veff_d):
        call("b200_hamilt_set_veff", self._h, ptr(veff_d))

    def set_vkb(self, ik, vkb_d):
        nkb, npwx = (0, 0) if vkb_d is None else (int(vkb_d.shape[0]), int(vkb_d.shape[1]))
        call("b200_hamilt_set_vkb", self._h, ik, nkb, npwx, ptr(vkb_d))

    def set_deeq(self, na, nh, deeq_d):
        na_a = (C.c_int * len(na))(*na)
        nh_a = (C.c_int * len(nh))(*nh)
        ns, dx, dy, dz = (int(v) for v in deeq_d.shape)
        call("b200_hamilt_set_deeq", self._h, len(na), na_a, nh_a, ns, dx, dy, dz, ptr(deeq_d))

    def set_veff_nc(self, veff4_d):
        """npol = 2: V_eff's four components, a (4, nrxx) float64 device tensor in set_veff's order."""
        torch = _torch()
        if veff4_d.dtype != torch.float64 or veff4_d.numel() < 4 * self.basis.nxyz:
            raise ValueError("veff4_d must be float64 with 4 x nrxx values")
        call("b200_hamilt_set_veff_nc", self._h, ptr(veff4_d))

    def set_deeq_nc(self, na, nh, deeq_nc_d):
        """npol = 2: D's four complex spin blocks, a (4, dx, dy, dz) complex128 device tensor."""
        na_a = (C.c_int * len(na))(*na)
        nh_a = (C.c_int * len(nh))(*nh)
        four, dx, dy, dz = (int(v) for v in deeq_nc_d.shape)
        if four != 4:
            raise ValueError("deeq_nc_d must have shape (4, dx, dy, dz)")
        call("b200_hamilt_set_deeq_nc", self._h, len(na), na_a, nh_a, dx, dy, dz, ptr(deeq_nc_d))

    def hpsi_nc(self, ik, psi, hpsi, nbands, ld, stream=None):
        """Operator::hPsi with npol = 2: band b's spinor components at psi[(2b + c) ld : ...]."""
        self._chk(psi, hpsi, 2 * nbands, ld)
        call("b200_hamilt_hpsi_nc", self._h, ik, nbands, ld, ptr(psi), ptr(hpsi), stream_ptr(stream))

    def _chk(self, psi, hpsi, nbands, ld):
        f64 = self.precision == PREC_FP64
        _check_block(psi, f64, nbands, ld, "psi")
        _check_block(hpsi, f64, nbands, ld, "hpsi")

    def hpsi(self, ik, psi, hpsi, nbands, ld, spin=0, stream=None):
        """Operator::hPsi: hpsi = H psi for bands [0, nbands)."""
        self._chk(psi, hpsi, nbands, ld)
        call("b200_hamilt_hpsi", self._h, ik, spin, nbands, ld, ptr(psi), ptr(hpsi), stream_ptr(stream))

    def hpsi_host(self, ik, psi_h, hpsi_h, psi_d, hpsi_d, nbands, ld, pieces=4, spin=0, stream=None):
        """H|psi> from a host psi_h into a host hpsi_h through the device buffers psi_d / hpsi_d, with the
        uploads, the H|psi> pieces and the downloads overlapped on three streams (pinned host tensors give
        the overlap).  Asynchronous: hpsi_h is complete when the stream is."""
        torch = _torch()
        self._chk(psi_d, hpsi_d, nbands, ld)
        want = torch.complex128 if self.precision == PREC_FP64 else torch.complex64
        for t, what in ((psi_h, "psi_h"), (hpsi_h, "hpsi_h")):
            if t.dtype != want or t.is_cuda or not t.is_contiguous() or t.numel() < int(nbands) * int(ld):
                raise ValueError(f"{what}: expected a contiguous host {want} tensor of at least nbands*ld elements")
        call("b200_hamilt_hpsi_host", self._h, ik, spin, nbands, ld, ptr(psi_h), ptr(hpsi_h), ptr(psi_d),
             ptr(hpsi_d), int(pieces), stream_ptr(stream))

    def hpsi_part(self, ik, psi, hpsi, nbands, ld, mode, spin=0, stream=None):
        self._chk(psi, hpsi, nbands, ld)
        call("b200_hamilt_hpsi_part", self._h, ik, spin, nbands, ld, ptr(psi), ptr(hpsi), mode, stream_ptr(stream))

    def hpsi_local_noalloc(self, ik, psi, hpsi, nbands, ld, stream=None):
        """Kinetic + local part of H|psi> without any device allocation during the call, for callers that
        cannot allocate (graph capture, externally owned memory pools); scratch is a fixed 32 MiB array
        inside the library shared by all calls, so concurrent calls on one device must be serialised."""
        self._chk(psi, hpsi, nbands, ld)
        call("b200_hamilt_hpsi_local_noalloc", self._h, ik, nbands, ld, ptr(psi), ptr(hpsi), stream_ptr(stream))

    def set_projectors(self, proj: ProjectorSet, tau_lat0):
        """Projector tables for on-device getvnl; tau_lat0: (nat, 3) positions in units of lat0, by type."""
        tab = np.ascontiguousarray(proj.tab, dtype=np.float64).reshape(-1)
        tau = np.ascontiguousarray(tau_lat0, dtype=np.float64).reshape(-1)
        call("b200_hamilt_set_projectors", self._h, proj.ntype, _ints(proj.na), _ints(proj.nbeta), _ints(proj.nh),
             proj.nhm, proj.lmax, _ints(np.asarray(proj.indv).reshape(-1)), _ints(np.asarray(proj.nhtol).reshape(-1)),
             _ints(np.asarray(proj.nhtolm).reshape(-1)), proj.tab_2, proj.tab_3, float(proj.dq),
             tab.ctypes.data_as(_lib.pf64), tau.ctypes.data_as(_lib.pf64))

    def build_vkb(self, ik, stream=None):
        """getvnl on the device for k-point ik (replaces any set_vkb of that k-point)."""
        call("b200_hamilt_build_vkb", self._h, ik, stream_ptr(stream))

    def copy_vkb(self, ik, out, stream=None):
        call("b200_hamilt_copy_vkb", self._h, ik, ptr(out), stream_ptr(stream))

    def _kbatch_args(self, iks, psis, hpsis, nbands, ld):
        nk = len(iks)
        if len(psis) != nk or len(hpsis) != nk:
            raise ValueError("iks, psis and hpsis must have the same length")
        for p, hp in zip(psis, hpsis):
            self._chk(p, hp, nbands, ld)
        return (nk, (C.c_int * nk)(*[int(i) for i in iks]), (_lib.vp * nk)(*[ptr(p) for p in psis]),
                (_lib.vp * nk)(*[ptr(p) for p in hpsis]))

    def hpsi_kbatch(self, iks, psis, hpsis, nbands, ld, spin=0, stream=None):
        """H|psi> of nbands bands for each k-point in iks (psis[q], hpsis[q]: that k-point's blocks); the
        kinetic + local part of all k-points in one launch per FFT pass."""
        nk, ik_a, p_a, h_a = self._kbatch_args(iks, psis, hpsis, nbands, ld)
        call("b200_hamilt_hpsi_kbatch", self._h, nk, ik_a, spin, nbands, ld, p_a, h_a, stream_ptr(stream))

    def capture_hpsi_kbatch(self, iks, psis, hpsis, nbands, ld, stream, spin=0):
        """hpsi_kbatch captured into a CUDA graph on a non-default stream; returns a HpsiGraph whose
        launch() replays it on the captured buffers."""
        nk, ik_a, p_a, h_a = self._kbatch_args(iks, psis, hpsis, nbands, ld)
        g = _lib.vp()
        call("b200_graph_capture_hpsi_kbatch", self._h, nk, ik_a, spin, nbands, ld, p_a, h_a, stream_ptr(stream),
             C.byref(g))
        return HpsiGraph(g, keep=(self, list(psis), list(hpsis)))

    def autotune(self, ik, psi, hpsi, nbands, ld, stream=None, with_variant=False):
        """Pick the band-chunk size and plane-pass variant of the local pass by timing candidates; returns the
        chosen chunk size (and the variant with with_variant=True)."""
        self._chk(psi, hpsi, nbands, ld)
        best, var = C.c_int(), C.c_int()
        call("b200_hamilt_autotune", self._h, ik, nbands, ld, ptr(psi), ptr(hpsi), stream_ptr(stream), C.byref(best),
             C.byref(var))
        return (best.value, var.value) if with_variant else best.value

    def set_chunk(self, chunk):
        """Bands per stick-buffer chunk of the local pass (0: the 48 MB default rule)."""
        call("b200_hamilt_set_band_chunk", self._h, int(chunk))

    def set_plane_variant(self, variant):
        """Plane pass of the register transforms (1: warp-shuffle lanes; 2-5: two-pass transforms; 0: default)
        for every handle of this basis in this handle's precision."""
        call("b200_hamilt_set_plane_variant", self._h, int(variant))

    def set_fp64_gemm(self, mode, nmods=16):
        """FP64 projector products: 0 cuBLAS ZGEMM; int8 tensor cores (exact modular emulation with nmods
        moduli) for calls of at least 48 bands (1, the default) or always (2).  Rebuilds the residue forms."""
        call("b200_hamilt_set_fp64_gemm", self._h, int(mode), int(nmods))

    def solve_kpoints(self, iks, precond_ds, psis, ld_psi, nband, thr, maxiter, david_ndim=4, precision=PREC_FP64,
                      nworkers=4, ntry_max=5, notconv_max=0, spin=0):
        """Davidson solves of the k-points iks, nworkers at a time on separate streams.  psis[q] (complex128,
        nband x ld_psi) is overwritten with the eigenvectors.  Returns (eigenvalues nk x nband, iterations)."""
        nk = len(iks)
        for p in psis:
            _check_block(p, True, nband, ld_psi, "psi")
        ik_a = (C.c_int * nk)(*[int(i) for i in iks])
        pc_a = (_lib.vp * nk)(*[ptr(p) for p in precond_ds])
        ps_a = (_lib.vp * nk)(*[ptr(p) for p in psis])
        eig = np.zeros((nk, nband))
        its = np.zeros(nk, dtype=np.int32)
        call("b200_solve_kpoints", self._h, nk, ik_a, spin, nband, david_ndim, precision,
             C.cast(pc_a, C.POINTER(_lib.vp)), ps_a, ld_psi, eig.ctypes.data_as(_lib.pf64), thr, maxiter, ntry_max,
             notconv_max, nworkers, its.ctypes.data_as(_lib.pi32))
        return eig, its

    def solve_kpoints_batched(self, iks, precond_ds, psis, ld_psi, nband, thr, maxiter, david_ndim=4, spin=0,
                              precision=PREC_FP64, stream=None):
        """Davidson of the k-points iks in lock-step (one batched call per phase for all k; FP64, or mixed: an FP32
        stage to 1e-7 refined in FP64).  psis[q]
        (complex128, nband x ld_psi, ld_psi >= the largest npw of the batch) is overwritten with the
        eigenvectors.  Returns (eigenvalues nk x nband, iteration after which each k-point had converged)."""
        nk = len(iks)
        for p in psis:
            _check_block(p, True, nband, ld_psi, "psi")
        ik_a = (C.c_int * nk)(*[int(i) for i in iks])
        pc_a = (_lib.vp * nk)(*[ptr(p) for p in precond_ds])
        ps_a = (_lib.vp * nk)(*[ptr(p) for p in psis])
        eig = np.zeros((nk, nband))
        its = np.zeros(nk, dtype=np.int32)
        call("b200_solve_kpoints_batched", self._h, nk, ik_a, spin, nband, david_ndim, precision,
             C.cast(pc_a, C.POINTER(_lib.vp)),
             C.cast(ps_a, C.POINTER(_lib.vp)), ld_psi, eig.ctypes.data_as(_lib.pf64), thr, maxiter,
             its.ctypes.data_as(_lib.pi32), stream_ptr(stream))
        return eig, its

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.b200_hamilt_destroy(self._h)
                self._h = None
        except Exception:
            pass


class HpsiGraph:
    """An instantiated CUDA graph of a captured H|psi> call (keeps its Hamiltonian and buffers alive)."""

    def __init__(self, handle, keep):
        self._h = handle
        self._keep = keep
        self._lib = _lib.load()

    def launch(self, stream=None):
        call("b200_graph_launch", self._h, stream_ptr(stream))

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.b200_graph_destroy(self._h)
                self._h = None
        except Exception:
            pass


# ------------------------------------------------------------------ Davidson
class DiagoDavid:
    """hsolver::DiagoDavid<T, DEVICE_GPU> (diago_david.h:19-84); S = I."""

    def __init__(self, precondition_d, nband, dim, david_ndim=4, precision=PREC_FP64):
        h = _lib.vp()
        call("b200_david_create", nband, dim, david_ndim, precision, ptr(precondition_d), C.byref(h))
        self._h = h
        self._lib = _lib.load()
        self.nband = nband
        self.dim = dim

    def diag(self, hpsi_func, ld_psi, psi, eigenvalue, thr, maxiter, ntry_max=5, notconv_max=0):
        """hpsi_func(x_ptr, hx_ptr, nvec, dim, id_start, id_end) with raw device pointers (HPsiFunc contract).
        eigenvalue: numpy float64 array of nband, filled on return. Returns the iteration count."""

        _check_block(psi, True, self.nband, ld_psi, "psi")
        if len(eigenvalue) < self.nband or eigenvalue.dtype != np.float64:
            raise ValueError("eigenvalue: need a float64 array of nband entries")
        cb = _lib.HostCallback(hpsi_func)
        it = C.c_int()
        cb.call_with("b200_david_diag", self._h, cb.cfn, None, ld_psi, ptr(psi), eigenvalue.ctypes.data_as(_lib.pf64), thr, maxiter,
             ntry_max, notconv_max, C.byref(it))
        return it.value

    def diag_hamilt(self, hamilt: HamiltPW, ik, ld_psi, psi, eigenvalue, thr, maxiter, ntry_max=5, notconv_max=0,
                    spin=0):
        _check_block(psi, True, self.nband, ld_psi, "psi")
        if len(eigenvalue) < self.nband or eigenvalue.dtype != np.float64:
            raise ValueError("eigenvalue: need a float64 array of nband entries")
        it = C.c_int()
        call("b200_david_diag_hamilt", self._h, hamilt.handle, ik, spin, ld_psi, ptr(psi),
             eigenvalue.ctypes.data_as(_lib.pf64), thr, maxiter, ntry_max, notconv_max, C.byref(it))
        return it.value

    def set_stream(self, stream):
        """Run the solver's work on a torch.cuda.Stream (or raw stream pointer)."""
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        call("b200_david_set_stream", self._h, sp)

    def set_verbosity(self, level):
        call("b200_david_set_verbosity", self._h, int(level))

    def set_mixed_threshold(self, thr):
        call("b200_david_set_mixed_threshold", self._h, float(thr))

    def set_fp64_gemm(self, mode):
        """FP64 subspace products: 0 cuBLAS ZGEMM, 1 int8 tensor-core emulation in a mixed solve's FP64
        refinement, 2 in every FP64 iteration (1, 2: on the shapes where it is faster), 3 for every product."""
        call("b200_david_set_fp64_gemm", self._h, int(mode))

    def set_low_ndim(self, ndim):
        """Mixed precision: david_ndim of the FP32 stage (smaller subspace, smaller FP64 eigensolves)."""
        call("b200_david_set_low_ndim", self._h, int(ndim))

    def set_trace(self, on=True):
        """Record per-iteration eigenvalues and times of the next solves (see trace())."""
        call("b200_david_set_trace", self._h, int(bool(on)))

    def trace(self):
        """(t seconds since the solve began, stage 0 = FP64 / 1 = FP32, eigenvalues iters x nband) of the last
        solve, one row per Davidson iteration (the initial Rayleigh-Ritz included)."""
        n = C.c_int()
        call("b200_david_trace", self._h, 0, self.nband, None, None, None, C.byref(n))
        m = n.value
        t = np.zeros(max(m, 1))
        st = np.zeros(max(m, 1), dtype=np.int32)
        e = np.zeros((max(m, 1), self.nband))
        call("b200_david_trace", self._h, m, self.nband, t.ctypes.data_as(_lib.pf64), st.ctypes.data_as(_lib.pi32),
             e.ctypes.data_as(_lib.pf64), C.byref(n))
        return t[:m], st[:m], e[:m]

    def stats(self):
        """(iterations in the FP32 stage, iterations in FP64, single-band H applications) of the last solve."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        call("b200_david_stats", self._h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.b200_david_destroy(self._h)
                self._h = None
        except Exception:
            pass


class DiagoDavSubspace:
    """hsolver::Diago_DavSubspace<T, DEVICE_GPU> (diago_dav_subspace.h:20-40), FP64, one rank.

    precondition_d: device float64 array of dim (HSolverPW passes |k+G|^2 tpiba2 for this method)."""

    def __init__(self, precondition_d, nband, dim, david_ndim, diag_thr, diag_nmax, need_subspace=False):
        h = _lib.vp()
        call("b200_dav_subspace_create", nband, dim, david_ndim, float(diag_thr), int(diag_nmax),
             int(bool(need_subspace)), ptr(precondition_d), C.byref(h))
        self._h = h
        self._lib = _lib.load()
        self.nband = nband
        self.dim = dim

    def _args(self, psi, psi_in_dmax, eigenvalue, is_occupied):
        _check_block(psi, True, self.nband, psi_in_dmax, "psi")
        if len(eigenvalue) < self.nband or eigenvalue.dtype != np.float64:
            raise ValueError("eigenvalue: need a float64 array of nband entries")
        occ = None
        if is_occupied is not None:
            occ = np.ascontiguousarray(np.asarray(is_occupied, dtype=bool).astype(np.int32))
            if len(occ) < self.nband:
                raise ValueError("is_occupied: need nband flags")
        return occ, (occ.ctypes.data_as(_lib.pi32) if occ is not None else None)

    def diag(self, hpsi_func, psi, psi_in_dmax, eigenvalue, is_occupied=None, scf_type=False):
        """hpsi_func(x_ptr, hx_ptr, nvec, dim, id_start, id_end) with raw device pointers (HPsiFunc contract).
        eigenvalue: numpy float64 array of nband (in: ignored; out: the eigenvalues).  Returns the total
        iteration count."""

        occ, occ_p = self._args(psi, psi_in_dmax, eigenvalue, is_occupied)
        cb = _lib.HostCallback(hpsi_func)
        it = C.c_int()
        cb.call_with("b200_dav_subspace_diag", self._h, cb.cfn, None, ptr(psi), psi_in_dmax,
             eigenvalue.ctypes.data_as(_lib.pf64), occ_p, int(bool(scf_type)), C.byref(it))
        return it.value

    def diag_hamilt(self, hamilt: HamiltPW, ik, psi, psi_in_dmax, eigenvalue, is_occupied=None, scf_type=False,
                    spin=0):
        occ, occ_p = self._args(psi, psi_in_dmax, eigenvalue, is_occupied)
        it = C.c_int()
        call("b200_dav_subspace_diag_hamilt", self._h, hamilt.handle, ik, spin, ptr(psi), psi_in_dmax,
             eigenvalue.ctypes.data_as(_lib.pf64), occ_p, int(bool(scf_type)), C.byref(it))
        return it.value

    def set_stream(self, stream):
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        call("b200_dav_subspace_set_stream", self._h, sp)

    def set_verbosity(self, level):
        call("b200_dav_subspace_set_verbosity", self._h, int(level))

    def stats(self):
        """(unconverged bands, single-band H applications) of the last solve."""
        a, b = C.c_int(), C.c_int()
        call("b200_dav_subspace_stats", self._h, C.byref(a), C.byref(b))
        return a.value, b.value

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.b200_dav_subspace_destroy(self._h)
                self._h = None
        except Exception:
            pass


class DiagoBPCG:
    """hsolver::DiagoBPCG<T, DEVICE_GPU> (diago_bpcg.h:18-337), FP64, one rank: the constructor and
    init_iter(psi) in one (nband, nbasis).  precondition_d: device float64 array of nbasis."""

    def __init__(self, precondition_d, nband, nbasis):
        h = _lib.vp()
        call("b200_bpcg_create", ptr(precondition_d), nband, nbasis, C.byref(h))
        self._h = h
        self._lib = _lib.load()
        self.nband = nband
        self.nbasis = nbasis

    def _check(self, psi, eigenvalue):
        _check_block(psi, True, self.nband, self.nbasis, "psi")
        if len(eigenvalue) < self.nband or eigenvalue.dtype != np.float64:
            raise ValueError("eigenvalue: need a float64 array of nband entries")

    def diag(self, hpsi_func, psi, eigenvalue, scf_iter=1):
        """hpsi_func(x_ptr, hx_ptr, nvec, dim, id_start, id_end) with raw device pointers (HPsiFunc contract),
        called for all bands.  scf_iter: DiagoIterAssist::SCF_ITER.  Returns the CG iterations."""

        self._check(psi, eigenvalue)
        cb = _lib.HostCallback(hpsi_func)
        it = C.c_int()
        cb.call_with("b200_bpcg_diag", self._h, cb.cfn, None, ptr(psi), eigenvalue.ctypes.data_as(_lib.pf64), int(scf_iter),
             C.byref(it))
        return it.value

    def diag_hamilt(self, hamilt: HamiltPW, ik, psi, eigenvalue, scf_iter=1, spin=0):
        self._check(psi, eigenvalue)
        it = C.c_int()
        call("b200_bpcg_diag_hamilt", self._h, hamilt.handle, ik, spin, ptr(psi),
             eigenvalue.ctypes.data_as(_lib.pf64), int(scf_iter), C.byref(it))
        return it.value

    def set_stream(self, stream):
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        call("b200_bpcg_set_stream", self._h, sp)

    def stats(self):
        """(largest residual norm of the last iteration, single-band H applications) of the last diag."""
        e, n = C.c_double(), C.c_int()
        call("b200_bpcg_stats", self._h, C.byref(e), C.byref(n))
        return e.value, n.value

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.b200_bpcg_destroy(self._h)
                self._h = None
        except Exception:
            pass


# ------------------------------------------------------------------ workloads
@dataclass
class Workload:
    spec: object
    cell: object
    basis: PWBasisK
    veff_h: np.ndarray          # host V_eff (reference r order)
    vkb_h: list                 # per k: (nkb, npwx) complex128
    deeq_h: np.ndarray
    psi0_h: list                # per k: (nbands, npwx) complex128

    @property
    def nkb(self):
        return self.cell.nkb


def build_workload(spec, kpts=None) -> Workload:
    """Synthetic cell + basis + host inputs for a CellSpec (see synth.py)."""
    from . import synth
    cell = synth.make_cell(spec)
    k = spec.kpts if kpts is None else kpts
    if k is None:
        k = np.zeros((1, 3))
    basis = PWBasisK(spec.a, cell.latvec, spec.ecut, k, grid=spec.grid)
    veff = cell.veff(basis.nx, basis.ny, basis.nz)
    npwx = basis.npwk_max
    vkbs, psis = [], []
    for ik in range(basis.nks):
        q = basis.gplusk_cart(ik)
        vkbs.append(cell.vkb(q, npwx, basis.omega))
        psis.append(cell.psi0(q, spec.nbands, npwx, seed_offset=ik))
    return Workload(spec, cell, basis, veff, vkbs, cell.deeq(), psis)


def device_hamilt(wl: Workload, precision=PREC_FP64) -> HamiltPW:
    torch = _torch()
    h = HamiltPW(wl.basis, precision)
    h._veff_d = torch.from_numpy(wl.veff_h).cuda()
    h.set_veff(h._veff_d)
    h._deeq_d = torch.from_numpy(wl.deeq_h).cuda()
    h.set_deeq([wl.cell.nat], [8], h._deeq_d)
    for ik, v in enumerate(wl.vkb_h):
        vd = torch.from_numpy(v).cuda()
        h.set_vkb(ik, vd)
    torch.cuda.synchronize()
    return h


def precondition_dav_subspace_d(basis: PWBasisK, ik: int):
    """h_diag = |k+G|^2 tpiba2, the preconditioner HSolverPW gives Diago_DavSubspace (hsolver_pw.cpp:573-580),
    as a device FP64 tensor."""
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(basis.gk2_k(ik) * basis.tpiba2)).cuda()


def precondition_d(basis: PWBasisK, ik: int):
    """h_diag = 1 + g2 + sqrt(1 + (g2-1)^2) (hsolver_pw.cpp:567-584) as a device FP64 tensor."""
    torch = _torch()
    g2 = basis.gk2_k(ik) * basis.tpiba2
    return torch.from_numpy(1.0 + g2 + np.sqrt(1.0 + (g2 - 1.0) ** 2)).cuda()
