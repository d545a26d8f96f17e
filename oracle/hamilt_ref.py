"""CPU oracle (test infrastructure only): the plane-wave H|psi> of ABACUS.

numpy restatement of the reference's CPU op functors and of the operator
chain that composes them.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` use it, as the checker.

Followed reference code (abacus-develop v3.8.0):
  * ekinetic_pw_op<CPU> ....... source/module_hamilt_pw/hamilt_pwdft/kernels/ekinetic_op.cpp:6-24
  * veff_pw_op<CPU> ........... source/module_hamilt_pw/hamilt_pwdft/kernels/veff_op.cpp:6-40
  * nonlocal_pw_op<CPU> ....... source/module_hamilt_pw/hamilt_pwdft/kernels/nonlocal_op.cpp:6-78
  * pw_op functors ............ source/module_basis/module_pw/kernels/pw_op.cpp:6-68
  * recip_to_real/real_to_recip source/module_basis/module_pw/pw_transform_k.cpp:336-476
    (FFTW/cuFFT convention: backward = exp(+iGr) un-normalised, forward =
    exp(-iGr), the 1/N applied at the gather) -- scipy's pocketfft has the
    same convention (fftn = forward, ifftn * N = backward).
  * Veff::act ................. source/module_hamilt_pw/hamilt_pwdft/operator_pw/veff_pw.cpp:38-109
                                (npol = 2 branch :73-104 in HamiltPWRefNC)
  * Ekinetic::act ............. source/module_hamilt_pw/hamilt_pwdft/operator_pw/ekinetic_pw.cpp:34-50
  * Nonlocal::act / add_nonlocal_pp
                                source/module_hamilt_pw/hamilt_pwdft/operator_pw/nonlocal_pw.cpp:64-283
  * Operator::hPsi (zero hpsi, then chain) source/module_hamilt_general/operator.cpp:39-88,134-167
  * update_precondition ....... source/module_hsolver/hsolver_pw.cpp:550-593
"""
from __future__ import annotations

import numpy as np
import scipy.fft

# threads for the oracle's FFTs (scipy's pocketfft; 1 = single thread)
FFT_WORKERS = 1


# ---------------------------------------------------------------- functors
def ekinetic_pw_op(nband, npw, max_npw, tpiba2, gk2, hpsi, psi):
    """hpsi[ib*max_npw + ig] += gk2[ig]*tpiba2*psi[...] (ekinetic_op.cpp:16-23). In place on hpsi."""
    for ib in range(nband):
        s = ib * max_npw
        hpsi[s:s + npw] += gk2[:npw] * tpiba2 * psi[s:s + npw]


def veff_pw_op(size, out, vin):
    """out[ir] *= in[ir] (veff_op.cpp:8-18). In place."""
    out[:size] *= vin[:size]


def veff_pw_op_npol2(size, out, out1, vin4):
    """2x2 spin form (veff_op.cpp:20-37). vin4 = 4 real arrays. In place on out, out1."""
    v0, v1, v2, v3 = (np.asarray(v)[:size] for v in vin4)
    a = out[:size].copy()
    b = out1[:size].copy()
    sup = a * (v0 + v3) + b * (v1 - 1j * v2)
    sdown = b * (v0 - v3) + a * (v1 + 1j * v2)
    out[:size] = sup
    out1[:size] = sdown


def nonlocal_pw_op(l1, l2, l3, sum_, iat, spin, nkb, deeq_x, deeq_y, deeq_z, deeq, ps, becp):
    """ps[(sum+ii*l3+kk)*l2+jj] += deeq[((spin*dx+iat+ii)*dy+xx)*dz+kk]*becp[jj*nkb+sum+ii*l3+xx]
    (nonlocal_op.cpp:8-41). Returns the updated (sum, iat)."""
    deeq = np.asarray(deeq).reshape(-1)
    for ii in range(l1):
        # D block (xx, kk) for this atom
        base = ((spin * deeq_x + iat + ii) * deeq_y) * deeq_z
        dblk = deeq[base: base + deeq_y * deeq_z].reshape(deeq_y, deeq_z)[:l3, :l3]
        for jj in range(l2):
            b = becp[jj * nkb + sum_ + ii * l3: jj * nkb + sum_ + ii * l3 + l3]
            contrib = dblk.T @ b  # sum_xx D[xx,kk] * becp[xx]
            for kk in range(l3):
                ps[(sum_ + ii * l3 + kk) * l2 + jj] += contrib[kk]
    return sum_ + l1 * l3, iat + l1


def nonlocal_pw_op_nc(l1, l2, l3, sum_, iat, nkb, deeq_x, deeq_y, deeq_z, deeq_nc, ps, becp):
    """Non-collinear form (nonlocal_op.cpp:43-74). Returns the updated (sum, iat)."""
    dnc = np.asarray(deeq_nc).reshape(-1)

    def d(s, ia, kk, xx):
        return dnc[((s * deeq_x + ia) * deeq_y + kk) * deeq_z + xx]

    for ii in range(l1):
        for jj in range(0, l2, 2):
            for kk in range(l3):
                for xx in range(l3):
                    psind = (sum_ + ii * l3 + kk) * l2 + jj
                    becpind = jj * nkb + sum_ + ii * l3 + xx
                    b1 = becp[becpind]
                    b2 = becp[becpind + nkb]
                    ia = iat + ii
                    ps[psind] += d(0, ia, kk, xx) * b1 + d(1, ia, kk, xx) * b2
                    ps[psind + 1] += d(2, ia, kk, xx) * b1 + d(3, ia, kk, xx) * b2
    return sum_ + l1 * l3, iat + l1


def set_3d_fft_box_op(npwk, box_index, inp, out):
    out[np.asarray(box_index[:npwk])] = inp[:npwk]


def set_recip_to_real_output_op(nrxx, add, factor, inp, out):
    if add:
        out[:nrxx] += factor * inp[:nrxx]
    else:
        out[:nrxx] = inp[:nrxx]


def set_real_to_recip_output_op(npw_k, nxyz, add, factor, box_index, inp, out):
    idx = np.asarray(box_index[:npw_k])
    if add:
        out[:npw_k] += factor / nxyz * inp[idx]
    else:
        out[:npw_k] = inp[idx] / nxyz


# ---------------------------------------------------------------- transforms
def recip_to_real(basis, inp, ik, out=None, add=False, factor=1.0):
    """PW_Basis_K::recip_to_real (pw_transform_k.cpp:404-476): sphere -> full r box."""
    nx, ny, nz = basis.nx, basis.ny, basis.nz
    N = nx * ny * nz
    box = np.zeros(N, dtype=np.complex128)
    npw = int(basis.npwk[ik])
    set_3d_fft_box_op(npw, basis.ig2ixyz(ik), inp, box)
    r = scipy.fft.ifftn(box.reshape(nx, ny, nz), workers=FFT_WORKERS).reshape(-1) * N
    if out is None:
        out = np.zeros(N, dtype=np.complex128)
    set_recip_to_real_output_op(N, add, factor, r, out)
    return out


def real_to_recip(basis, inp, ik, out=None, add=False, factor=1.0):
    """PW_Basis_K::real_to_recip (pw_transform_k.cpp:336-401): full r box -> sphere."""
    nx, ny, nz = basis.nx, basis.ny, basis.nz
    N = nx * ny * nz
    g = scipy.fft.fftn(np.asarray(inp, dtype=np.complex128).reshape(nx, ny, nz), workers=FFT_WORKERS).reshape(-1)
    npw = int(basis.npwk[ik])
    if out is None:
        out = np.zeros(npw, dtype=np.complex128)
    set_real_to_recip_output_op(npw, N, add, factor, basis.ig2ixyz(ik), g, out)
    return out


# ---------------------------------------------------------------- operators
class HamiltPWRef:
    """Ekinetic -> Veff -> Nonlocal chain for one k-point, npol = 1, nspin = 1."""

    def __init__(self, basis, ik, veff, vkb, deeq, nh, natoms_per_type):
        self.basis = basis
        self.ik = ik
        self.veff = np.asarray(veff, dtype=np.float64)
        self.vkb = np.asarray(vkb)  # (nkb, npwx) row-major
        self.nkb = self.vkb.shape[0]
        self.npwx = self.vkb.shape[1]
        self.deeq = np.asarray(deeq)
        self.nh = nh  # per type
        self.na = natoms_per_type

    def ekinetic_act(self, nbands, nbasis, psi, hpsi):
        npw = int(self.basis.npwk[self.ik])
        ekinetic_pw_op(nbands, npw, nbasis, self.basis.tpiba2, self.basis.gk2_k(self.ik), hpsi, psi)

    def veff_act(self, nbands, nbasis, psi, hpsi):
        N = self.basis.nxyz
        npw = int(self.basis.npwk[self.ik])
        for ib in range(nbands):
            porter = recip_to_real(self.basis, psi[ib * nbasis: ib * nbasis + npw], self.ik)
            veff_pw_op(N, porter, self.veff)
            seg = hpsi[ib * nbasis: ib * nbasis + npw]
            real_to_recip(self.basis, porter, self.ik, out=seg, add=True)
            hpsi[ib * nbasis: ib * nbasis + npw] = seg

    def nonlocal_act(self, nbands, nbasis, psi, hpsi):
        npw = int(self.basis.npwk[self.ik])
        nkb = self.nkb
        V = self.vkb[:, :npw]  # (nkb, npw)
        P = np.stack([psi[ib * nbasis: ib * nbasis + npw] for ib in range(nbands)], 1)  # npw x nb
        becp = (V.conj() @ P).T.reshape(-1)  # gemm('C','N') column-major nkb x nb: becp[ib*nkb + j]
        ps = np.zeros(nkb * nbands, dtype=np.complex128)
        sum_, iat = 0, 0
        dx, dy, dz = self.deeq.shape[1], self.deeq.shape[2], self.deeq.shape[3]
        for it in range(len(self.na)):
            sum_, iat = nonlocal_pw_op(self.na[it], nbands, self.nh[it], sum_, iat, 0, nkb, dx, dy, dz,
                                       self.deeq, ps, becp)
        PS = ps.reshape(nkb, nbands)  # ps[j*nb + ib]
        add = V.T @ PS  # gemm('N','T'): npw x nb
        for ib in range(nbands):
            hpsi[ib * nbasis: ib * nbasis + npw] += add[:, ib]

    def hpsi(self, psi, nbands, nbasis):
        """Operator::hPsi: zero hpsi then Ekinetic, Veff, Nonlocal (operator.cpp:39-88, :165)."""
        hpsi = np.zeros(nbands * nbasis, dtype=np.complex128)
        psi = np.asarray(psi).reshape(-1)
        self.ekinetic_act(nbands, nbasis, psi, hpsi)
        self.veff_act(nbands, nbasis, psi, hpsi)
        self.nonlocal_act(nbands, nbasis, psi, hpsi)
        return hpsi

    def hpsi_local(self, psi, nbands, nbasis):
        hpsi = np.zeros(nbands * nbasis, dtype=np.complex128)
        psi = np.asarray(psi).reshape(-1)
        self.ekinetic_act(nbands, nbasis, psi, hpsi)
        self.veff_act(nbands, nbasis, psi, hpsi)
        return hpsi

    def dense(self):
        """The full npw x npw Hamiltonian matrix (small cases only)."""
        npw = int(self.basis.npwk[self.ik])
        eye = np.zeros(npw * npw, dtype=np.complex128)
        for i in range(npw):
            eye[i * npw + i] = 1.0
        h = self.hpsi(eye, npw, npw).reshape(npw, npw)  # row ib = H e_ib
        return h.T


class HamiltPWRefNC:
    """Ekinetic -> Veff -> Nonlocal chain with npol = 2 for one k-point: band b's spinor components are the
    columns 2b and 2b + 1 (pitch nbasis).  Ekinetic::act on every column (ekinetic_pw.cpp:34-50 with
    max_npw = nbasis), Veff::act's spinor branch (veff_pw.cpp:73-104: both components to real space,
    veff_pw_op's npol = 2 form, both back), Nonlocal::act with add_nonlocal_pp's spinor branch
    (nonlocal_pw.cpp:117-160, 211-283; nonlocal_pw_op's deeq_nc overload)."""

    def __init__(self, basis, ik, veff4, vkb, deeq_nc, nh, natoms_per_type):
        self.basis = basis
        self.ik = ik
        self.veff4 = [np.asarray(v, dtype=np.float64) for v in veff4]
        self.vkb = np.asarray(vkb)  # (nkb, npwx) row-major
        self.nkb = self.vkb.shape[0]
        self.deeq_nc = np.asarray(deeq_nc)  # (4, dx, dy, dz) complex
        self.nh = nh
        self.na = natoms_per_type

    def hpsi(self, psi, nbands, nbasis):
        """hpsi of nbands spinor bands (2 nbands columns of nbasis)."""
        ncol = 2 * nbands
        npw = int(self.basis.npwk[self.ik])
        N = self.basis.nxyz
        psi = np.asarray(psi).reshape(-1)
        hpsi = np.zeros(ncol * nbasis, dtype=np.complex128)
        ekinetic_pw_op(ncol, npw, nbasis, self.basis.tpiba2, self.basis.gk2_k(self.ik), hpsi, psi)
        for ib in range(nbands):
            up, dn = (2 * ib) * nbasis, (2 * ib + 1) * nbasis
            porter = recip_to_real(self.basis, psi[up: up + npw], self.ik)
            porter1 = recip_to_real(self.basis, psi[dn: dn + npw], self.ik)
            veff_pw_op_npol2(N, porter, porter1, self.veff4)
            for off, buf in ((up, porter), (dn, porter1)):
                seg = hpsi[off: off + npw]
                real_to_recip(self.basis, buf, self.ik, out=seg, add=True)
                hpsi[off: off + npw] = seg
        nkb = self.nkb
        if nkb:
            V = self.vkb[:, :npw]
            P = np.stack([psi[c * nbasis: c * nbasis + npw] for c in range(ncol)], 1)
            becp = (V.conj() @ P).T.reshape(-1)  # becp[c*nkb + j]
            ps = np.zeros(nkb * ncol, dtype=np.complex128)
            sum_, iat = 0, 0
            dx, dy, dz = self.deeq_nc.shape[1], self.deeq_nc.shape[2], self.deeq_nc.shape[3]
            for it in range(len(self.na)):
                sum_, iat = nonlocal_pw_op_nc(self.na[it], ncol, self.nh[it], sum_, iat, nkb, dx, dy, dz,
                                              self.deeq_nc, ps, becp)
            add = V.T @ ps.reshape(nkb, ncol)
            for c in range(ncol):
                hpsi[c * nbasis: c * nbasis + npw] += add[:, c]
        return hpsi


def precondition_dav_subspace(basis, ik):
    """h_diag = g2 = |k+G|^2 tpiba2, what update_precondition gives the "dav_subspace" method (hsolver_pw.cpp,
    update_precondition: the method's own preconditioner is applied in Diago_DavSubspace::cal_grad)."""
    return basis.gk2_k(ik) * basis.tpiba2


def precondition(basis, ik):
    """h_diag = 1 + g2 + sqrt(1 + (g2-1)^2), g2 = |k+G|^2 tpiba2 (hsolver_pw.cpp:567-584)."""
    g2 = basis.gk2_k(ik) * basis.tpiba2
    return 1.0 + g2 + np.sqrt(1.0 + (g2 - 1.0) ** 2)
