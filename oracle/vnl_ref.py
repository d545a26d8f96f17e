"""Oracle (test infrastructure only): CPU restatement of the reference's projector generation.

Only the tests and the benchmark's CPU baseline use this module; the product never imports it.

Follows, step for step:
  * ``cal_ylm_real_op<CPU>`` (module_base/kernels/math_op.cpp:27-130): real spherical harmonics by the
    Legendre recursion on l, order per l: m = 0, then (cos, sin) pairs for m = 1..l;
  * ``_polynomial_interpolation`` (module_hamilt_pw/hamilt_pwdft/kernels/vnl_tools.hpp:6-28): 4-point
    Lagrange interpolation of the radial table at |k+G| * tpiba;
  * ``cal_sk_op<CPU>`` (module_hamilt_pw/hamilt_pwdft/kernels/wf_op.cpp:6-77): structure factor
    e^{-i k.tau} * eigts1[ix] * eigts2[iy] * eigts3[iz];
  * ``cal_vnl_op<CPU>`` (module_hamilt_pw/hamilt_pwdft/kernels/vnl_op.cpp:8-108): vkb rows ordered by
    type, atom, ih, each = Ylm(lm(ih)) * vq(indv(ih)) * sk(atom) * (-i)^l(ih);
  * ``pseudopot_cell_vnl::getvnl`` (module_hamilt_pw/hamilt_pwdft/VNL_in_pw.cpp:412-540): the
    composition of the three for one k-point.

Pinned against the reference's own literals (tests/golden/{ylm_op,wf_op,vnl_op}.npz).
"""
from __future__ import annotations

import math

import numpy as np

_PREF = np.array([1.0 + 0.0j, -1.0j, -1.0 + 0.0j, 1.0j])  # (-i)^n for n mod 4


def _fact(n: int) -> float:
    f = 1.0
    for i in range(n, 1, -1):
        f *= i
    return f


def _semi_fact(n: int) -> int:
    f = 1
    for i in range(n, 2, -2):
        f *= i
    return f


def ylm_real(lmax: int, g: np.ndarray) -> np.ndarray:
    """cal_ylm_real_op: g (ng, 3) -> ylm ((lmax+1)^2, ng)."""
    g = np.asarray(g, dtype=np.float64).reshape(-1, 3)
    ng = len(g)
    nlm = (lmax + 1) ** 2
    ylm = np.zeros((nlm, ng))
    if lmax == 0:
        ylm[0] = 1.0 / math.sqrt(4.0 * math.pi)
        return ylm
    gx, gy, gz = g[:, 0], g[:, 1], g[:, 2]
    gmod = np.sqrt(gx * gx + gy * gy + gz * gz)
    cost = np.where(gmod < 1.0e-9, 0.0, gz / np.where(gmod < 1.0e-9, 1.0, gmod))
    with np.errstate(divide="ignore", invalid="ignore"):
        at = np.arctan(gy / gx)
    phi = np.where(gx > 1.0e-9, at, np.where(gx < -1.0e-9, at + math.pi, (math.pi / 2) * np.where(gy >= 0.0, 1.0, -1.0)))
    p = np.zeros((lmax + 1, lmax + 1, ng))  # p[m, l]
    lm = -1
    for l in range(lmax + 1):
        c = math.sqrt((2 * l + 1) / (4.0 * math.pi))
        if l == 0:
            p[0, 0] = 1.0
        elif l == 1:
            p[0, 1] = cost
            p[1, 1] = -np.sqrt(np.maximum(0.0, 1.0 - cost * cost))
        else:
            l1, l2, l3 = l - 1, l - 2, 2 * l - 1
            for m in range(l2 + 1):
                p[m, l] = (cost * l3 * p[m, l1] - (l1 + m) * p[m, l2]) / (l - m)
            p[l1, l] = cost * l3 * p[l1, l1]
            x2 = np.maximum(0.0, 1.0 - cost * cost)
            p[l, l] = _semi_fact(l3) * x2 ** (l / 2.0)
            if l % 2 == 1:
                p[l, l] *= -1
        lm += 1
        ylm[lm] = c * p[0, l]
        for m in range(1, l + 1):
            same = c * math.sqrt(_fact(l - m) / _fact(l + m)) * math.sqrt(2.0)
            lm += 1
            ylm[lm] = same * p[m, l] * np.cos(m * phi)
            lm += 1
            ylm[lm] = same * p[m, l] * np.sin(m * phi)
    return ylm


def interp(table: np.ndarray, it: int, ib: int, tab_2: int, tab_3: int, dq: float, x: np.ndarray) -> np.ndarray:
    """_polynomial_interpolation on a flat (ntype, tab_2, tab_3) table."""
    pos = x / dq
    iq = pos.astype(np.int64)
    x0 = pos - iq
    x1, x2, x3 = 1.0 - x0, 2.0 - x0, 3.0 - x0
    base = (it * tab_2 + ib) * tab_3 + iq
    t = table
    return (t[base] * x1 * x2 * x3 / 6.0 + t[base + 1] * x0 * x2 * x3 / 2.0 - t[base + 2] * x1 * x0 * x3 / 2.0
            + t[base + 3] * x1 * x2 * x0 / 6.0)


def cal_sk(ik, ntype, nx, ny, nz, rho_nx, rho_ny, rho_nz, npw, npwx, fftny, e1nc, e2nc, e3nc, atom_na, igl2isz,
           is2fftixy, two_pi, kvec_c, atom_tau, eigts1, eigts2, eigts3) -> np.ndarray:
    """cal_sk_op: sk (nat, npw)."""
    nat = int(np.sum(atom_na))
    sk = np.zeros((nat, npw), dtype=np.complex128)
    isz = np.asarray(igl2isz[ik * npwx: ik * npwx + npw], dtype=np.int64)
    iz = isz % nz
    ixy = np.asarray(is2fftixy)[isz // nz]
    ix, iy = ixy // fftny, ixy % fftny
    ix = np.where(ix >= nx // 2 + 1, ix - nx, ix) + rho_nx
    iy = np.where(iy >= ny // 2 + 1, iy - ny, iy) + rho_ny
    iz = np.where(iz >= nz // 2 + 1, iz - nz, iz) + rho_nz
    iat = 0
    for it in range(ntype):
        for _ in range(atom_na[it]):
            arg = two_pi * sum(kvec_c[ik * 3 + i] * atom_tau[iat * 3 + i] for i in range(3))
            kph = complex(math.cos(arg), -math.sin(arg))
            sk[iat] = kph * eigts1[iat * e1nc + ix] * eigts2[iat * e2nc + iy] * eigts3[iat * e3nc + iz]
            iat += 1
    return sk


def cal_vnl(ntype, npw, npwx, nhm, tab_2, tab_3, atom_na, atom_nb, atom_nh, dq, tpiba, gk, ylm, indv, nhtol,
            nhtolm, tab, sk) -> np.ndarray:
    """cal_vnl_op: vkb (nkb, npwx) complex128, rows beyond npw zero.

    gk (npw, 3) in 2pi/a units; ylm ((lmax+1)^2, npw); indv/nhtol/nhtolm (ntype, nhm); tab flat
    (ntype, tab_2, tab_3); sk (nat, npw)."""
    gk = np.asarray(gk, dtype=np.float64).reshape(-1, 3)[:npw]
    indv = np.asarray(indv).reshape(ntype, nhm)
    nhtol = np.asarray(nhtol).reshape(ntype, nhm)
    nhtolm = np.asarray(nhtolm).reshape(ntype, nhm)
    ylm = np.asarray(ylm).reshape(-1, npw)
    sk = np.asarray(sk).reshape(-1, npw)
    table = np.asarray(tab).reshape(-1)
    nkb = int(sum(atom_na[it] * atom_nh[it] for it in range(ntype)))
    vkb = np.zeros((nkb, npwx), dtype=np.complex128)
    gnorm = np.sqrt(np.sum(gk * gk, axis=1)) * tpiba
    jkb = iat = 0
    for it in range(ntype):
        nh = atom_nh[it]
        vkb1 = np.zeros((nh, npw))
        for ib in range(atom_nb[it]):
            vq = interp(table, it, ib, tab_2, tab_3, dq, gnorm)
            for ih in range(nh):
                if ib == indv[it, ih]:
                    vkb1[ih] = ylm[int(nhtolm[it, ih])] * vq
        for _ in range(atom_na[it]):
            for ih in range(nh):
                pref = _PREF[int(nhtol[it, ih]) % 4]
                vkb[jkb, :npw] = vkb1[ih] * sk[iat] * pref
                jkb += 1
            iat += 1
    return vkb


def getvnl(basis, ik: int, proj, tau_lat0: np.ndarray) -> np.ndarray:
    """getvnl for k-point ik of a PW_Basis_K-like basis (``gplusk_cart`` in bohr^-1, ``tpiba2``, ``npwk_max``);
    ``proj`` carries the projector tables (ntype, na, nbeta, nh, nhm, lmax, indv, nhtol, nhtolm, tab, dq).

    The structure factor is e^{-i 2 pi (k+G).tau} with tau in lat0 units (the value cal_sk_op assembles from
    its per-axis phase tables)."""
    q = basis.gplusk_cart(ik)                      # bohr^-1
    tpiba = math.sqrt(basis.tpiba2)
    gk = q / tpiba                                  # 2pi/a units, as PW_Basis_K::getgpluskcar
    npw = len(gk)
    ylm = ylm_real(proj.lmax, gk)
    sk = np.exp(-2j * math.pi * (gk @ np.asarray(tau_lat0, dtype=np.float64).T)).T  # (nat, npw)
    tab = np.asarray(proj.tab)
    return cal_vnl(proj.ntype, npw, basis.npwk_max, proj.nhm, tab.shape[1], tab.shape[2], proj.na, proj.nbeta,
                   proj.nh, proj.dq, tpiba, gk, ylm, proj.indv, proj.nhtol, proj.nhtolm, tab, sk)
