"""Oracle (test infrastructure only): CPU restatement of psi -> rho.

Only the tests and the benchmark's CPU baseline use this module; the product never imports it.

Follows ``elecstate_pw_op<CPU>`` (module_elecstate/kernels/elecstate_op.cpp:6-83, both overloads) and the
collinear band loop of ``ElecStatePW::psiToRho`` (module_elecstate/elecstate_pw.cpp:199-216): for every band
with a non-zero weight, recip_to_real of the band into the box, then rho[spin][r] += w1 * |psi(r)|^2.
Pinned against the reference's literals (tests/golden/elecstate_op.npz).
"""
from __future__ import annotations

import numpy as np

from .hamilt_ref import recip_to_real


def elecstate_pw_op(spin, nrxx, w1, rho, wfcr):
    """rho: list of per-spin float arrays, updated in place."""
    wfcr = np.asarray(wfcr)[:nrxx]
    rho[spin][:nrxx] += w1 * (wfcr.real ** 2 + wfcr.imag ** 2)


def elecstate_pw_op_nc(domag, domag_z, nrxx, w1, rho, a, b):
    a = np.asarray(a)[:nrxx]
    b = np.asarray(b)[:nrxx]
    na = a.real ** 2 + a.imag ** 2
    nb = b.real ** 2 + b.imag ** 2
    rho[0][:nrxx] += w1 * (na + nb)
    if domag:
        rho[1][:nrxx] += w1 * 2.0 * (a.real * b.real + a.imag * b.imag)
        rho[2][:nrxx] += w1 * 2.0 * (a.real * b.imag - b.real * a.imag)
        rho[3][:nrxx] += w1 * (na - nb)
    elif domag_z:
        rho[1][:nrxx] = 0.0
        rho[2][:nrxx] = 0.0
        rho[3][:nrxx] += w1 * (na - nb)
    else:
        for i in (1, 2, 3):
            rho[i][:nrxx] = 0.0


def psi_to_rho(basis, ik, psi, nbands, ld, w1, rho):
    """The collinear band loop; psi band ib at psi[ib*ld:], rho (N,) float64 accumulated in place."""
    npw = int(basis.npwk[ik])
    for ib in range(nbands):
        if w1[ib] == 0.0:
            continue
        box = recip_to_real(basis, np.asarray(psi)[ib * ld: ib * ld + npw], ik)
        elecstate_pw_op(0, len(rho), w1[ib], [rho], box)
    return rho
