"""Oracle (test infrastructure only): numpy restatement of the reference's DiagoBPCG
(module_hsolver/diago_bpcg.cpp, the "bpcg" method of HSolverPW) with the CPU kernels it calls
(module_hsolver/kernels/math_kernel_op.cpp:10-100).  Pinned against the reference's own CPU solver compiled
from its sources (oracle/_ref, tests/test_bpcg.py).

One diag call (diago_bpcg.cpp:254-306):
* calc_hsub_with_block (:215-233): H psi, the Rayleigh-Ritz of psi (hsub = psi^H H psi, all pairs,
  upper triangle, zheevd), psi and H psi rotated to the Ritz vectors;
* grad_old = 0, beta = +inf; up to nline = 4 iterations (6 nline on the first SCF step, SCF_ITER == 1):
  - calc_grad_with_block (:109-131, kernel :51-100): per band, psi and H psi normalised, eps = <psi|H psi>,
    r = H psi - eps psi, err = |r|, beta = sum |r|^2 / prec, grad = -r / prec + beta / beta_old grad_old;
  - orth_projection (:139-156): grad -= psi (psi^H grad) over all bands;
  - grad_old = grad; H grad;
  - line_minimize_with_block (:75-83, kernel :10-48): per band, grad and H grad normalised,
    e0 = <psi|H psi>, e1 = Re <H psi|grad>, e2 = Re <H grad|grad>, theta = |atan(2 e1 / (e0 - e2))| / 2,
    psi <- cos(theta) psi + sin(theta) grad (and H psi alike);
  - orth_cholesky (:86-106): S = psi^H psi = U^H U (upper Cholesky), psi <- psi U^-1, H psi <- H psi U^-1;
  - on the first SCF step, every nline iterations calc_hsub_with_block again (H psi recomputed);
  - stop when no band has err > 1e-5 (test_error :56-69) or at the iteration limit;
* calc_hsub_with_block_exit (:235-250): the Rayleigh-Ritz again (H psi of the loop, not recomputed), psi
  rotated; the eigenvalues are its Ritz values.
Arrays are band-major (psi[m] is band m), as the reference's {n_band, n_basis} tensors.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg


class DiagoBPCGRef:
    nline = 4
    all_band_cg_thr = 1e-5

    def __init__(self, precondition, nband, nbasis):
        self.prec = np.asarray(precondition, dtype=np.float64)[:nbasis].copy()
        self.nband, self.nbasis = nband, nbasis
        self.err = np.zeros(nband)

    # ---------------------------------------------------------------- pieces
    @staticmethod
    def _rayleigh_ritz(psi, hpsi, rotate_h):
        # hsub(a, b) = <H psi_a | psi_b>, upper triangle read (lapack_dnevd 'V', 'U'); psi_i <- sum_j V(j, i) psi_j
        hs = np.conj(hpsi) @ psi.T
        e, v = scipy.linalg.eigh(hs, lower=False, driver="evd")
        psi[:] = v.T @ psi
        if rotate_h:
            hpsi[:] = v.T @ hpsi
        return e

    def _calc_grad(self, psi, hpsi, grad, grad_old, beta):
        nrm = 1.0 / np.sqrt(np.sum(psi.real ** 2 + psi.imag ** 2, axis=1))
        psi *= nrm[:, None]
        hpsi *= nrm[:, None]
        eps = np.sum((hpsi * np.conj(psi)).real, axis=1)
        r = hpsi - eps[:, None] * psi
        r2 = r.real ** 2 + r.imag ** 2
        self.err = np.sqrt(np.sum(r2, axis=1))
        b = np.sum(r2 / self.prec[None, :], axis=1)
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = b / beta
        grad[:] = -r / self.prec[None, :] + ratio[:, None] * grad_old
        beta[:] = b

    @staticmethod
    def _line_minimize(grad, hgrad, psi, hpsi):
        nrm = 1.0 / np.sqrt(np.sum(grad.real ** 2 + grad.imag ** 2, axis=1))
        grad *= nrm[:, None]
        hgrad *= nrm[:, None]
        e0 = np.sum((hpsi * np.conj(psi)).real, axis=1)
        e1 = np.sum((grad * np.conj(hpsi)).real, axis=1)
        e2 = np.sum((grad * np.conj(hgrad)).real, axis=1)
        theta = 0.5 * np.abs(np.arctan(2.0 * e1 / (e0 - e2)))
        c, s = np.cos(theta)[:, None], np.sin(theta)[:, None]
        psi[:] = psi * c + grad * s
        hpsi[:] = hpsi * c + hgrad * s

    @staticmethod
    def _orth_cholesky(psi, hpsi):
        s = np.conj(psi) @ psi.T                       # S(a, b) = <psi_a | psi_b>
        u = scipy.linalg.cholesky(s, lower=False)      # S = U^H U
        uinv = scipy.linalg.solve_triangular(u, np.eye(len(s)), lower=False)
        psi[:] = uinv.T @ psi
        hpsi[:] = uinv.T @ hpsi

    # ---------------------------------------------------------------- driver
    def diag(self, hpsi_fn, psi, eig, scf_iter=1):
        """hpsi_fn(X) -> H X for the rows of X; psi (nband x nbasis) and eig (nband) in place.  Returns the
        number of iterations of the loop."""
        nb, n = self.nband, self.nbasis
        hpsi = hpsi_fn(psi)
        eig[:] = self._rayleigh_ritz(psi, hpsi, True)
        grad_old = np.zeros((nb, n), complex)
        grad = np.zeros((nb, n), complex)
        beta = np.full(nb, np.inf)
        max_iter = self.nline if scf_iter > 1 else self.nline * 6
        ntry = 0
        while True:
            ntry += 1
            self._calc_grad(psi, hpsi, grad, grad_old, beta)
            grad -= (np.conj(psi) @ grad.T).T @ psi     # hsub(i, k) = <psi_k | grad_i>
            grad_old[:] = grad
            hgrad = hpsi_fn(grad)
            self._line_minimize(grad, hgrad, psi, hpsi)
            self._orth_cholesky(psi, hpsi)
            if scf_iter == 1 and ntry % self.nline == 0:
                hpsi = hpsi_fn(psi)
                eig[:] = self._rayleigh_ritz(psi, hpsi, True)
            if not (ntry < max_iter and np.any(self.err > self.all_band_cg_thr)):
                break
        eig[:] = self._rayleigh_ritz(psi, hpsi, False)
        return ntry
