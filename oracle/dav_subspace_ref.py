"""Oracle (test infrastructure only): numpy restatement of the reference's Diago_DavSubspace
(module_hsolver/diago_dav_subspace.cpp), the "dav_subspace" method of HSolverPW.  Pinned against the
reference's own CPU solver compiled from its sources (oracle/_ref, tests/test_dav_subspace.py).

The iteration, as the reference's CPU path runs it:
* diag (:804-838): tries diag_once up to 6 times (test_exit_cond, :841-857); every try after the first (or
  every try with need_subspace) starts with diagH_subspace (:860-957): a Rayleigh-Ritz of psi with the
  generalised eigenproblem (psi^H H psi, psi^H psi), psi rotated to its Ritz vectors;
* diag_once (:86-291): the first Rayleigh-Ritz of the nband input vectors as a standard eigenproblem (the
  input is taken as orthonormal); then per iteration: residuals of the unconverged Ritz pairs, divided by
  the preconditioner 0.5 (1 + x + sqrt(1 + (x - 1)^2)) with x = |h_diag - lambda| and normalised, but not
  orthogonalised (cal_grad :294-428); their H|psi>; the new columns of the subspace matrices hcc = B^H H B
  and scc = B^H B, made Hermitian (cal_elem :431-574); the lowest nband pairs of the generalised problem
  (hcc, scc) (diag_zhegvx :577-706, the CPU branch's dngvx_op); a band is converged when its eigenvalue
  moved less than thr; when all are, or the basis would exceed nbase_x - 1 (:245), or at maxiter: psi
  becomes the Ritz vectors and the basis is restarted from them (refresh :709-801).
The reference applies H to all nbase_x vectors of its first step (:122), of which only the first nband are
read; here it is applied to those nband.
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import eigh


class DavSubspaceRef:
    def __init__(self, precondition, nband, dim, david_ndim, thr, maxiter, need_subspace=False):
        assert david_ndim > 1 and david_ndim * nband < dim
        self.pc = np.asarray(precondition, dtype=np.float64)[:dim]
        self.nband, self.dim = nband, dim
        self.nbase_x = nband * david_ndim
        self.thr, self.maxiter, self.is_subspace = thr, maxiter, need_subspace
        nx = self.nbase_x
        self.psi_iter = np.zeros((nx, dim), complex)   # basis vectors, one per row
        self.hphi = np.zeros((nx, dim), complex)
        self.hcc = np.zeros((nx, nx), complex)         # hcc[r, c]: element (row r, column c)
        self.scc = np.zeros((nx, nx), complex)
        self.vcc = np.zeros((nx, nx), complex)         # Ritz vectors in columns
        self.notconv = 0

    # ---------------------------------------------------------------- pieces
    def _diag_zhegvx(self, nbase, init):
        nb = self.nband
        h = self.hcc[:nbase, :nbase]
        if init and self.is_subspace:
            e = np.real(np.diag(h))[:nb].copy()
            for m in range(nb):
                self.vcc[m, m] = 1.0
            return e
        if init:
            w, v = eigh(h, subset_by_index=[0, nb - 1])
        else:
            w, v = eigh(h, self.scc[:nbase, :nbase], subset_by_index=[0, nb - 1])
        self.vcc[:nbase, :nb] = v
        return w

    def _cal_grad(self, hpsi, nbase, unconv, e_iter):
        nc = len(unconv)
        # compaction of the unconverged Ritz columns and eigenvalues (:306-315)
        for i in range(nc):
            if unconv[i] != i:
                self.vcc[:nbase, i] = self.vcc[:nbase, unconv[i]]
                e_iter[i] = e_iter[unconv[i]]
        vc = self.vcc[:nbase, :nc]
        x = vc.T @ self.psi_iter[:nbase]                 # psi_iter[:, :nbase] * vcc[:nbase, :nc]
        x *= -e_iter[:nc, None]
        x += vc.T @ self.hphi[:nbase]
        xx = np.abs(self.pc[None, :] - e_iter[:nc, None])
        x /= 0.5 * (1.0 + xx + np.sqrt(1.0 + (xx - 1.0) ** 2))
        x /= np.sqrt(np.sum(np.abs(x) ** 2, axis=1))[:, None]
        self.psi_iter[nbase:nbase + nc] = x
        self.hphi[nbase:nbase + nc] = hpsi(self.psi_iter[nbase:nbase + nc])

    def _cal_elem(self, nbase, nc):
        new = slice(nbase, nbase + nc)
        b = self.psi_iter[:nbase + nc]
        self.hcc[:nbase + nc, new] = b.conj() @ self.hphi[new].T
        self.scc[:nbase + nc, new] = b.conj() @ self.psi_iter[new].T
        last, nbase = nbase, nbase + nc
        # real diagonal of the new columns; row j >= last, column i < j from column j, row i (:542-556)
        for a in (self.hcc, self.scc):
            d = np.arange(last, nbase)
            a[d, d] = a[d, d].real
            j, i = np.tril_indices(nbase, -1)
            keep = j >= last
            a[j[keep], i[keep]] = np.conj(a[i[keep], j[keep]])
        self.hcc[nbase:, nbase:] = 0.0
        self.scc[nbase:, nbase:] = 0.0
        return nbase

    def _refresh(self, nbase, e_in):
        nb = self.nband
        self.hphi[:nb] = self.vcc[:nbase, :nb].T @ self.hphi[:nbase]
        for a in (self.hcc, self.scc, self.vcc):
            a[:nb, :nb] = 0.0
        for i in range(nb):
            self.hcc[i, i] = e_in[i]
            self.scc[i, i] = 1.0
            self.vcc[i, i] = 1.0
        return nb

    def _diag_once(self, hpsi, psi, eig, occupied):
        nb, dim = self.nband, self.dim
        unconv = list(range(nb))
        self.notconv = nb
        self.psi_iter[:nb] = psi[:, :dim]
        self.hphi[:nb] = hpsi(self.psi_iter[:nb])
        nbase = self._cal_elem(0, nb)
        e_iter = np.zeros(self.nbase_x)
        e_iter[:nb] = self._diag_zhegvx(nbase, True)
        eig[:] = e_iter[:nb]
        it = 0
        while True:
            it += 1
            self._cal_grad(hpsi, nbase, unconv, e_iter)
            nbase = self._cal_elem(nbase, self.notconv)
            e_iter[:nb] = self._diag_zhegvx(nbase, False)
            # an empty band converges at max(5 thr, 1e-5) (:186-194)
            thr_m = [self.thr if occupied[m] else max(self.thr * 5.0, 1e-5) for m in range(nb)]
            unconv = [m for m in range(nb) if not abs(e_iter[m] - eig[m]) < thr_m[m]]
            self.notconv = len(unconv)
            eig[:] = e_iter[:nb]
            if self.notconv == 0 or nbase + self.notconv + 1 > self.nbase_x or it == self.maxiter:
                psi[:, :] = 0.0
                psi[:, :dim] = self.vcc[:nbase, :nb].T @ self.psi_iter[:nbase]
                self.psi_iter[:nb] = psi[:, :dim]
                nbase = self._refresh(nbase, eig)
                if self.notconv == 0 or it == self.maxiter:
                    return it

    def _diagh_subspace(self, hpsi, psi, eig):
        nb, dim = self.nband, self.dim
        x = psi[:, :dim]
        hx = hpsi(x)
        w, v = eigh(x.conj() @ hx.T, x.conj() @ x.T)
        eig[:] = w[:nb]
        psi[:, :dim] = v[:, :nb].T @ x

    # ---------------------------------------------------------------- driver
    def diag(self, hpsi, psi, eig, scf=False, occupied=None):
        """hpsi(X) -> H X for the rows of X (m x dim); psi (nband x ld, ld >= dim) and eig (nband) in place;
        occupied: nband flags (None: all occupied).  Returns the total iteration count."""
        occupied = [True] * self.nband if occupied is None else [bool(o) for o in occupied]
        total, ntry = 0, 0
        self.notconv = 0
        while True:
            if self.is_subspace or ntry > 0:
                self._diagh_subspace(hpsi, psi, eig)
            total += self._diag_once(hpsi, psi, eig, occupied)
            ntry += 1
            f1 = ntry <= 5
            f2 = (not scf) and self.notconv > 0
            f3 = scf and self.notconv > 5
            if not (f1 and (f2 or f3)):
                return total
