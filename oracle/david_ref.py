"""CPU oracle (test infrastructure only): ABACUS's block Davidson, restated in numpy.

Follows source/module_hsolver/diago_david.cpp (abacus-develop v3.8.0) step by
step, with the same storage conventions:
  * basis / hpsi / spsi: nbase_x vectors of length dim, vector m at m*dim
    (ctor :34-148);
  * hcc / scc / vcc: column-major nbase_x x nbase_x, element (i, j) at
    j*nbase_x + i; cal_elem fills rows nbase..nbase+notconv-1 (:626-717);
  * the subspace eigensolve takes the lower triangle and the lowest nband
    eigenpairs (dnevx_op<CPU> = LAPACK zheevx 'V','I','L', dngvd_op.cpp:142-235);
  * convergence: |lambda_new - lambda_old| < thr per band (:270-280);
  * restart/refresh when nbase + notconv > nbase_x (:283-330, refresh :797-934);
  * Gram-Schmidt with the blocked plan of planSchmidtOrth (:950-1147);
  * diag() retries diag_once while notconv > notconv_max, at most ntry_max+1
    times (:1173-1240).
Only ``tests/`` and the CPU-baseline leg of ``bench.py`` use it.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg


def plan_schmidt_orth(nband):
    """planSchmidtOrth (diago_david.cpp:1087-1147)."""
    mm = [0] * nband
    mv = [0] * nband
    if nband <= 0:
        return mm, mv
    last = nband
    msize = nband // 2
    divide_times = 0
    points = [0] * nband
    res = nband - msize
    while msize > 1:
        index = nband - msize
        if divide_times == 0:
            points[0] = index
            mm[index] = msize
            mv[index] = 1 if res == msize else 2
            divide_times = 1
        else:
            for i in range(divide_times - 1, -1, -1):
                points[i * 2] = points[i] - msize
                points[i * 2 + 1] = points[i * 2] + last
                mm[points[i * 2]] = msize
                mm[points[i * 2 + 1]] = msize
                v = 1 if res == msize else 2
                mv[points[i * 2]] = v
                mv[points[i * 2 + 1]] = v
            divide_times *= 2
        last = msize
        msize = res // 2
        res -= msize
    mv[0] = 1
    for m in range(1, nband):
        if mv[m] == 0:
            mv[m] = mv[m - 1] + 1
    return mm, mv


class DiagoDavidRef:
    def __init__(self, precondition, nband, dim, david_ndim=4):
        self.precondition = np.asarray(precondition, dtype=np.float64)
        self.nband = nband
        self.dim = dim
        self.david_ndim = david_ndim
        self.nbase_x = david_ndim * nband
        assert david_ndim > 1 and david_ndim * nband < dim
        nx = self.nbase_x
        self.basis = np.zeros(nx * dim, dtype=np.complex128)
        self.hpsi = np.zeros(nx * dim, dtype=np.complex128)
        self.spsi = np.zeros(nx * dim, dtype=np.complex128)
        self.hcc = np.zeros(nx * nx, dtype=np.complex128)
        self.scc = np.zeros(nx * nx, dtype=np.complex128)
        self.vcc = np.zeros(nx * nx, dtype=np.complex128)
        self.eigenvalue = np.zeros(nx)
        self.notconv = 0
        self.hpsi_calls = 0

    # helpers on the flat storage
    def _vec(self, arr, m):
        return arr[m * self.dim:(m + 1) * self.dim]

    def _mat(self, arr, m0, m1):
        """columns m0..m1-1 as a dim x (m1-m0) matrix (views)."""
        return arr[m0 * self.dim:m1 * self.dim].reshape(m1 - m0, self.dim).T

    def schmidt_orth(self, nband, m, spsi, lagrange_m, mm_size, mv_size):
        """SchmidtOrth (diago_david.cpp:950-1075); lagrange_m is a length-nband view."""
        dim = self.dim
        psi_m = self._vec(self.basis, m)
        spsi_m = spsi[m * dim:(m + 1) * dim]
        if mm_size != 0:
            s0 = m - mv_size + 1 - mm_size
            A = self._mat(self.basis, s0, s0 + mm_size)
            # gemm('C','N', mm, mm, dim, basis(s0..), spsi[m*dim] with ldb=dim, ldc=nband): only column 0 matters
            # for the vector update below; the reference computes an mm x mm block whose first column lands in
            # lagrange_m[s0 .. s0+mm) and whose other columns land in later vectors' lagrange rows.
            B = spsi[m * dim:(m + mm_size) * dim].reshape(mm_size, dim).T
            C = A.conj().T @ B
            lag2d = self._lag_full
            base = self._lag_base  # flat offset of lagrange_m inside the full lagrange buffer
            for j in range(mm_size):
                off = base + j * nband + s0
                lag2d[off:off + mm_size] = C[:, j]
        s1 = m - mv_size + 1
        A = self._mat(self.basis, s1, s1 + mv_size)
        lagrange_m[s1:s1 + mv_size] = A.conj().T @ spsi_m
        psi_norm = lagrange_m[m].real
        assert psi_norm > 0.0
        if m > 0:
            Bm = self._mat(self.basis, 0, m)
            psi_m -= Bm @ lagrange_m[:m]
        psi_norm -= float(np.real(np.vdot(lagrange_m[:m], lagrange_m[:m])))
        assert psi_norm > 0.0
        psi_norm = np.sqrt(psi_norm)
        if psi_norm < 1.0e-12:
            raise RuntimeError("SchmidtOrth aborted for psi_norm < 1e-12")
        psi_m /= psi_norm

    def cal_elem(self, nbase, notconv):
        """cal_elem (diago_david.cpp:626-717)."""
        if notconv == 0:
            return nbase
        nx = self.nbase_x
        Bn = self._mat(self.basis, nbase, nbase + notconv)
        H = self._mat(self.hpsi, 0, nbase + notconv)
        S = self._mat(self.spsi, 0, nbase + notconv)
        hc = Bn.conj().T @ H  # notconv x (nbase+notconv)
        sc = Bn.conj().T @ S
        hcc = self.hcc.reshape(nx, nx)  # [col, row]
        scc = self.scc.reshape(nx, nx)
        for j in range(nbase + notconv):
            hcc[j, nbase:nbase + notconv] = hc[:, j]
            scc[j, nbase:nbase + notconv] = sc[:, j]
        return nbase + notconv

    def diag_zhegvx(self, nbase, nband):
        """dnevx_op<CPU>: lowest nband eigenpairs of the lower triangle of hcc (dngvd_op.cpp:142-235)."""
        nx = self.nbase_x
        h = self.hcc.reshape(nx, nx).T[:nbase, :nbase]  # [row, col]
        low = np.tril(h)
        full = low + np.tril(h, -1).conj().T
        w, v = scipy.linalg.eigh(full, lower=True, subset_by_index=[0, nband - 1], driver="evx")
        self.eigenvalue[:nband] = w
        vcc = self.vcc.reshape(nx, nx)
        for j in range(nband):
            vcc[j, :nbase] = v[:, j]

    def cal_grad(self, hpsi_func, spsi_func, nbase, notconv, unconv):
        """cal_grad (diago_david.cpp:359-611)."""
        if notconv == 0:
            return
        dim = self.dim
        nx = self.nbase_x
        vcc = self.vcc.reshape(nx, nx)
        vc = np.stack([vcc[unconv[m], :nbase] for m in range(notconv)], 1)  # nbase x notconv
        H = self._mat(self.hpsi, 0, nbase)
        S = self._mat(self.spsi, 0, nbase)
        new = H @ vc
        vc = vc * (-self.eigenvalue[np.asarray(unconv[:notconv])])[None, :]
        new = new + S @ vc
        new = new / self.precondition[:, None]
        self.basis[nbase * dim:(nbase + notconv) * dim] = new.T.reshape(-1)
        for m in range(notconv):
            spsi_func(self._vec(self.basis, nbase + m), self.spsi[(nbase + m) * dim:(nbase + m + 1) * dim])
        ld = nbase + notconv
        lagrange = np.zeros(notconv * ld, dtype=np.complex128)
        Ball = self._mat(self.basis, 0, nbase)
        Sn = self._mat(self.spsi, nbase, nbase + notconv)
        lag0 = Ball.conj().T @ Sn  # nbase x notconv -> columns of lagrange (ldc = nbase+notconv)
        for m in range(notconv):
            lagrange[m * ld:m * ld + nbase] = lag0[:, m]
        mm, mv = plan_schmidt_orth(notconv)
        self._lag_full = lagrange
        for m in range(notconv):
            self._lag_base = m * ld
            self.schmidt_orth(ld, nbase + m, self.spsi, lagrange[m * ld:(m + 1) * ld], mm[m], mv[m])
            spsi_func(self._vec(self.basis, nbase + m), self.spsi[(nbase + m) * dim:(nbase + m + 1) * dim])
        self.hpsi[nbase * dim:(nbase + notconv) * dim] = hpsi_func(
            self.basis[nbase * dim:(nbase + notconv) * dim], notconv)
        self.hpsi_calls += notconv

    def refresh(self, nband, eigenvalue_in, psi, ldpsi):
        """refresh (diago_david.cpp:797-934)."""
        dim = self.dim
        nx = self.nbase_x
        nbase = self._nbase
        vcc = self.vcc.reshape(nx, nx)
        V = vcc[:nband, :nbase].T  # nbase x nband
        H = self._mat(self.hpsi, 0, nbase)
        S = self._mat(self.spsi, 0, nbase)
        hnew = H @ V
        snew = S @ V
        self.basis[:] = 0
        self.hpsi[:nband * dim] = hnew.T.reshape(-1)
        self.spsi[:nband * dim] = snew.T.reshape(-1)
        for m in range(nband):
            self.basis[m * dim:(m + 1) * dim] = psi[m * ldpsi:m * ldpsi + dim]
        self.hcc[:] = 0
        self.scc[:] = 0
        for i in range(nband):
            self.hcc[i * nx + i] = eigenvalue_in[i]
            self.scc[i * nx + i] = 1.0
            self.vcc[i * nx + i] = 1.0
        self._nbase = nband

    def diag_once(self, hpsi_func, spsi_func, ldpsi, psi, eigenvalue_in, thr, maxiter):
        """diag_once (diago_david.cpp:151-341)."""
        nband, dim = self.nband, self.dim
        unconv = list(range(nband))
        nbase = 0
        self.notconv = nband
        mm, mv = plan_schmidt_orth(nband)
        for m in range(nband):
            spsi_func(psi[m * ldpsi:m * ldpsi + dim], self.spsi[m * dim:(m + 1) * dim])
        lagrange = np.zeros(nband * nband, dtype=np.complex128)
        self._lag_full = lagrange
        for m in range(nband):
            self.basis[m * dim:(m + 1) * dim] = psi[m * ldpsi:m * ldpsi + dim]
            self._lag_base = m * nband
            self.schmidt_orth(nband, m, self.spsi, lagrange[m * nband:(m + 1) * nband], mm[m], mv[m])
            spsi_func(self._vec(self.basis, m), self.spsi[m * dim:(m + 1) * dim])
        self.hpsi[:nband * dim] = hpsi_func(self.basis[:nband * dim], nband)
        self.hpsi_calls += nband
        nbase = self.cal_elem(nbase, self.notconv)
        self.diag_zhegvx(nbase, nband)
        eigenvalue_in[:nband] = self.eigenvalue[:nband]
        dav_iter = 0
        while True:
            dav_iter += 1
            self.cal_grad(hpsi_func, spsi_func, nbase, self.notconv, unconv)
            nbase = self.cal_elem(nbase, self.notconv)
            self.diag_zhegvx(nbase, nband)
            self.notconv = 0
            for m in range(nband):
                conv = abs(self.eigenvalue[m] - eigenvalue_in[m]) < thr
                if not conv:
                    unconv[self.notconv] = m
                    self.notconv += 1
                eigenvalue_in[m] = self.eigenvalue[m]
            if (not self.notconv) or (nbase + self.notconv > self.nbase_x) or dav_iter == maxiter:
                nx = self.nbase_x
                vcc = self.vcc.reshape(nx, nx)
                B = self._mat(self.basis, 0, nbase)
                newpsi = B @ vcc[:nband, :nbase].T
                psi[:nband * ldpsi] = 0
                for m in range(nband):
                    psi[m * ldpsi:m * ldpsi + dim] = newpsi[:, m]
                if (not self.notconv) or dav_iter == maxiter:
                    break
                self._nbase = nbase
                self.refresh(nband, eigenvalue_in, psi, ldpsi)
                nbase = self._nbase
        return dav_iter

    def diag(self, hpsi_func, spsi_func, ldpsi, psi, eigenvalue_in, thr, maxiter, ntry_max=5, notconv_max=0):
        """diag (diago_david.cpp:1173-1200) with check_block_conv (:1223-1240)."""
        ntry = 0
        self.notconv = 0
        total = 0
        while True:
            total += self.diag_once(hpsi_func, spsi_func, ldpsi, psi, eigenvalue_in, thr, maxiter)
            ntry += 1
            if ntry > ntry_max or self.notconv <= notconv_max:
                break
        return total


def copy_spsi(x, out):
    """HamiltPW::sPsi for norm-conserving pseudopotentials: S = I (hamilt_pw.cpp:203-240)."""
    out[:] = x
