"""GPU Davidson with subspace rotation (Diago_DavSubspace<T, DEVICE_GPU> drop-in) against the oracle
(oracle/dav_subspace_ref.py, itself pinned against the reference's compiled CPU solver):

* Si2.mat (pyabacus' golden matrix) through the callback HPsiFunc interface, with and without the initial
  subspace rotation, SCF and NSCF exit rules, psi with a padded leading dimension: eigenvalues within 1e-8
  of the oracle run from the same start and of the dense spectrum, iteration counts close to the oracle's;
* the same with empty bands (converged at max(5 thr, 1e-5));
* the 8-atom plane-wave cell through the built-in H|psi> of a Hamiltonian handle, against the oracle run on
  the oracle's own H (assembled densely) and the dense spectrum.
"""
from __future__ import annotations

import os

import numpy as np
import pytest
import scipy.sparse

from oracle import hamilt_ref as H
from oracle.dav_subspace_ref import DavSubspaceRef

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


class DevPtr:
    """Wrap a raw device pointer so torch can view it."""

    def __init__(self, p, n, typestr="<c16"):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (p, False), "version": 3}


@pytest.fixture(scope="module")
def si2():
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "pyabacus_si2.npz"))
    A = scipy.sparse.csc_matrix((d["data"], d["indices"], d["indptr"]), shape=tuple(d["shape"])).toarray()
    return A.astype(np.complex128)


def _dense_callback(Ad):
    def hpsi(x, hx, nvec, dim, i0, i1):
        m = i1 - i0 + 1
        X = torch.as_tensor(DevPtr(x, nvec * dim), device="cuda").view(nvec, dim)[i0:i1 + 1]
        HX = torch.as_tensor(DevPtr(hx, m * dim), device="cuda").view(m, dim)
        HX.copy_((Ad @ X.T).T)
    return hpsi


def _start(n, nband, seed=5):
    q, _ = np.linalg.qr(np.random.default_rng(seed).standard_normal((n, nband)) + 0j)
    return np.ascontiguousarray(q.T)


@pytest.mark.parametrize("need_subspace,scf", [(False, False), (True, True), (True, False)])
def test_dav_subspace_si2_callback(pkg, si2, need_subspace, scf):
    A = si2
    n, nband, ndim, thr = A.shape[0], 8, 4, 1e-10
    pc = np.abs(np.diag(A)).real
    psi0 = _start(n, nband)
    e_o, p_o = np.zeros(nband), psi0.copy()
    it_o = DavSubspaceRef(pc, nband, n, ndim, thr, 300, need_subspace).diag(lambda x: (A @ x.T).T, p_o, e_o, scf)

    ld = n + 5  # padded psi_in_dmax
    psi_h = np.full((nband, ld), 7.0 + 7.0j)
    psi_h[:, :n] = psi0
    psi = torch.from_numpy(psi_h.reshape(-1).copy()).cuda()
    dav = pkg.pwdft.DiagoDavSubspace(torch.from_numpy(pc).cuda(), nband, n, ndim, thr, 300, need_subspace)
    e = np.zeros(nband)
    it = dav.diag(_dense_callback(torch.from_numpy(A).cuda()), psi, ld, e, scf_type=scf)
    notconv, nh = dav.stats()
    w = np.linalg.eigvalsh(A)[:nband]
    assert np.max(np.abs(e - e_o)) < 1e-8, e - e_o
    assert np.max(np.abs(e - w)) < 1e-8, e - w
    assert abs(it - it_o) <= max(3, it_o // 20), (it, it_o)
    assert nh > it and (scf or notconv == 0)
    X = psi.cpu().numpy().reshape(nband, ld)
    assert np.all(X[:, n:] == 0)  # the exit step zeroes psi before writing the Ritz vectors (:210)
    res = np.linalg.norm(X[:, :n] @ A.T - e[:, None] * X[:, :n], axis=1)
    assert np.max(res) < 1e-4, res


def test_dav_subspace_si2_empty_bands(pkg, si2):
    A = si2
    n, nband, ndim, thr = A.shape[0], 8, 4, 1e-10
    occ = [True] * 5 + [False] * 3
    pc = np.abs(np.diag(A)).real
    psi0 = _start(n, nband, seed=9)
    e_o, p_o = np.zeros(nband), psi0.copy()
    it_o = DavSubspaceRef(pc, nband, n, ndim, thr, 300).diag(lambda x: (A @ x.T).T, p_o, e_o, False, occ)
    e_all = np.zeros(nband)
    it_all = DavSubspaceRef(pc, nband, n, ndim, thr, 300).diag(lambda x: (A @ x.T).T, psi0.copy(), e_all, False)
    assert it_o < it_all  # the oracle itself: empty bands stop earlier

    psi = torch.from_numpy(psi0.reshape(-1).copy()).cuda()
    dav = pkg.pwdft.DiagoDavSubspace(torch.from_numpy(pc).cuda(), nband, n, ndim, thr, 300)
    e = np.zeros(nband)
    it = dav.diag(_dense_callback(torch.from_numpy(A).cuda()), psi, n, e, is_occupied=occ)
    w = np.linalg.eigvalsh(A)[:nband]
    assert np.max(np.abs(e[:5] - e_o[:5])) < 1e-8 and np.max(np.abs(e[:5] - w[:5])) < 1e-8
    assert np.max(np.abs(e[5:] - w[5:])) < 1e-3
    assert abs(it - it_o) <= max(3, it_o // 20), (it, it_o)


def test_dav_subspace_diamond8_hamilt(pkg, diamond8_dense_h):
    wl, hm, w, ref_b = diamond8_dense_h
    pc_ref = H.precondition_dav_subspace(ref_b, 0)
    P = pkg.pwdft
    ld = wl.basis.npwk_max
    npw = int(wl.basis.npwk[0])
    nband, ndim, thr = wl.spec.nbands, 4, 1e-9
    psi0 = wl.psi0_h[0][:nband].copy()
    q, _ = np.linalg.qr(psi0[:, :npw].T)
    psi0[:, :npw] = q.T
    e_o, p_o = np.zeros(nband), psi0.copy()
    it_o = DavSubspaceRef(pc_ref, nband, npw, ndim, thr, 100).diag(lambda x: (hm @ x.T).T, p_o, e_o)

    h = P.device_hamilt(wl, P.PREC_FP64)
    pc = P.precondition_dav_subspace_d(wl.basis, 0)
    assert np.allclose(pc.cpu().numpy()[:npw], pc_ref[:npw], rtol=1e-14, atol=0)
    dav = P.DiagoDavSubspace(pc, nband, npw, ndim, thr, 100)
    psi = torch.from_numpy(psi0.reshape(-1).copy()).cuda()
    e = np.zeros(nband)
    it = dav.diag_hamilt(h, 0, psi, ld, e)
    assert np.max(np.abs(e - e_o)) < 1e-8, e - e_o
    assert np.max(np.abs(e - w[:nband])) < 1e-8, e - w[:nband]
    assert abs(it - it_o) <= 3, (it, it_o)
    notconv, nh = dav.stats()
    assert notconv == 0 and nh >= nband * (it + 1) // 4
