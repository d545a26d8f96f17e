"""pyabacus.hsolver's functions on this library's device solvers: ``dav_subspace`` and ``davidson`` with the
reference's Python signatures and semantics (python/pyabacus/src/pyabacus/hsolver/_hsolver.py:18-176), so a
pyabacus script switches by changing the import.

As there: mvv_op(X) takes a (dim, nvec) complex block (the vectors as columns, Fortran order) and returns
H X of the same shape; init_v holds num_eigs start vectors of dim entries one after another (any shape;
flattened in C order, as pyabacus's set_psi reads it); the result is (eigenvalues, flat eigenvectors).
The iterations run on the GPU (b200_dav_subspace_diag / b200_david_diag); mvv_op runs on the host, so each
application copies its block to the host and H X back.
"""
from __future__ import annotations

import numpy as np

from . import pwdft as P


def _torch():
    import torch
    return torch


def _start_block(init_v, dim, num_eigs):
    v = np.asarray(init_v)
    if v.ndim != 1 or v.dtype != np.complex128:
        v = v.flatten().astype(np.complex128, order="C")
    if v.size != dim * num_eigs:
        raise ValueError("init_v must hold num_eigs vectors of dim entries")
    return v


def _host_callback(mvv_op, dim_check):
    """HPsiFunc over device pointers: block X (vectors i0..i1 of stride dim) -> mvv_op on the host -> HX."""
    torch = _torch()

    def cb(x, hx, nvec, dim, i0, i1):
        if dim != dim_check:
            raise ValueError("vector length differs from dim")
        m = i1 - i0 + 1
        n = nvec * dim
        X = torch.as_tensor(_DevView(x, n), device="cuda").view(nvec, dim)[i0:i1 + 1]
        Xh = X.cpu().numpy()                       # (m, dim): its transpose is the (dim, m) Fortran block
        HXh = np.asarray(mvv_op(np.asfortranarray(Xh.T)), dtype=np.complex128)
        if HXh.shape != (dim, m):
            raise ValueError(f"mvv_op returned shape {HXh.shape}, expected {(dim, m)}")
        HX = torch.as_tensor(_DevView(hx, m * dim), device="cuda").view(m, dim)
        HX.copy_(torch.from_numpy(np.ascontiguousarray(HXh.T)))
        torch.cuda.synchronize()
    return cb


class _DevView:
    """A raw device pointer as a CUDA-array-interface object (complex128)."""

    def __init__(self, p, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<c16", "data": (p, False), "version": 3}


def dav_subspace(mvv_op, init_v, dim, num_eigs, pre_condition, dav_ndim=2, tol=1e-2, max_iter=1000,
                 need_subspace=False, is_occupied=None, scf_type=False):
    """Diagonalise with the Davidson-subspace method (Diago_DavSubspace) on the GPU.  Returns
    (eigenvalues (num_eigs,), eigenvectors flat (num_eigs * dim,), band after band)."""
    if not callable(mvv_op):
        raise TypeError("mvv_op must be a callable object.")
    if is_occupied is None:
        is_occupied = [True] * num_eigs
    assert dav_ndim > 1, "dav_ndim must be greater than 1."
    assert dav_ndim * num_eigs < dim, "dav_ndim * num_eigs must be less than dim * comm_info.nproc."
    torch = _torch()
    v = _start_block(init_v, dim, num_eigs)
    pc = torch.from_numpy(np.ascontiguousarray(np.asarray(pre_condition, dtype=np.float64)[:dim])).cuda()
    psi = torch.from_numpy(v.copy()).cuda()
    solver = P.DiagoDavSubspace(pc, num_eigs, dim, dav_ndim, tol, max_iter, need_subspace)
    e = np.zeros(num_eigs)
    solver.diag(_host_callback(mvv_op, dim), psi, dim, e, is_occupied=is_occupied, scf_type=scf_type)
    torch.cuda.synchronize()
    return e, psi.cpu().numpy()


def davidson(mvv_op, init_v, dim, num_eigs, pre_condition, dav_ndim=2, tol=1e-2, max_iter=1000, use_paw=False):
    """Diagonalise with the block Davidson method (DiagoDavid, ntry_max 5, notconv_max 0 as the reference's
    defaults) on the GPU.  Returns (eigenvalues, flat eigenvectors).  S = I only: use_paw is refused."""
    if not callable(mvv_op):
        raise TypeError("mvv_op must be a callable object.")
    if use_paw:
        raise NotImplementedError("PAW overlap operators are not supported by this library (S = I)")
    torch = _torch()
    v = _start_block(init_v, dim, num_eigs)
    pc = torch.from_numpy(np.ascontiguousarray(np.asarray(pre_condition, dtype=np.float64)[:dim])).cuda()
    psi = torch.from_numpy(v.copy()).cuda()
    solver = P.DiagoDavid(pc, num_eigs, dim, dav_ndim, P.PREC_FP64)
    e = np.zeros(num_eigs)
    solver.diag(_host_callback(mvv_op, dim), dim, psi, e, tol, max_iter, ntry_max=5, notconv_max=0)
    torch.cuda.synchronize()
    return e, psi.cpu().numpy()


class diag_comm_info:  # noqa: N801  (the reference's name)
    """pyabacus.hsolver.diag_comm_info: one process per pool here (rank 0 of 1)."""

    def __init__(self, rank: int = 0, nproc: int = 1) -> None:
        if nproc != 1 or rank != 0:
            raise ValueError("one process per solve: k-points are distributed across GPUs instead")
        self._rank, self._nproc = rank, nproc

    @property
    def rank(self) -> int:
        return self._rank

    @property
    def nproc(self) -> int:
        return self._nproc


__all__ = ["dav_subspace", "davidson", "diag_comm_info"]
