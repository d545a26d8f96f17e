"""Oracle (test infrastructure only): ctypes access to the reference's own CPU DiagoDavid,
Diago_DavSubspace and DiagoBPCG, compiled from the reference sources into oracle/_ref/libref_david.so by
oracle/build_ref.py.  Only the tests and the
benchmark's CPU reference arm use it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libref_david.so"
_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int)
_lib = None


def available() -> bool:
    return LIB.exists()


def _load():
    global _lib
    if _lib is None:
        lib = C.CDLL(str(LIB))
        lib.ref_david.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), _CB, C.c_void_p,
                                  C.c_void_p, C.POINTER(C.c_double), C.c_double, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_int)]
        lib.ref_david.restype = C.c_int
        lib.ref_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def diag(hpsi, precond, nband, dim, david_ndim, ldpsi, psi, eig, thr, maxiter, ntry_max=5, notconv_max=0):
    """DiagoDavid<complex<double>, CPU>::diag.  hpsi(x, nvec, dim, i0, i1) -> H applied to vectors i0..i1 of
    the block x (nvec x dim complex128), returned as ((i1-i0+1) x dim).  psi (complex128, nband vectors at
    m*ldpsi) and eig (float64, nband) are updated in place; returns the iteration count."""
    lib = _load()
    assert psi.dtype == np.complex128 and psi.flags.c_contiguous and eig.dtype == np.float64

    def cb(user, x, hx, nvec, d, i0, i1):
        m = i1 - i0 + 1
        X = np.ctypeslib.as_array(C.cast(x, C.POINTER(C.c_double)), shape=(nvec * d * 2,)).view(np.complex128)
        HX = np.ctypeslib.as_array(C.cast(hx, C.POINTER(C.c_double)), shape=(m * d * 2,)).view(np.complex128)
        HX[:] = hpsi(X.reshape(nvec, d), nvec, d, i0, i1).reshape(-1)

    fn = _CB(cb)
    pc = np.ascontiguousarray(precond, dtype=np.float64)
    it = C.c_int()
    rc = lib.ref_david(nband, dim, david_ndim, ldpsi, pc.ctypes.data_as(C.POINTER(C.c_double)), fn, None, psi.ctypes.data,
                       eig.ctypes.data_as(C.POINTER(C.c_double)), thr, maxiter, ntry_max, notconv_max, C.byref(it))
    if rc != 0:
        raise RuntimeError("reference DiagoDavid failed: " + lib.ref_last_error().decode())
    return it.value


def dav_subspace(hpsi, precond, nband, dim, david_ndim, ldpsi, psi, eig, thr, maxiter, need_subspace=False, scf=False,
                 occupied=None):
    """Diago_DavSubspace<complex<double>, CPU>::diag; occupied: nband flags (None: all bands occupied).  hpsi as
    for diag; psi and eig are updated in place; returns the iteration count."""
    lib = _load()
    if not hasattr(lib, "_ds_ready"):
        lib.ref_dav_subspace.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), _CB, C.c_void_p,
                                         C.c_void_p, C.POINTER(C.c_double), C.c_double, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.ref_dav_subspace.restype = C.c_int
        lib.ref_dav_subspace_last_error.restype = C.c_char_p
        lib._ds_ready = True
    assert psi.dtype == np.complex128 and psi.flags.c_contiguous and eig.dtype == np.float64

    def cb(user, x, hx, nvec, d, i0, i1):
        m = i1 - i0 + 1
        X = np.ctypeslib.as_array(C.cast(x, C.POINTER(C.c_double)), shape=(nvec * d * 2,)).view(np.complex128)
        HX = np.ctypeslib.as_array(C.cast(hx, C.POINTER(C.c_double)), shape=(m * d * 2,)).view(np.complex128)
        HX[:] = hpsi(X.reshape(nvec, d), nvec, d, i0, i1).reshape(-1)

    fn = _CB(cb)
    pc = np.ascontiguousarray(precond, dtype=np.float64)
    it = C.c_int()
    occ = None if occupied is None else np.ascontiguousarray(np.asarray(occupied, dtype=bool).astype(np.int32))
    rc = lib.ref_dav_subspace(nband, dim, david_ndim, ldpsi, pc.ctypes.data_as(C.POINTER(C.c_double)), fn, None,
                              psi.ctypes.data, eig.ctypes.data_as(C.POINTER(C.c_double)), thr, maxiter,
                              int(bool(need_subspace)), int(bool(scf)),
                              None if occ is None else occ.ctypes.data_as(C.POINTER(C.c_int)), C.byref(it))
    if rc != 0:
        raise RuntimeError("reference Diago_DavSubspace failed: " + lib.ref_dav_subspace_last_error().decode())
    return it.value


def bpcg(hpsi, precond, nband, nbasis, psi, eig, scf_iter=1, ncalls=1):
    """DiagoBPCG<complex<double>, CPU>: init_iter on psi (nband x nbasis) and ncalls diag calls with
    DiagoIterAssist::SCF_ITER = scf_iter.  hpsi(X, nvec, dim, i0, i1) -> H applied to rows i0..i1 of X; psi and
    eig updated in place."""
    lib = _load()
    if not hasattr(lib, "_bp_ready"):
        lib.ref_bpcg.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), _CB, C.c_void_p, C.c_void_p,
                                 C.POINTER(C.c_double), C.c_int, C.c_int]
        lib.ref_bpcg.restype = C.c_int
        lib.ref_bpcg_last_error.restype = C.c_char_p
        lib._bp_ready = True
    assert psi.dtype == np.complex128 and psi.flags.c_contiguous and eig.dtype == np.float64

    def cb(user, x, hx, nvec, d, i0, i1):
        m = i1 - i0 + 1
        X = np.ctypeslib.as_array(C.cast(x, C.POINTER(C.c_double)), shape=(nvec * d * 2,)).view(np.complex128)
        HX = np.ctypeslib.as_array(C.cast(hx, C.POINTER(C.c_double)), shape=(m * d * 2,)).view(np.complex128)
        HX[:] = hpsi(X.reshape(nvec, d), nvec, d, i0, i1).reshape(-1)

    fn = _CB(cb)
    pc = np.ascontiguousarray(precond, dtype=np.float64)
    rc = lib.ref_bpcg(nband, nbasis, pc.ctypes.data_as(C.POINTER(C.c_double)), fn, None, psi.ctypes.data,
                      eig.ctypes.data_as(C.POINTER(C.c_double)), int(scf_iter), int(ncalls))
    if rc != 0:
        raise RuntimeError("reference DiagoBPCG failed: " + lib.ref_bpcg_last_error().decode())


def gweights(ekb, wk, nelec, sigma, ngauss):
    """Occupy::gweights (nspin 1): (wg, ef, demet) from the reference's compiled occupation code."""
    lib = _load()
    if not hasattr(lib, "_occ_ready"):
        pd = C.POINTER(C.c_double)
        lib.ref_gweights.argtypes = [C.c_int, pd, C.c_int, C.c_double, C.c_double, C.c_int, pd, pd, pd, pd]
        lib.ref_gweights.restype = C.c_int
        lib.ref_occupy_last_error.restype = C.c_char_p
        lib._occ_ready = True
    e = np.ascontiguousarray(ekb, dtype=np.float64)
    w = np.ascontiguousarray(wk, dtype=np.float64)
    nks, nband = e.shape
    wg = np.zeros_like(e)
    ef, demet = C.c_double(), C.c_double()
    pd = C.POINTER(C.c_double)
    rc = lib.ref_gweights(nks, w.ctypes.data_as(pd), nband, float(nelec), float(sigma), int(ngauss),
                          e.ctypes.data_as(pd), C.byref(ef), C.byref(demet), wg.ctypes.data_as(pd))
    if rc != 0:
        raise RuntimeError("reference Occupy::gweights failed: " + lib.ref_occupy_last_error().decode())
    return wg, ef.value, demet.value


def pw_basis_k(lat0, latvec, ecutwfc, kvec_d, ecutrho=None, grid=None):
    """The reference's own PW_Basis_K set-up (as ESolver_KS_PW builds the wavefunction basis): returns
    (nx, ny, nz), npwk per k-point, and per k-point ig2ixyz (iz + iy nz + ix ny nz) and gk2 arrays."""
    lib = _load()
    pd, pi = C.POINTER(C.c_double), C.POINTER(C.c_int)
    if not hasattr(lib, "_pw_ready"):
        lib.ref_pw_basis_k.argtypes = [C.c_double, pd, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                       pd, pi, pi, C.c_int, pi, pd]
        lib.ref_pw_basis_k.restype = C.c_int
        lib.ref_pw_basis_last_error.restype = C.c_char_p
        lib._pw_ready = True
    kd = np.ascontiguousarray(np.atleast_2d(kvec_d), dtype=np.float64)
    nks = len(kd)
    lv = np.ascontiguousarray(np.asarray(latvec, dtype=np.float64).reshape(9))
    gx, gy, gz = grid if grid is not None else (0, 0, 0)
    ecutrho = 4.0 * ecutwfc if ecutrho is None else ecutrho
    dims = np.zeros(4, dtype=np.int32)
    npwk = np.zeros(nks, dtype=np.int32)

    def call(cap, ig, g2):
        rc = lib.ref_pw_basis_k(lat0, lv.ctypes.data_as(pd), ecutwfc, ecutrho, gx, gy, gz, nks, kd.ctypes.data_as(pd),
                                dims.ctypes.data_as(pi), npwk.ctypes.data_as(pi), cap,
                                None if ig is None else ig.ctypes.data_as(pi),
                                None if g2 is None else g2.ctypes.data_as(pd))
        if rc != 0:
            raise RuntimeError("reference PW_Basis_K set-up failed: " + lib.ref_pw_basis_last_error().decode())

    call(0, None, None)
    cap = int(dims[3])
    ig = np.zeros((nks, cap), dtype=np.int32)
    g2 = np.zeros((nks, cap))
    call(cap, ig, g2)
    return (tuple(int(v) for v in dims[:3]), npwk.astype(np.int64),
            [ig[ik, :npwk[ik]].astype(np.int64) for ik in range(nks)], [g2[ik, :npwk[ik]].copy() for ik in range(nks)])


def pw_transform(lat0, latvec, ecutwfc, kvec_d, ik, inp, inverse, add=False, factor=1.0, out=None, ecutrho=None,
                 grid=None):
    """The reference's own PW_Basis_K::recip2real (inverse) / real2recip <double> of k-point ik on the basis
    pw_basis_k() builds, its FFT lines evaluated by the oracle build's mixed-radix stand-in for FFTW.  inp / out
    are complex128 arrays (npwk coefficients or the nx ny nz box in r order); out is updated in place (add)."""
    lib = _load()
    pd = C.POINTER(C.c_double)
    if not hasattr(lib, "_pwt_ready"):
        lib.ref_pw_transform.argtypes = [C.c_double, pd, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                         pd, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_double]
        lib.ref_pw_transform.restype = C.c_int
        lib._pwt_ready = True
    (nx, ny, nz), npwk, _, _ = pw_basis_k(lat0, latvec, ecutwfc, kvec_d, ecutrho=ecutrho, grid=grid)
    kd = np.ascontiguousarray(np.atleast_2d(kvec_d), dtype=np.float64)
    lv = np.ascontiguousarray(np.asarray(latvec, dtype=np.float64).reshape(9))
    src = np.ascontiguousarray(inp, dtype=np.complex128)
    n_out = nx * ny * nz if inverse else int(npwk[ik])
    dst = np.zeros(n_out, dtype=np.complex128) if out is None else out
    assert dst.dtype == np.complex128 and dst.flags.c_contiguous and dst.size == n_out
    gx, gy, gz = grid if grid is not None else (0, 0, 0)
    rc = lib.ref_pw_transform(lat0, lv.ctypes.data_as(pd), ecutwfc, 4.0 * ecutwfc if ecutrho is None else ecutrho,
                              gx, gy, gz, len(kd), kd.ctypes.data_as(pd), ik, int(bool(inverse)), src.ctypes.data,
                              dst.ctypes.data, int(bool(add)), float(factor))
    if rc != 0:
        raise RuntimeError("reference PW_Basis_K transform failed: " + lib.ref_pw_basis_last_error().decode())
    return dst


def hpsi_local(lat0, latvec, ecutwfc, kvec_d, ik, veff, psi, nbands, ecutrho=None, grid=None):
    """The kinetic + local part of H|psi> of k-point ik by the reference's own Ekinetic and Veff operators on
    the basis pw_basis_k() builds: psi (nbands x npwk_max complex) -> hpsi of the same shape."""
    lib = _load()
    pd = C.POINTER(C.c_double)
    if not hasattr(lib, "_hl_ready"):
        lib.ref_hpsi_local.argtypes = [C.c_double, pd, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, pd,
                                       C.c_int, pd, C.c_int, C.c_void_p, C.c_void_p]
        lib.ref_hpsi_local.restype = C.c_int
        lib._hl_ready = True
    kd = np.ascontiguousarray(np.atleast_2d(kvec_d), dtype=np.float64)
    lv = np.ascontiguousarray(np.asarray(latvec, dtype=np.float64).reshape(9))
    v = np.ascontiguousarray(veff, dtype=np.float64)
    x = np.ascontiguousarray(psi, dtype=np.complex128)
    out = np.zeros_like(x)
    gx, gy, gz = grid if grid is not None else (0, 0, 0)
    rc = lib.ref_hpsi_local(lat0, lv.ctypes.data_as(pd), ecutwfc, 4.0 * ecutwfc if ecutrho is None else ecutrho,
                            gx, gy, gz, len(kd), kd.ctypes.data_as(pd), ik, v.ctypes.data_as(pd), nbands, x.ctypes.data,
                            out.ctypes.data)
    if rc != 0:
        raise RuntimeError("reference local H|psi> failed: " + lib.ref_pw_basis_last_error().decode())
    return out


def nonlocal_act(na, nh, vkb, deeq, psi, npw, hpsi=None):
    """The nonlocal part of H|psi> by the reference's own Nonlocal operator (operator_pw/nonlocal_pw.cpp:
    init + act, add_nonlocal_pp with nonlocal_pw_op, gemm_op / gemv_op), compiled against stand-ins for
    UnitCell and pseudopot_cell_vnl that hold na[it], nh[it], the projectors and D.  vkb: (nkb, npwx) complex;
    deeq: (nspin, natoms, nhm, nhm) real, spin 0 used; psi: (nbands, ld) complex.  Returns hpsi + V_NL psi
    (hpsi defaults to zeros), the act() of one k-point with npol = 1."""
    lib = _load()
    if not hasattr(lib, "_nl_ready"):
        pi = C.POINTER(C.c_int)
        lib.ref_nonlocal_act.argtypes = [C.c_int, pi, pi, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                         C.c_char_p, C.c_int]
        lib.ref_nonlocal_act.restype = C.c_int
        lib._nl_ready = True
    na_a = np.ascontiguousarray(na, dtype=np.int32)
    nh_a = np.ascontiguousarray(nh, dtype=np.int32)
    v = np.ascontiguousarray(vkb, dtype=np.complex128)
    d = np.ascontiguousarray(deeq, dtype=np.float64)
    x = np.ascontiguousarray(psi, dtype=np.complex128)
    out = np.zeros_like(x) if hpsi is None else np.ascontiguousarray(hpsi, dtype=np.complex128).copy()
    nb, ld = x.shape
    err = C.create_string_buffer(512)
    pi = C.POINTER(C.c_int)
    rc = lib.ref_nonlocal_act(len(na_a), na_a.ctypes.data_as(pi), nh_a.ctypes.data_as(pi), v.shape[0], v.shape[1],
                              v.ctypes.data, d.shape[0], d.shape[1], d.shape[2], d.ctypes.data_as(C.POINTER(C.c_double)),
                              nb, int(npw), ld, x.ctypes.data, out.ctypes.data, err, 512)
    if rc != 0:
        raise RuntimeError("reference Nonlocal::act failed: " + err.value.decode())
    return out
