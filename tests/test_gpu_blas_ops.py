"""The FP64 BLAS functor drop-ins (gemm_op, gemv_op, dot_real_op of math_kernel_op.h) on the device against
numpy on the same column-major buffers; their argument checks on CPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest


def test_blas_ops_reject_bad_arguments_without_gpu_calls(pkg):
    lib = pkg._lib.load()
    one = (C.c_double * 2)(1.0, 0.0)
    fake = C.c_void_p(16)
    assert lib.b200_gemm_op_f64(b"X", b"N", 2, 2, 2, one, fake, 2, fake, 2, one, fake, 2, None) == 1
    assert b"trans" in lib.b200_last_error()
    assert lib.b200_gemm_op_f64(b"N", b"N", -1, 2, 2, one, fake, 2, fake, 2, one, fake, 2, None) == 1
    assert lib.b200_gemv_op_f64(b"N", 2, 2, one, fake, 2, fake, 0, one, fake, 1, None) == 1
    res = C.c_double()
    assert lib.b200_dot_real_op_f64(4, None, fake, 0, C.byref(res), None) == 1


def _dev(torch, a):
    """A numpy matrix as a flat device buffer in column-major order."""
    return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).cuda()


def _host(t, shape):
    return t.cpu().numpy().reshape(shape, order="F")


@pytest.mark.gpu
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("C", "N"), ("N", "T"), ("T", "C")])
def test_gemm_op_f64(pkg, ta, tb):
    torch = pytest.importorskip("torch")
    lib = pkg._lib.load()
    rng = np.random.default_rng(3)
    m, n, k = 37, 23, 51
    def op(x, t):
        return x if t == "N" else (x.T if t == "T" else x.conj().T)
    a = rng.standard_normal((m, k) if ta == "N" else (k, m)) + 1j * rng.standard_normal((m, k) if ta == "N" else (k, m))
    b = rng.standard_normal((k, n) if tb == "N" else (n, k)) + 1j * rng.standard_normal((k, n) if tb == "N" else (n, k))
    c = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    al, be = 0.7 - 0.2j, -0.3 + 0.5j
    ad, bd, cd = _dev(torch, a), _dev(torch, b), _dev(torch, c)
    alpha = (C.c_double * 2)(al.real, al.imag)
    beta = (C.c_double * 2)(be.real, be.imag)
    rc = lib.b200_gemm_op_f64(ta.encode(), tb.encode(), m, n, k, alpha, ad.data_ptr(), a.shape[0], bd.data_ptr(),
                              b.shape[0], beta, cd.data_ptr(), m, None)
    assert rc == 0, lib.b200_last_error()
    torch.cuda.synchronize()
    ref = al * (op(a, ta) @ op(b, tb)) + be * c
    assert np.max(np.abs(_host(cd, (m, n)) - ref)) < 1e-12 * np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("t", ["N", "C"])
def test_gemv_op_f64(pkg, t):
    torch = pytest.importorskip("torch")
    lib = pkg._lib.load()
    rng = np.random.default_rng(5)
    m, n = 41, 29
    a = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    x = rng.standard_normal(n if t == "N" else m) + 1j * rng.standard_normal(n if t == "N" else m)
    y = rng.standard_normal(m if t == "N" else n) + 1j * rng.standard_normal(m if t == "N" else n)
    al, be = 1.1 + 0.3j, 0.4 - 0.1j
    ad, xd, yd = _dev(torch, a), torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    alpha = (C.c_double * 2)(al.real, al.imag)
    beta = (C.c_double * 2)(be.real, be.imag)
    rc = lib.b200_gemv_op_f64(t.encode(), m, n, alpha, ad.data_ptr(), m, xd.data_ptr(), 1, beta, yd.data_ptr(), 1,
                              None)
    assert rc == 0, lib.b200_last_error()
    torch.cuda.synchronize()
    ref = al * ((a if t == "N" else a.conj().T) @ x) + be * y
    assert np.max(np.abs(yd.cpu().numpy() - ref)) < 1e-12 * np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [1, 1000, 1 << 20])
def test_dot_real_op(pkg, dim):
    torch = pytest.importorskip("torch")
    lib = pkg._lib.load()
    rng = np.random.default_rng(dim)
    lh = rng.standard_normal(dim) + 1j * rng.standard_normal(dim)
    rh = rng.standard_normal(dim) + 1j * rng.standard_normal(dim)
    ref = np.vdot(lh, rh).real
    l64, r64 = torch.from_numpy(lh).cuda(), torch.from_numpy(rh).cuda()
    res = C.c_double()
    assert lib.b200_dot_real_op_f64(dim, l64.data_ptr(), r64.data_ptr(), 1, C.byref(res), None) == 0
    assert abs(res.value - ref) <= 1e-12 * (np.sum(np.abs(lh) * np.abs(rh)) + 1e-300)
    res2 = C.c_double()
    assert lib.b200_dot_real_op_f64(dim, l64.data_ptr(), r64.data_ptr(), 1, C.byref(res2), None) == 0
    assert res2.value == res.value  # deterministic
    l32, r32 = l64.to(torch.complex64), r64.to(torch.complex64)
    res32 = C.c_float()
    assert lib.b200_dot_real_op_f32(dim, l32.data_ptr(), r32.data_ptr(), 1, C.byref(res32), None) == 0
    ref32 = np.vdot(lh.astype(np.complex64).astype(np.complex128), rh.astype(np.complex64).astype(np.complex128)).real
    assert abs(res32.value - ref32) <= 1e-6 * (np.sum(np.abs(lh) * np.abs(rh)) + 1e-30)
