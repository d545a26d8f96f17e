"""GPU parity of the tcgen05 split-precision complex GEMM (gemm_op<complex<float>, GPU> on tensor cores).

Checked against a complex128 product of the same FP32 inputs; the bar is the
accuracy of a plain FP32 GEMM (cuBLAS CGEMM on the same inputs, via torch),
since 3xTF32 is meant to be FP32-accurate: error <= 3 x CGEMM's error + 3e-7.
Integer-valued inputs (exact products and sums) must give bit-exact results.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = [
    # transa, M, N, K, lda_pad, alpha, beta
    ("N", 100, 40, 37, 0, 1.0, 0.0),
    ("C", 64, 70, 5000, 2, 0.5 - 1.5j, 2.0 + 0.5j),
    ("N", 3000, 160, 512, 0, 1.0, 1.0),
    ("C", 512, 160, 51626, 2, 1.0, 0.0),
    ("C", 33, 17, 129, 1, 1.0j, -1.0),
    ("N", 1, 1, 1, 1, 1.0, 0.0),
    # many M tiles: B split once in HBM ("C" and "N", odd K, ragged N)
    ("C", 1100, 90, 3001, 2, 1.0 - 1.0j, 0.5j),
    ("N", 2100, 33, 77, 1, -0.5, 1.0 + 1.0j),
]


def cplx(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_tc_cgemm_matches_fp64(pkg, case):
    ta, M, N, K, pad, alpha, beta = CASES[case]
    rng = np.random.default_rng(100 + case)
    rows_a = M if ta == "N" else K
    cols_a = K if ta == "N" else M
    lda = rows_a + pad
    lda += lda % 2
    ldb = K + (K % 2)
    ldc = M + 3
    A_store = cplx(rng, cols_a, lda)  # column-major rows_a x cols_a, leading dimension lda
    B_store = cplx(rng, N, ldb)
    C_store = cplx(rng, N, ldc)
    A = A_store[:, :rows_a].T  # rows_a x cols_a
    opA = A if ta == "N" else A.conj().T
    Bm = B_store[:, :K].T
    C0 = C_store[:, :M].T
    ref = alpha * (opA.astype(np.complex128) @ Bm.astype(np.complex128)) + beta * C0.astype(np.complex128)
    ad, bd, cd = (torch.from_numpy(x.copy()).cuda() for x in (A_store, B_store, C_store))
    pkg.pwdft.tc_cgemm(ta, M, N, K, alpha, ad, lda, bd, ldb, beta, cd, ldc)
    torch.cuda.synchronize()
    assert pkg.pwdft.tc_cgemm_error() == 0
    out = cd.cpu().numpy()[:, :M].T
    # padding rows of C untouched
    assert np.array_equal(cd.cpu().numpy()[:, M:], C_store[:, M:])
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    # plain FP32 GEMM of the same inputs as the accuracy bar
    f32 = alpha * (torch.from_numpy(opA.copy()).cuda() @ torch.from_numpy(Bm.copy()).cuda()).cpu().numpy() + beta * C0
    err32 = np.linalg.norm(f32 - ref) / np.linalg.norm(ref)
    assert err <= 3 * err32 + 3e-7, (err, err32)


def test_tc_cgemm_rejects_odd_leading_dimension(pkg):
    a = torch.zeros(8 * 9, dtype=torch.complex64, device="cuda")
    with pytest.raises(pkg._lib.B200Error):
        pkg.pwdft.tc_cgemm("N", 9, 8, 8, 1.0, a, 9, a, 8, 0.0, a, 9)


@pytest.mark.parametrize("ta,M,N,K", [("C", 512, 160, 51626), ("N", 1000, 160, 3000), ("C", 33, 17, 129)])
def test_tc_cgemm_integer_inputs_exact(pkg, ta, M, N, K):
    """Small integers: every product and partial sum is exact in FP32, so any tiling, expansion or
    pipelining slip shows up as a nonzero difference."""
    rng = np.random.default_rng(7)
    rows_a = M if ta == "N" else K
    cols_a = K if ta == "N" else M
    lda = rows_a + rows_a % 2
    ldb = K + K % 2
    A_store = (rng.integers(-8, 9, (cols_a, lda)) + 1j * rng.integers(-8, 9, (cols_a, lda))).astype(np.complex64)
    B_store = (rng.integers(-8, 9, (N, ldb)) + 1j * rng.integers(-8, 9, (N, ldb))).astype(np.complex64)
    A = A_store[:, :rows_a].T
    opA = A if ta == "N" else A.conj().T
    ref = opA.astype(np.complex128) @ B_store[:, :K].T.astype(np.complex128)
    cd = torch.zeros((N, M), dtype=torch.complex64, device="cuda")
    pkg.pwdft.tc_cgemm(ta, M, N, K, 1.0, torch.from_numpy(A_store).cuda(), lda, torch.from_numpy(B_store).cuda(), ldb,
                       0.0, cd, M)
    torch.cuda.synchronize()
    assert np.array_equal(cd.cpu().numpy().T.astype(np.complex128), ref)


def test_tc_cgemm_wait_runout_reports_and_recovers(pkg):
    """The kernel's bounded waits: with a limit no pipeline can meet (1 ns) a GEMM gives up, drains its own
    copies and MMAs, frees its tensor memory and sets the error word, which the host reads (and which the read
    clears); the context stays usable and the next GEMM with the default limit is correct."""
    P = pkg.pwdft
    rng = np.random.default_rng(7)
    M, N, K = 512, 160, 6000
    A = cplx(rng, M, K)  # column-major K x M (op 'C')
    B = cplx(rng, N, K)
    ad, bd = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    cd = torch.zeros((N, M), dtype=torch.complex64, device="cuda")
    assert P.tc_cgemm_error() == 0
    try:
        P.tc_set_wait_limit_ns(1)
        P.tc_cgemm("C", M, N, K, 1.0, ad, K, bd, K, 0.0, cd, M)
        torch.cuda.synchronize()
    finally:
        P.tc_set_wait_limit_ns(0)
    code = P.tc_cgemm_error()
    assert code != 0, "a 1 ns wait limit should have run out"
    assert P.tc_cgemm_error() == 0, "the read clears the error word"
    P.tc_cgemm("C", M, N, K, 1.0, ad, K, bd, K, 0.0, cd, M)
    torch.cuda.synchronize()
    assert P.tc_cgemm_error() == 0
    ref = A.astype(np.complex128).conj() @ B.astype(np.complex128).T  # (M, N)
    out = cd.cpu().numpy().T
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err < 1e-6, err
