"""The FP64 complex GEMM on the int8 tensor cores (exact modular emulation, b200_zgemm_i8).

CPU: the library's recombination constants against Python integers, and a numpy model of the whole
scheme built on those constants (power-of-two scaling by row / column maxima, symmetric residues, one exact
integer product per modulus, the floating-point recombination of the kernel) against exact rational
products.  GPU: the device GEMM against numpy's FP64 product, to a few ulps of every entry on
integer-valued inputs, and within FP64 rounding (relative to |op(A)| |B|) on random ones; NaN
propagation; the K split path.
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np
import pytest

MODS16 = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193]


def _bigint_constants(n):
    ms = MODS16[:n]
    M = 1
    for m in ms:
        M *= m
    wa, wb = [], []
    for m in ms:
        Ml = M // m
        w = (Ml * pow(Ml % m, -1, m)) % M
        a = (w << 40) // M
        wa.append(a / 2.0**40)
        wb.append(float(Fraction(w, M) - Fraction(a, 1 << 40)))
    return ms, M, wa, wb


@pytest.mark.parametrize("n", [12, 14, 16])
@pytest.mark.parametrize("kr", [1, 1024, 103254, 248578])
def test_constants_match_integers(pkg, n, kr):
    mods, wa, wb, mprod, q = pkg.pwdft.zgemm_i8_constants(n, kr)
    ms, M, wa_ref, wb_ref = _bigint_constants(n)
    assert mods == ms
    assert wa == wa_ref  # 40-bit prefixes: exact
    np.testing.assert_allclose(wb, wb_ref, rtol=1e-15, atol=0)
    assert mprod == float(M)
    assert q == math.floor((math.log2(M) - 2 - math.log2(kr)) / 2)
    assert kr * 4.0**q * 4 <= M  # |C'| <= K' 2^2q <= M / 4


def _model(A, B, n, pkg):
    """numpy restatement of the device scheme for real C = A @ B (A: rows x K', B: K' x cols)."""
    kr = A.shape[1]
    mods, wa, wb, mprod, q = pkg.pwdft.zgemm_i8_constants(n, kr)

    def exps(mx):
        e = np.zeros(mx.shape, dtype=np.int64)
        nz = mx > 0
        e[nz] = q - np.frexp(mx[nz])[1]
        return e

    ea = exps(np.abs(A).max(axis=1))
    eb = exps(np.abs(B).max(axis=0))
    Ai = np.rint(np.ldexp(A, ea[:, None])).astype(np.int64)
    Bi = np.rint(np.ldexp(B, eb[None, :])).astype(np.int64)
    assert np.abs(Ai).max() < 2**62 and np.abs(Bi).max() < 2**62
    s = np.zeros((A.shape[0], B.shape[1]))
    t = np.zeros_like(s)
    for m, a, b in zip(mods, wa, wb):
        ra = np.mod(Ai, m)
        ra = np.where(ra > (m - 1) // 2, ra - m, ra)
        rb = np.mod(Bi, m)
        rb = np.where(rb > (m - 1) // 2, rb - m, rb)
        assert np.abs(ra).max() <= 128 and np.abs(rb).max() <= 128
        P = ra @ rb  # exact: |P| <= 128^2 K' < 2^31 for K' <= 130944
        c = np.mod(P, m).astype(np.float64)
        s = s + c * a  # exact: 40 fraction bits, integer part below 2^12
        t = t + c * b
    x = s - np.rint(s)
    x = x + t
    x = x - np.rint(x)
    return np.ldexp(x * mprod, -(ea[:, None] + eb[None, :])), (Ai, Bi, ea, eb)


def _exact(A, B):
    out = np.zeros((A.shape[0], B.shape[1]))
    for i in range(A.shape[0]):
        for j in range(B.shape[1]):
            out[i, j] = float(sum(Fraction(float(a)) * Fraction(float(b)) for a, b in zip(A[i], B[:, j])))
    return out


@pytest.mark.parametrize("n", [14, 16])
def test_scheme_model_matches_exact_products(pkg, n):
    rng = np.random.default_rng(7 + n)
    K = 2000
    # decaying rows / columns, one zero row, widely different scales
    A = rng.standard_normal((5, K)) * np.exp(-10.0 * np.arange(K) / K)[None, :]
    A[1] *= 1e-200
    A[2] = 0.0
    A[3] *= 1e250
    B = rng.standard_normal((K, 4)) * np.exp(-8.0 * np.arange(K) / K)[:, None]
    B[:, 1] *= 1e-30
    C, _ = _model(A, B, n, pkg)
    E = _exact(A, B)
    bound = np.abs(A) @ np.abs(B)
    err = np.abs(C - E) / np.where(bound > 0, bound, 1.0)
    assert np.all(C[2] == 0.0)
    # FP64-level: a plain FP64 dot product's error bar is K eps relative to |a||b|
    assert err.max() < 2e-16 * math.sqrt(K) * (4 if n == 14 else 1), err.max()


def test_scheme_model_worst_case_range(pkg):
    # every entry at its row maximum with one sign: |C'| reaches K' 2^2q, the top of the recoverable range
    K = 130944
    A = np.full((2, K), 0.75)
    A[1] *= -1.0
    B = np.full((K, 2), 0.6)
    C, (Ai, Bi, ea, eb) = _model(A, B, 16, pkg)
    exact = (Ai[:, :1].astype(object) * int(Bi[0, 0])) * K
    for i in range(2):
        got = Fraction(C[i, 0]) * Fraction(2) ** int(ea[i] + eb[0])
        assert abs(got - int(exact[i, 0])) <= abs(int(exact[i, 0])) * Fraction(1, 2**50)
    np.testing.assert_allclose(C[:, 0], [0.45 * K, -0.45 * K], rtol=1e-15)


# ---------------------------------------------------------------------------------------------- GPU

CASES = [
    # transa, M, N, K, lda_pad, alpha, beta
    ("N", 100, 40, 37, 0, 1.0, 0.0),
    ("C", 64, 70, 5000, 3, 0.5 - 1.5j, 2.0 + 0.5j),
    ("N", 3000, 160, 512, 0, 1.0, 1.0),
    # B' resident in shared memory with fewer K blocks; a last column tile partly empty
    ("N", 1500, 160, 384, 0, 1.0, 0.5),
    ("N", 1000, 150, 512, 2, 1.0 - 0.5j, 0.0),
    ("C", 512, 160, 51627, 0, 1.0, 0.0),
    ("C", 33, 17, 129, 1, 1.0j, -1.0),
    ("N", 1, 1, 1, 1, 1.0, 0.0),
    ("N", 2100, 133, 77, 5, -0.5, 1.0 + 1.0j),
    # K' = 2K above one split's exact int32 range: several K splits
    ("C", 96, 24, 140001, 0, 1.0, 0.0),
]


def _cplx(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _run(pkg, torch, ta, M, N, K, lda, A_store, B_store, C_store, alpha, beta, ldb, ldc, nmods=16):
    ad, bd, cd = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (A_store, B_store, C_store))
    pkg.pwdft.zgemm_i8(ta, M, N, K, alpha, ad, lda, bd, ldb, beta, cd, ldc, nmods=nmods)
    torch.cuda.synchronize()
    assert pkg.pwdft.zgemm_i8_error() == 0
    return cd.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
def test_zgemm_i8_matches_fp64(pkg, case):
    torch = pytest.importorskip("torch")
    ta, M, N, K, pad, alpha, beta = CASES[case]
    rng = np.random.default_rng(300 + case)
    rows_a = M if ta == "N" else K
    cols_a = K if ta == "N" else M
    lda, ldb, ldc = rows_a + pad, K + 1, M + 2
    A_store = _cplx(rng, cols_a, lda)
    B_store = _cplx(rng, N, ldb)
    C_store = _cplx(rng, N, ldc)
    A = A_store[:, :rows_a].T
    opA = A if ta == "N" else A.conj().T
    Bm = B_store[:, :K].T
    C0 = C_store[:, :M].T
    ref = alpha * (opA @ Bm) + beta * C0
    out_store = _run(pkg, torch, ta, M, N, K, lda, A_store, B_store, C_store, alpha, beta, ldb, ldc)
    assert np.array_equal(out_store[:, M:], C_store[:, M:])  # padding rows of C untouched
    out = out_store[:, :M].T
    bound = abs(alpha) * (np.abs(opA) @ np.abs(Bm)) + abs(beta) * np.abs(C0)
    err = np.abs(out - ref) / bound
    # numpy's FP64 product is itself off by ~sqrt(K) eps: the bar is FP64 rounding of a length-K sum
    assert err.max() < 4e-16 * math.sqrt(K) + 4e-16, err.max()


@pytest.mark.gpu
@pytest.mark.parametrize("ta", ["N", "C"])
def test_zgemm_i8_integer_inputs_to_ulps(pkg, ta):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(11)
    M, N, K = 300, 50, 4000
    A_store = rng.integers(-1000, 1000, (K if ta == "N" else M, M if ta == "N" else K)) + 1j * rng.integers(
        -1000, 1000, (K if ta == "N" else M, M if ta == "N" else K))
    B_store = rng.integers(-1000, 1000, (N, K)) + 1j * rng.integers(-1000, 1000, (N, K))
    C_store = np.zeros((N, M), dtype=np.complex128)
    A = A_store.T
    opA = A if ta == "N" else A.conj().T
    ref = opA @ B_store.T  # exact: integers below 2^53
    out = _run(pkg, torch, ta, M, N, K, A.shape[0], A_store.astype(np.complex128), B_store.astype(np.complex128),
               C_store, 1.0, 0.0, K, M)
    # integer inputs are scaled without rounding: only the recombination's few roundings remain, relative to
    # each entry (a zero entry comes out exactly zero)
    assert np.all(np.abs(out.T - ref) <= 8 * 2.0**-53 * np.abs(ref))


@pytest.mark.gpu
def test_zgemm_i8_nan_rows_and_zero_blocks(pkg):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    M, N, K = 200, 30, 700
    A_store = _cplx(rng, K, M)  # 'N': A is M x K -> storage K columns of M
    A_store[10, 7] = np.nan  # row 7 of A
    A_store[:, 20] = 0.0  # row 20 of A is zero
    B_store = _cplx(rng, N, K)
    B_store[3, 100] = np.inf  # column 3 of B
    C_store = np.full((N, M), np.nan + 0j)  # beta = 0: C must not be read
    out = _run(pkg, torch, "N", M, N, K, M, A_store, B_store, C_store, 1.0, 0.0, K, M).T
    bad = np.zeros((M, N), dtype=bool)
    bad[7, :] = True
    bad[:, 3] = True
    assert np.all(np.isnan(out[bad]))
    assert np.all(np.isfinite(out[~bad]))
    assert np.all(out[20, [j for j in range(N) if j != 3]] == 0)
    ref = A_store.T @ B_store.T
    ok = ~bad
    bound = (np.abs(A_store.T) @ np.abs(B_store.T))[ok]
    assert (np.abs(out[ok] - ref[ok]) / np.where(bound > 0, bound, 1)).max() < 1e-14


@pytest.mark.gpu
def test_zgemm_i8_repeated_calls_agree(pkg):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(9)
    M, N, K = 1000, 64, 3000
    A_store = _cplx(rng, M, K)  # 'C': A is K x M
    B_store = _cplx(rng, N, K)
    C_store = np.zeros((N, M), dtype=np.complex128)
    o1 = _run(pkg, torch, "C", M, N, K, K, A_store, B_store, C_store, 1.0, 0.0, K, M)
    o2 = _run(pkg, torch, "C", M, N, K, K, A_store, B_store, C_store, 1.0, 0.0, K, M)
    assert np.array_equal(o1, o2)


@pytest.mark.gpu
@pytest.mark.parametrize("nmods", [12, 14])
def test_zgemm_i8_fewer_moduli(pkg, nmods):
    """Fewer moduli, smaller scale exponent q: the error stays within the rounding of op(A) and B to q bits."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(40 + nmods)
    M, N, K = 200, 30, 3000
    A_store = _cplx(rng, M, K)  # 'C': A is K x M
    B_store = _cplx(rng, N, K)
    C_store = np.zeros((N, M), dtype=np.complex128)
    out = _run(pkg, torch, "C", M, N, K, K, A_store, B_store, C_store, 1.0, 0.0, K, M, nmods=nmods).T
    ref = A_store.conj() @ B_store.T
    q = pkg.pwdft.zgemm_i8_constants(nmods, 2 * K)[4]
    amax = np.maximum(np.abs(A_store.real), np.abs(A_store.imag)).max(axis=1)[:, None]
    bmax = np.maximum(np.abs(B_store.real), np.abs(B_store.imag)).max(axis=1)[None, :]
    # each of the 2K products carries the two operands' roundings (half a unit of 2^-q of the row maximum)
    bar = 2.0 * 2 * K * 2.0 ** -q * amax * bmax
    assert np.all(np.abs(out - ref) <= bar)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [("C", 512, 160, 6000), ("N", 3000, 160, 512)])
def test_zgemm_i8_wait_runout_reports_and_recovers(pkg, shape):
    """The GEMM kernel's bounded waits (streamed and shared-memory-resident B'): with a limit no pipeline can meet
    (1 ns) the kernel gives up, drains its own copies and MMAs, frees its tensor memory and sets the error word,
    which the host reads (and the read clears); the next product with the default limit is correct."""
    torch = pytest.importorskip("torch")
    P = pkg.pwdft
    ta, M, N, K = shape
    rng = np.random.default_rng(17)
    A_store = _cplx(rng, M, K) if ta == "C" else _cplx(rng, K, M)
    lda = K if ta == "C" else M
    B_store = _cplx(rng, N, K)
    ad, bd = torch.from_numpy(A_store).cuda(), torch.from_numpy(B_store).cuda()
    cd = torch.zeros((N, M), dtype=torch.complex128, device="cuda")
    assert P.zgemm_i8_error() == 0
    try:
        P.tc_set_wait_limit_ns(1)
        P.zgemm_i8(ta, M, N, K, 1.0, ad, lda, bd, K, 0.0, cd, M)
        torch.cuda.synchronize()
    finally:
        P.tc_set_wait_limit_ns(0)
    assert P.zgemm_i8_error() != 0, "a 1 ns wait limit should have run out"
    assert P.zgemm_i8_error() == 0, "the read clears the error word"
    P.zgemm_i8(ta, M, N, K, 1.0, ad, lda, bd, K, 0.0, cd, M)
    torch.cuda.synchronize()
    assert P.zgemm_i8_error() == 0
    A = A_store.T
    opA = A if ta == "N" else A.conj().T
    ref = opA @ B_store.T
    bound = np.abs(opA) @ np.abs(B_store.T)
    assert (np.abs(cd.cpu().numpy().T - ref) / bound).max() < 4e-16 * np.sqrt(K) + 4e-16
