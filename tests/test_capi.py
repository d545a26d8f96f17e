"""CPU tests of the C-ABI library: it loads, exports every declared entry point,
and its host-side plane-wave basis set-up matches the oracle index for index."""
from __future__ import annotations

import ctypes
import subprocess

import numpy as np
import pytest

from oracle.pw_basis_ref import PWBasisKRef


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg._lib.load()
    declared = pkg._lib.header_symbols()
    assert len(declared) >= 40
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(pkg._lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    assert set(pkg._lib._SIGS) == set(declared)


def test_version_and_error_without_gpu_calls(pkg):
    lib = pkg._lib.load()
    assert b"sm_100a" in lib.b200_version()
    # invalid arguments are reported as a status, never an exit
    rc = lib.b200_pw_basis_create(-1.0, None, 0.0, 0.0, 0, 0, 0, 0, None, ctypes.byref(ctypes.c_void_p()))
    assert rc == 1
    assert b"NULL" in lib.b200_last_error() or b"invalid" in lib.b200_last_error()


CELLS = [
    (10.26, np.eye(3), 30.0, np.zeros((1, 3)), None),
    (5.13, np.eye(3), 30.0, np.zeros((1, 3)), None),
    (10.26, np.diag([1.0, 1.0, 2.0]), 40.0, np.zeros((1, 3)), None),
    (10.26, np.eye(3), 30.0, np.array([[0.125, -0.375, 0.375], [0.375, 0.375, -0.125], [-0.125, 0.125, 0.125]]), None),
    (7.0, np.array([[1.0, 0.0, 0.0], [0.5, 0.8660254037844386, 0.0], [0.0, 0.0, 1.6]]), 20.0,
     np.array([[0.1, 0.2, 0.3]]), None),
    (10.26, np.eye(3), 30.0, np.zeros((1, 3)), (40, 40, 40)),
]


@pytest.mark.parametrize("case", range(len(CELLS)))
def test_host_basis_matches_oracle(pkg, case):
    lat0, lv, ec, kd, grid = CELLS[case]
    ref = PWBasisKRef(lat0, lv, ec, kd, grid=grid)
    b = pkg.pwdft.PWBasisK(lat0, lv, ec, kd, grid=grid)
    assert (b.nx, b.ny, b.nz) == (ref.nx, ref.ny, ref.nz)
    assert b.nst == ref.nst and b.npw == ref.npw
    assert np.array_equal(b.npwk, ref.npwk)
    assert b.npwk_max == ref.npwk_max
    assert abs(b.tpiba2 - ref.tpiba2) < 1e-14 and abs(b.omega - ref.omega) < 1e-9 * ref.omega
    for ik in range(len(kd)):
        assert np.array_equal(b.ig2ixyz(ik), ref.ig2ixyz(ik))
        np.testing.assert_allclose(b.gk2_k(ik), ref.gk2_k(ik), rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(b.gplusk_cart(ik), ref.gplusk_cart(ik), rtol=1e-13, atol=1e-13)


def test_host_basis_rejects_bad_input(pkg):
    with pytest.raises(pkg._lib.B200Error):
        pkg.pwdft.PWBasisK(10.0, np.zeros((3, 3)), 30.0, np.zeros((1, 3)))
    with pytest.raises(pkg._lib.B200Error):
        pkg.pwdft.PWBasisK(10.0, np.eye(3), -1.0, np.zeros((1, 3)))


def test_solver_entry_points_reject_bad_arguments_without_gpu_calls(pkg):
    """The Diago_DavSubspace and DiagoBPCG entry points check their arguments before any device call; a bad
    one is a B200_STATUS_INVALID_ARGUMENT status with a message, never an exit."""
    lib = pkg._lib.load()
    out = ctypes.c_void_p()
    fake = ctypes.c_void_p(16)  # never dereferenced: every call below fails its checks first
    no_cb = pkg._lib.HPSI_CB()  # a NULL callback
    cases = [
        (lib.b200_dav_subspace_create, (4, 100, 2, 1e-9, 50, 0, None, ctypes.byref(out)), b"NULL"),
        (lib.b200_dav_subspace_create, (4, 10, 3, 1e-9, 50, 0, fake, ctypes.byref(out)), b"david_ndim"),
        (lib.b200_dav_subspace_create, (4, 100, 2, 1e-9, 0, 0, fake, ctypes.byref(out)), b"diag_nmax"),
        (lib.b200_dav_subspace_diag, (None, no_cb, None, fake, 100, None, None, 0, None), b"NULL"),
        (lib.b200_dav_subspace_diag_hamilt, (None, None, 0, 0, fake, 100, None, None, 0, None), b"NULL"),
        (lib.b200_dav_subspace_set_stream, (None, None), b"NULL"),
        (lib.b200_dav_subspace_stats, (None, None, None), b"NULL"),
        (lib.b200_bpcg_create, (None, 4, 100, ctypes.byref(out)), b"NULL"),
        (lib.b200_bpcg_create, (fake, 8, 4, ctypes.byref(out)), b"nband"),
        (lib.b200_bpcg_diag, (None, no_cb, None, fake, None, 1, None), b"NULL"),
        (lib.b200_bpcg_diag_hamilt, (None, None, 0, 0, fake, None, 1, None), b"NULL"),
        (lib.b200_bpcg_set_stream, (None, None), b"NULL"),
        (lib.b200_bpcg_stats, (None, None, None), b"NULL"),
        (lib.b200_david_set_fp64_gemm, (None, 1), b"NULL"),
        (lib.b200_server_set_express, (None, 1, 0.03), b"NULL"),
    ]
    for fn, args, msg in cases:
        assert fn(*args) == 1, fn.__name__
        assert msg in lib.b200_last_error(), (fn.__name__, lib.b200_last_error())
    assert out.value is None  # nothing was created
