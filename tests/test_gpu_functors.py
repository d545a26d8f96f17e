"""GPU parity of the op functors against the reference's golden vectors and the oracle.

Mirrors ekinetic_op_test.cpp, veff_op_test.cpp, nonlocal_op_test.cpp and
pw_op_test.cpp (same inputs, same tolerances), then checks random inputs
bit-for-bit (FP64) against the oracle restatement of the CPU functors.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import hamilt_ref as H

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_ekinetic_golden(pkg, golden):
    g = golden("ekinetic_op")
    P = pkg.pwdft
    hpsi = dev(np.zeros_like(g["expected_hpsi"]))
    P.ekinetic_pw_op(int(g["band"]), int(g["dim"]), int(g["dim"]), float(g["tpiba2"]), dev(g["gk2"]), hpsi, dev(g["psi"]))
    assert np.max(np.abs(host(hpsi) - g["expected_hpsi"])) < 1e-6
    # FP32 instantiation
    hpsi32 = dev(np.zeros_like(g["expected_hpsi"]).astype(np.complex64))
    P.ekinetic_pw_op(int(g["band"]), int(g["dim"]), int(g["dim"]), float(g["tpiba2"]), dev(g["gk2"].astype(np.float32)),
                     hpsi32, dev(g["psi"].astype(np.complex64)))
    assert np.max(np.abs(host(hpsi32) - g["expected_hpsi"])) < 1e-5


def test_ekinetic_random_exact(pkg):
    rng = np.random.default_rng(1)
    nb, npw, ld = 7, 1001, 1010
    gk2 = rng.random(npw) * 40
    psi = rng.standard_normal(nb * ld) + 1j * rng.standard_normal(nb * ld)
    h0 = rng.standard_normal(nb * ld) + 1j * rng.standard_normal(nb * ld)
    ref = h0.copy()
    H.ekinetic_pw_op(nb, npw, ld, 0.375, gk2, ref, psi)
    hd = dev(h0)
    pkg.pwdft.ekinetic_pw_op(nb, npw, ld, 0.375, dev(gk2), hd, dev(psi))
    assert np.max(np.abs(host(hd) - ref)) <= 1e-14 * np.max(np.abs(ref))


def test_veff_golden(pkg, golden):
    g = golden("veff_op")
    n = int(g["size"])
    out = dev(g["out"])
    pkg.pwdft.veff_pw_op(n, out, dev(g["vin"]))
    assert np.max(np.abs(host(out) - g["expected_out"])) < 6e-5
    o, o1 = dev(g["out_spin"]), dev(np.zeros_like(g["out_spin"]))
    vin = [dev(g["in_spin"][i * n:(i + 1) * n]) for i in range(4)]
    pkg.pwdft.veff_pw_op_npol2(n, o, o1, vin)
    assert np.max(np.abs(host(o) - g["expected_out_spin"])) < 7.5e-5
    assert np.max(np.abs(host(o1))) < 6e-5


def test_veff_npol2_random_exact(pkg):
    rng = np.random.default_rng(2)
    n = 5000
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    v = [rng.standard_normal(n) for _ in range(4)]
    ra, rb = a.copy(), b.copy()
    H.veff_pw_op_npol2(n, ra, rb, v)
    da, db = dev(a), dev(b)
    pkg.pwdft.veff_pw_op_npol2(n, da, db, [dev(x) for x in v])
    assert np.max(np.abs(host(da) - ra)) < 1e-13 and np.max(np.abs(host(db) - rb)) < 1e-13


def test_nonlocal_golden(pkg, golden):
    g = golden("nonlocal_op")
    ps = dev(np.zeros_like(g["expected_ps"]))
    s, i = pkg.pwdft.nonlocal_pw_op(int(g["l1"]), int(g["l2"]), int(g["l3"]), 0, 0, int(g["spin"]), int(g["nkb"]),
                                    int(g["deeq_x"]), int(g["deeq_y"]), int(g["deeq_z"]), dev(g["deeq"]), ps,
                                    dev(g["becp"]))
    assert np.max(np.abs(host(ps) - g["expected_ps"])) < 5e-6
    assert (s, i) == (int(g["expected_sum"]), int(g["expected_iat"]))
    ps = dev(np.zeros_like(g["expected_ps_spin"]))
    s, i = pkg.pwdft.nonlocal_pw_op_nc(int(g["l1"]), int(g["l2_spin"]), int(g["l3"]), 0, 0, int(g["nkb"]),
                                       int(g["deeq_x"]), int(g["deeq_y"]), int(g["deeq_z"]), dev(g["deeq_spin"]), ps,
                                       dev(g["becp_spin"]))
    assert np.max(np.abs(host(ps) - g["expected_ps_spin"])) < 5e-6
    assert (s, i) == (int(g["expected_sum"]), int(g["expected_iat"]))


def test_nonlocal_random_block_d(pkg):
    """Full (non-diagonal) nh x nh D blocks, two atom types, spin 1 of 2."""
    rng = np.random.default_rng(3)
    na, nh, nb = [3, 2], [4, 6], 5
    nkb = sum(a * h for a, h in zip(na, nh))
    nat, nhm = sum(na), max(nh)
    deeq = rng.standard_normal((2, nat, nhm, nhm))
    becp = rng.standard_normal(nkb * nb) + 1j * rng.standard_normal(nkb * nb)
    ref = np.zeros(nkb * nb, dtype=np.complex128)
    s, i = 0, 0
    for it in range(2):
        s, i = H.nonlocal_pw_op(na[it], nb, nh[it], s, i, 1, nkb, nat, nhm, nhm, deeq, ref, becp)
    ps = dev(np.zeros(nkb * nb, dtype=np.complex128))
    dd, db = dev(deeq), dev(becp)
    s2, i2 = 0, 0
    for it in range(2):
        s2, i2 = pkg.pwdft.nonlocal_pw_op(na[it], nb, nh[it], s2, i2, 1, nkb, nat, nhm, nhm, dd, ps, db)
    assert (s2, i2) == (s, i)
    assert np.max(np.abs(host(ps) - ref)) < 1e-13


def test_pw_ops_golden(pkg, golden):
    g = golden("pw_op")
    P = pkg.pwdft
    npwk, nxyz = int(g["npwk"]), int(g["nxyz"])
    idx = dev(g["box_index"].astype(np.int32))
    out = dev(np.zeros(nxyz, dtype=np.complex128))
    P.set_3d_fft_box_op(npwk, idx, dev(g["in_1"]), out)
    assert np.max(np.abs(host(out) - g["out_1"])) < 1e-12
    out = dev(np.zeros(nxyz, dtype=np.complex128))
    P.set_recip_to_real_output_op(nxyz, False, float(g["factor"]), dev(g["in_2"]), out)
    assert np.max(np.abs(host(out) - g["out_2"])) < 1e-12
    out = dev(g["out_3_init"])
    P.set_real_to_recip_output_op(npwk, nxyz, True, float(g["factor"]), idx, dev(g["in_3"]), out)
    assert np.max(np.abs(host(out) - g["out_3"])) < 5e-6
