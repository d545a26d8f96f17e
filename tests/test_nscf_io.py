"""NSCF file formats (abacus-develop_b200/nscf_io.py) against the reference's own test fixtures and known
answers (tests/golden/make_golden.py):

* WAVEFUNC1.dat (module_io/test/support) read through this package's PW_Basis_K on the reference test's
  cell (lat0 5.3233, fcc, 12^3 grid, ecut 20 Ry): read_wfc_pw_test.cpp's coefficients exactly; written
  back, the same 8492 bytes; the reader's consistency checks;
* SPIN1_CHG.cube (module_io/test_serial/support): rho_io_test.cpp's Fermi energy and values; written back,
  the same data block, character for character; the trilinear interpolation's known values;
* nscf_band_test.cpp's band-structure line; the NSCF threshold rule (pw_nscf.cpp:63-68).
"""
from __future__ import annotations

import zlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def io(pkg):
    import importlib
    return importlib.import_module(pkg.__name__ + ".nscf_io")


@pytest.fixture(scope="module")
def wfc_case(pkg, golden, tmp_path_factory):
    g = golden("wfc_pw")
    b = pkg.pwdft.PWBasisK(float(g["lat0"]), g["latvec"], float(g["ecutwfc"]), np.zeros((int(g["nks"]), 3)),
                           ecutrho=-1.0, grid=tuple(int(x) for x in g["grid"]))
    d = tmp_path_factory.mktemp("wfc")
    fn = d / "WAVEFUNC1.dat"
    fn.write_bytes(g["raw"].tobytes())
    return g, b, fn, d


def test_read_wfc_pw_known_answers(io, wfc_case):
    g, b, fn, _ = wfc_case
    assert (b.nx, b.ny, b.nz) == (12, 12, 12)
    psi = io.read_wfc_pw(fn, b, 0, int(g["nkstot"]), int(g["nbands"]), g["latvec"])
    assert psi.shape == (int(g["nbands"]), int(b.npwk[0]))
    for ib, which, part, val in g["expect"]:
        v = psi[int(ib), int(which)]
        assert (v.real if part == 0 else v.imag) == val


def test_write_wfc_pw_reproduces_the_reference_file(io, wfc_case):
    g, b, fn, d = wfc_case
    psi = io.read_wfc_pw(fn, b, 0, int(g["nkstot"]), int(g["nbands"]), g["latvec"])
    hd = io.read_wfc_pw_header(fn)
    names = io.write_wfc_pw(str(d / "OUT"), b, [psi] * b.nks, np.zeros((b.nks, 3)), np.full(b.nks, hd.weight),
                            hd.ecutwfc, g["latvec"], nkstot=hd.nkstot, fmt=2)
    assert (d / "OUT1.dat").read_bytes() == g["raw"].tobytes()
    assert len(names) == b.nks
    # the text format: header, G vectors in box indices, 4 complex numbers per line at 6 digits
    io.write_wfc_pw(str(d / "TXT"), b, [psi] * b.nks, np.zeros((b.nks, 3)), np.full(b.nks, hd.weight),
                    hd.ecutwfc, g["latvec"], nkstot=hd.nkstot, fmt=1)
    txt = (d / "TXT1.txt").read_text()
    lines = txt.split("\n")
    assert lines[1].split() == ["1", "8", "0", "0", "0", "0.25", str(b.npwk[0]), "8", "20", "5.3233", "1.18032"]
    band1 = txt[txt.index("< Band 1 >") + len("< Band 1 >\n"):]
    rows = band1[:band1.index("\n< Band 1 >")].split("\n")
    assert len(rows) == (int(b.npwk[0]) + 3) // 4 and all(len(r) == 15 * 8 for r in rows[:-1])
    vals = np.array(" ".join(rows).split(), dtype=float)
    assert np.allclose(vals[0::2] + 1j * vals[1::2], psi[0], rtol=1e-5, atol=1e-12)


def test_read_wfc_pw_checks(io, wfc_case, tmp_path):
    g, b, fn, _ = wfc_case
    with pytest.raises(ValueError, match="nbands_in = 8"):
        io.read_wfc_pw(fn, b, 0, int(g["nkstot"]), 4, g["latvec"])
    with pytest.raises(ValueError, match="Can't open file"):
        io.read_wfc_pw(tmp_path / "notfound.dat", b, 0, 8, 8, g["latvec"])
    with pytest.raises(ValueError, match="Unknown file type"):
        io.read_wfc_pw(tmp_path / "notfound", b, 0, 8, 8, g["latvec"])
    with pytest.raises(ValueError, match="nkstot"):
        io.read_wfc_pw(fn, b, 0, 7, 8, g["latvec"])
    with pytest.raises(ValueError, match="G_in != G"):
        io.read_wfc_pw(fn, b, 0, 8, 8, np.asarray(g["latvec"]) * 1.0000001)


def test_reciprocal_lattice_bits(io, golden):
    g = golden("wfc_pw")
    G = io.reciprocal_lattice(g["latvec"])
    assert np.array_equal(G, np.array([[-1.0, -1.0, 1.0], [1.0, 1.0, 1.0], [-1.0, 1.0, -1.0]]))
    lv = np.array([[1.0, 0.1, 0.0], [0.3, 1.7, 0.2], [0.0, 0.4, 2.1]])
    assert np.allclose(io.reciprocal_lattice(lv), np.linalg.inv(lv).T, rtol=1e-14, atol=0)


@pytest.fixture(scope="module")
def cube_case(golden, tmp_path_factory):
    c = golden("cube_chg")
    d = tmp_path_factory.mktemp("cube")
    fn = d / "SPIN1_CHG.cube"
    fn.write_text(zlib.decompress(c["zraw"].tobytes()).decode())
    return c, fn, d


def test_read_cube_known_answers(io, cube_case):
    c, fn, _ = cube_case
    cb = io.read_cube(fn, 36, 36, 36, nspin=1, nat=2)
    assert cb.ef == c["ef"]
    for i, v in zip(c["rho_idx"], c["rho_val"]):
        assert cb.data[int(i)] == v
    with pytest.raises(ValueError, match="nspin mismatch"):
        io.read_cube(fn, nspin=2)


def test_write_cube_reproduces_the_data_block(io, cube_case):
    c, fn, d = cube_case
    cb = io.read_cube(fn)
    lat = cb.axes * np.array(cb.grid)[:, None]  # lattice vectors in bohr: written with lat0 = 1
    io.write_cube(d / "W.cube", cb.data, *cb.grid, 1.0, lat, cb.atoms, nspin=1, ef=cb.ef, precision=11)
    ref = fn.read_text().split("\n")
    out = (d / "W.cube").read_text().split("\n")
    assert out[8:] == ref[8:]  # 46656 values, six a line, a new line per z column
    assert out[:3] == ref[:3]
    # the header in the writer's current fixed format (the fixture predates it for the cell lines)
    assert out[3] == "36 -0.141667 0.000000 0.141667" and out[7] == " 14 4.000000 -7.650000 7.650000 7.650000"
    back = io.read_cube(d / "W.cube")
    assert np.array_equal(back.data, cb.data) and back.ef == cb.ef


def test_trilinear_interpolation_known_answers(io, cube_case):
    c, fn, _ = cube_case
    nx, ny, nz = (int(v) for v in c["interp_dims"])
    cb = io.read_cube(fn, nx, ny, nz)
    assert cb.data.size == nx * ny * nz
    for k, v in zip(c["interp_idx"], c["interp_val"]):
        # the reference test indexes its one-process z-major layout: k = iz * nx * ny + ix * ny + iy
        iz, ixy = divmod(int(k), nx * ny)
        assert cb.data[ixy * nz + iz] == v
    # same grid: no interpolation, identity
    src = io.read_cube(fn).data
    assert np.array_equal(io.trilinear_interpolate(src, 36, 36, 36, 36, 36, 36), src)


def test_nscf_band_line(io, golden, tmp_path):
    b = golden("nscf_band")
    lines = io.nscf_band(tmp_path / "band.dat", b["ekb"], b["kvec_c"], b["kl_segids"], float(b["fermie"]),
                         int(b["precision"]))
    assert str(b["line"]) in (tmp_path / "band.dat").read_text()
    assert lines[1].startswith("   2 1.00000000 ")


def test_nscf_threshold_rule(io):
    assert io.nscf_diag_thr(1e-2, 1e-9, 8.0) == max(1e-13, 0.1 * min(1e-2, 1e-9 / 8.0))
    assert io.nscf_diag_thr(5e-3, 1e-9, 8.0) == 5e-3
    assert io.nscf_diag_thr(1e-2, 1e-15, 8.0) == 1e-13
