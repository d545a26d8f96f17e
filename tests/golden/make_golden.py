"""Extract the reference's own golden vectors into small numpy fixtures.

Run in a container where the reference source tree is mounted, with its path in
ABACUS_REF or as the first argument.  Reads the literal arrays of the
reference's unit tests as text and writes ``tests/golden/*.npz``:

  ekinetic_op.npz  <- source/module_hamilt_pw/hamilt_pwdft/kernels/test/ekinetic_op_test.cpp
  nonlocal_op.npz  <- .../kernels/test/nonlocal_op_test.cpp
  veff_op.npz      <- .../kernels/test/veff_op_test.cpp
  pw_op.npz        <- source/module_basis/module_pw/kernels/test/pw_op_test.cpp
  vnl_op.npz       <- .../kernels/test/vnl_op_test.cpp
  wf_op.npz        <- .../kernels/test/wf_op_test.cpp
  ylm_op.npz       <- source/module_base/kernels/test/math_op_test.cpp
  elecstate_op.npz <- source/module_elecstate/kernels/test/elecstate_op_test.cpp
  pyabacus_si2.npz <- python/pyabacus/tests/test_diag/Si2.mat (sparse H, CSC arrays)
  wfc_pw.npz       <- source/module_io/test/support/WAVEFUNC1.dat (bytes) + read_wfc_pw_test.cpp's
                      basis set-up and expected coefficients (one process per pool)
  cube_chg.npz     <- source/module_io/test_serial/support/SPIN1_CHG.cube (bytes, zlib) + rho_io_test.cpp's
                      expected Fermi energy, values and trilinear-interpolation values
  nscf_band.npz    <- source/module_io/test_serial/nscf_band_test.cpp: band energies, k-points and the
                      expected output line

The fixtures are committed; tests never read the reference tree.
"""
from __future__ import annotations

import os
import re
import sys
from pathlib import Path

import numpy as np

REF = Path(os.environ["ABACUS_REF"]) if os.environ.get("ABACUS_REF") else None
OUT = Path(__file__).resolve().parent

_num = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"


def _parse_block(text: str):
    """Parse the body of a C++ initializer list: complex pairs {a,b} or plain numbers."""
    pairs = re.findall(r"\{\s*(" + _num + r")\s*,\s*(" + _num + r")\s*\}", text)
    if pairs:
        return np.array([complex(float(a), float(b)) for a, b in pairs])
    return np.array([float(x) for x in re.findall(_num, text)])


def _vectors(path: Path) -> dict:
    src = path.read_text()
    out = {}
    for m in re.finditer(r"std::vector<[^=;{]*?>\s+(\w+)\s*=?\s*\{", src):
        name = m.group(1)
        i = m.end()
        depth = 1
        while depth:
            c = src[i]
            depth += (c == "{") - (c == "}")
            i += 1
        out[name] = _parse_block(src[m.end():i - 1])
    return out


def _scalars(path: Path, names):
    src = path.read_text()
    res = {}
    for n in names:
        m = re.search(r"\b" + n + r"\s*=\s*(" + _num + r")\s*[;,]", src)
        res[n] = float(m.group(1))
    return res


def main():
    kt = REF / "source/module_hamilt_pw/hamilt_pwdft/kernels/test"
    v = _vectors(kt / "ekinetic_op_test.cpp")
    s = _scalars(kt / "ekinetic_op_test.cpp", ["dim", "band", "tpiba2"])
    np.savez(OUT / "ekinetic_op.npz", gk2=v["gk2"], psi=v["psi"], expected_hpsi=v["expected_hpsi"],
             dim=int(s["dim"]), band=int(s["band"]), tpiba2=s["tpiba2"])

    v = _vectors(kt / "nonlocal_op_test.cpp")
    s = _scalars(kt / "nonlocal_op_test.cpp",
                 ["l1", "l2", "l2_spin", "l3", "spin", "nkb", "deeq_x", "deeq_y", "deeq_z", "expected_sum", "expected_iat"])
    np.savez(OUT / "nonlocal_op.npz", deeq=v["deeq"], deeq_spin=v["deeq_spin"], becp=v["becp"],
             becp_spin=v["becp_spin"], expected_ps=v["expected_ps"], expected_ps_spin=v["expected_ps_spin"],
             **{k: int(x) for k, x in s.items()})

    v = _vectors(kt / "veff_op_test.cpp")
    s = _scalars(kt / "veff_op_test.cpp", ["size"])
    np.savez(OUT / "veff_op.npz", vin=v["in"], out=v["out"], expected_out=v["expected_out"],
             out_spin=v["out_spin"], in_spin=v["in_spin"], expected_out_spin=v["expected_out_spin"],
             size=int(s["size"]))

    pt = REF / "source/module_basis/module_pw/kernels/test/pw_op_test.cpp"
    v = _vectors(pt)
    s = _scalars(pt, ["npwk", "nxyz", "factor"])
    np.savez(OUT / "pw_op.npz", box_index=v["box_index"].astype(np.int64), in_1=v["in_1"], out_1=v["out_1"],
             in_2=v["in_2"], out_2=v["out_2"], in_3=v["in_3"], out_3=v["out_3"], out_3_init=v["out_3_init"],
             npwk=int(s["npwk"]), nxyz=int(s["nxyz"]), factor=s["factor"])

    # projector generation: cal_vnl_op, cal_sk_op and cal_ylm_real_op literals
    v = _vectors(kt / "vnl_op_test.cpp")
    s = _scalars(kt / "vnl_op_test.cpp", ["ntype", "npw", "npwx", "nhm", "tab_2", "tab_3", "DQ", "tpiba"])
    src = (kt / "vnl_op_test.cpp").read_text()
    brace = {n: int(re.search(r"std::vector<int>\s+" + n + r"\{(\d+)\}", src).group(1))
             for n in ("atom_na", "atom_nb", "atom_nh")}
    np.savez(OUT / "vnl_op.npz", gk=v["gk"], ylm=v["ylm"], indv=v["indv"], nhtol=v["nhtol"], nhtolm=v["nhtolm"],
             tab=v["tab"], sk=v["sk"], expected_vkb=v["expected_vkb"],
             **{k: (x if k in ("DQ", "tpiba") else int(x)) for k, x in s.items()}, **brace)

    wt = kt / "wf_op_test.cpp"
    v = _vectors(wt)
    s = _scalars(wt, ["ik", "ntype", "nx", "ny", "nz", "rho_nx", "rho_ny", "rho_nz", "npw", "npwx", "fftny",
                      "eigts1_nc", "eigts2_nc", "eigts3_nc", "TWO_PI"])
    src = wt.read_text()
    na = int(re.search(r"std::vector<int>\s+atom_na\{(\d+)\}", src).group(1))
    np.savez(OUT / "wf_op.npz", igl2isz=v["igl2isz"].astype(np.int64), is2fftixy=v["is2fftixy"].astype(np.int64),
             kvec_c=v["kvec_c"], atom_tau=v["atom_tau"], eigts1=v["eigts1"], eigts2=v["eigts2"],
             eigts3=v["eigts3"], expected_sk=v["expected_sk"], atom_na=na,
             **{k: (x if k == "TWO_PI" else int(x)) for k, x in s.items()})

    mt = REF / "source/module_base/kernels/test/math_op_test.cpp"
    v = _vectors(mt)
    s = _scalars(mt, ["ng", "lmax"])
    np.savez(OUT / "ylm_op.npz", g=v["g"], expected_ylm=v["expected_ylm"], ng=int(s["ng"]), lmax=int(s["lmax"]))

    et = REF / "source/module_elecstate/kernels/test/elecstate_op_test.cpp"
    v = _vectors(et)
    s = _scalars(et, ["spin", "nrxx", "w1", "w2"])
    src = et.read_text()
    flags = {n: int(re.search(r"\b" + n + r"\s*=\s*(true|false)", src).group(1) == "true") for n in ("DOMAG", "DOMAG_Z")}
    np.savez(OUT / "elecstate_op.npz", wfcr=v["wfcr"], expected_rho=v["expected_rho"], wfcr_2=v["wfcr_2"],
             wfcr_another_spin_2=v["wfcr_another_spin_2"], expected_rho_2=v["expected_rho_2"],
             spin=int(s["spin"]), nrxx=int(s["nrxx"]), w1=s["w1"], w2=s["w2"], **flags)

    try:
        import scipy.io
        import scipy.sparse
        mat = scipy.io.loadmat(REF / "python/pyabacus/tests/test_diag/Si2.mat")["Problem"]["A"][0, 0]
        csc = scipy.sparse.csc_matrix(mat)
        np.savez_compressed(OUT / "pyabacus_si2.npz", data=csc.data, indices=csc.indices, indptr=csc.indptr,
                            shape=np.array(csc.shape))
    except Exception as exc:  # pragma: no cover
        print("Si2.mat skipped:", exc, file=sys.stderr)
    io_fixtures()
    print("golden fixtures written to", OUT)


def _expect_doubles(src: str):
    """(expression, value) of every EXPECT_DOUBLE_EQ(expr, value) in src, in order."""
    return [(a.strip(), float(b)) for a, b in re.findall(r"EXPECT_DOUBLE_EQ\((.*),\s*(" + _num + r")\s*\);", src)]


def io_fixtures():
    import zlib
    # plane-wave wavefunction file and the reader's known answers (read_wfc_pw_test.cpp, one process)
    test = (REF / "source/module_io/test/read_wfc_pw_test.cpp").read_text()
    body = test[test.index("TEST_F(ReadWfcPwTest, ReadWfcPw)"):test.index("else if (GlobalV::NPROC_IN_POOL == 4)")]
    exp = _expect_doubles(body)
    m = re.search(r"initgrids\(\s*(" + _num + r")\s*,\s*ModuleBase::Matrix3\(([^)]*)\)\s*,\s*(\d+)\s*,\s*(\d+)\s*,\s*(\d+)\)", body)
    lat0, latvec = float(m.group(1)), np.array([float(x) for x in m.group(2).split(",")]).reshape(3, 3)
    grid = np.array([int(m.group(3)), int(m.group(4)), int(m.group(5))])
    m2 = re.search(r"initparameters\(\s*false\s*,\s*(" + _num + r")\s*,\s*(\d+)", body)
    nbands = int(re.search(r"GlobalV::NBANDS\s*=\s*(\d+)", body).group(1))
    nkstot = int(re.search(r"int nkstot\s*=\s*(\d+)", test).group(1))
    # wfcatom(ib, ig) with ig = 0 or npwk-1 ("last"): band, which, real/imag, value
    rows = []
    for expr, val in exp:
        mm = re.match(r"wfcatom\((\d+),\s*(0|wfcpw->npwk\[0\] - 1)\)\.(real|imag)\(\)", expr)
        rows.append((int(mm.group(1)), 0 if mm.group(2) == "0" else -1, 0 if mm.group(3) == "real" else 1, val))
    raw = (REF / "source/module_io/test/support/WAVEFUNC1.dat").read_bytes()
    np.savez(OUT / "wfc_pw.npz", raw=np.frombuffer(raw, dtype=np.uint8), lat0=lat0, latvec=latvec, grid=grid,
             ecutwfc=float(m2.group(1)), nks=int(m2.group(2)), nkstot=nkstot, nbands=nbands,
             expect=np.array(rows, dtype=np.float64))

    # cube file and the reader's known answers (rho_io_test.cpp)
    test = (REF / "source/module_io/test_serial/rho_io_test.cpp").read_text()
    read = _expect_doubles(test[test.index("TEST_F(RhoIOTest, Read)"):test.index("TEST_F(RhoIOTest, TrilinearInterpolate)")])
    interp = _expect_doubles(test[test.index("TEST_F(RhoIOTest, TrilinearInterpolate)"):])
    dims = re.findall(r"int n([xyz])(?:_read)?\s*=\s*(\d+);", test[test.index("TEST_F(RhoIOTest, TrilinearInterpolate)"):])
    raw = (REF / "source/module_io/test_serial/support/SPIN1_CHG.cube").read_bytes()
    np.savez(OUT / "cube_chg.npz", zraw=np.frombuffer(zlib.compress(raw, 9), dtype=np.uint8),
             ef=read[0][1], rho_idx=np.array([int(re.search(r"\[(\d+)\]$", e).group(1)) for e, _ in read[1:]]),
             rho_val=np.array([v for _, v in read[1:]]),
             interp_dims=np.array([int(v) for _, v in dims[:3]]),
             interp_idx=np.array([int(re.search(r"\[(\d+)\]", e).group(1)) for e, _ in interp]),
             interp_val=np.array([v for _, v in interp]))

    # band-structure file line (nscf_band_test.cpp)
    test = (REF / "source/module_io/test_serial/nscf_band_test.cpp").read_text()
    ekb = {(int(a), int(b)): float(c) for a, b, c in re.findall(r"ekb\((\d+),\s*(\d+)\)\s*=\s*(" + _num + r");", test)}
    nks = 1 + max(k[0] for k in ekb)
    nband = 1 + max(k[1] for k in ekb)
    kv = [tuple(float(x) for x in g) for g in re.findall(r"kvec_c\[\d\] = ModuleBase::Vector3<double>\((" + _num +
                                                         r"),\s*(" + _num + r"),\s*(" + _num + r")\)", test)]
    seg = [int(x) for x in re.findall(r"kl_segids\[\d\] = (\d+);", test)]
    line = re.search(r'HasSubstr\("([^"]*)"\)', test[test.index("TEST_F(BandTest, nscf_band)"):]).group(1)
    prec = int(re.search(r"nscf_band\(is, out_band_dir, nband, fermie, (\d+),", test).group(1))
    np.savez(OUT / "nscf_band.npz", ekb=np.array([[ekb[(k, b)] for b in range(nband)] for k in range(nks)]),
             kvec_c=np.array(kv), kl_segids=np.array(seg), precision=prec, fermie=0.0, line=np.array(line))


if __name__ == "__main__":
    if len(sys.argv) > 1:
        REF = Path(sys.argv[1])
    if REF is None or not REF.exists():
        sys.exit("give the reference checkout: ABACUS_REF=<path> or make_golden.py <path>")
    main()
