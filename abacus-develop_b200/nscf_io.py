"""File formats of the non-self-consistent inputs and outputs, restating the reference's writers and readers:

* plane-wave wavefunctions, ``out_wfc_pw`` / ``init_wfc file`` (module_io/write_wfc_pw.cpp:13-283,
  module_io/read_wfc_pw.cpp:11-341): ``<prefix><ik+1>.dat`` (binary records) or ``.txt`` (formatted text);
* real-space grids, ``out_pot`` / ``out_chg`` cube files (module_io/write_cube.cpp:5-300,
  module_io/read_cube.cpp:3-275), with the trilinear interpolation a reader applies when the file's grid
  differs from the calculation's;
* the band-structure file of an NSCF run (module_io/nscf_band.cpp:9-124) and the eigenvalue lines of its
  running log (module_esolver/pw_nscf.cpp:76-103);
* the NSCF diagonalisation threshold rule (pw_nscf.cpp:63-68).

Host code (numpy): these files are read once per cell and written once per run.  Real-space arrays are in
ABACUS's r order, index (ix * ny + iy) * nz + iz (z fastest), which is also the order of a cube file's
values; wavefunctions are (nbands, npwk) arrays in the order of the basis's G sphere for that k-point.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

RY_TO_EV = 13.605698  # ModuleBase::Ry_to_eV (module_base/constants.h)
TWO_PI = 2.0 * math.pi


# ------------------------------------------------------------------ lattice helpers
def reciprocal_lattice(latvec) -> np.ndarray:
    """G = (latvec^-1)^T in units of 2 pi / lat0, with ModuleBase::Matrix3's Det / Inverse expansion order
    (module_base/matrix3.cpp:29-59) so that the bits match the reference's (the wavefunction reader compares
    them exactly)."""
    a = [float(x) for x in np.asarray(latvec, dtype=np.float64).reshape(9)]
    e11, e12, e13, e21, e22, e23, e31, e32, e33 = a
    d = e11 * e22 * e33 - e11 * e32 * e23 + e21 * e32 * e13 - e21 * e12 * e33 + e31 * e12 * e23 - e31 * e22 * e13
    if d == 0:
        d = 1.0
    gt = [(e22 * e33 - e23 * e32) / d, -(e12 * e33 - e13 * e32) / d, (e12 * e23 - e13 * e22) / d,
          -(e21 * e33 - e23 * e31) / d, (e11 * e33 - e13 * e31) / d, -(e11 * e23 - e13 * e21) / d,
          (e21 * e32 - e22 * e31) / d, -(e11 * e32 - e12 * e31) / d, (e11 * e22 - e12 * e21) / d]
    return np.array(gt).reshape(3, 3).T.copy()


def kvec_cartesian(kvec_d, latvec) -> np.ndarray:
    """kvec_c = kvec_d * G (ModuleBase::Vector3 * Matrix3, left to right), units of 2 pi / lat0."""
    g = reciprocal_lattice(latvec)
    kd = np.atleast_2d(np.asarray(kvec_d, dtype=np.float64))
    out = np.zeros_like(kd)
    for i, (x, y, z) in enumerate(kd):
        for j in range(3):
            out[i, j] = x * g[0, j] + y * g[1, j] + z * g[2, j]
    return out


def _box_indices(basis, ik):
    """(ix, iy, iz) FFT-box indices of the plane waves of k-point ik, in the basis's order
    (write_wfc_pw.cpp:131-139: isz -> (is, iz), is -> ixy -> (ix, iy))."""
    idx = basis.ig2ixyz(ik)
    nyz = basis.ny * basis.nz
    return idx // nyz, (idx // basis.nz) % basis.ny, idx % basis.nz


# ------------------------------------------------------------------ wavefunctions
@dataclass
class WfcHeader:
    ikstot: int        # 1-based k index in the file
    nkstot: int
    kvec_c: np.ndarray  # units of 2 pi / lat0
    weight: float
    npwtot: int
    nbands: int
    ecutwfc: float
    lat0: float
    tpiba: float
    G: np.ndarray = field(default_factory=lambda: np.zeros((3, 3)))


def _cxx_g(x: float, width: int = 10) -> str:
    """std::setw(width) << x with the default float format at precision 6 (printf %g)."""
    return f"{x:{width}.6g}"


def wfc_filename(prefix: str, ik: int, fmt: int) -> str:
    return f"{prefix}{ik + 1}.{'txt' if fmt == 1 else 'dat'}"


def write_wfc_pw(prefix, basis, psis, kvec_c, wk, ecutwfc, latvec, nbands=None, fmt=2, nkstot=None):
    """ModuleIO::write_wfc_pw for one pool of one process, npol = 1: one file per k-point,
    ``<prefix><ik+1>.dat`` (fmt 2, binary) or ``.txt`` (fmt 1).  psis[ik]: (>= nbands, >= npwk) complex
    array in the basis's plane-wave order; kvec_c: (nks, 3) in units of 2 pi / lat0; wk: k weights.
    Returns the file names."""
    nks = basis.nks
    nkstot = nks if nkstot is None else nkstot
    return [write_wfc_pw_k(prefix, basis, ik, psis[ik], kvec_c[ik], wk[ik], ecutwfc, latvec, nbands, fmt, nkstot)
            for ik in range(nks)]


def write_wfc_pw_k(prefix, basis, ik, psi, kvec_c, wk, ecutwfc, latvec, nbands=None, fmt=2, nkstot=None):
    """The file of k-point ik alone (write_wfc_pw.cpp:62-280 for one ik); returns its name."""
    nkstot = basis.nks if nkstot is None else nkstot
    G = reciprocal_lattice(latvec)
    tpiba = TWO_PI / basis.lat0
    psi = np.asarray(psi)
    nb = psi.shape[0] if nbands is None else nbands
    ng = int(basis.npwk[ik])
    ix, iy, iz = _box_indices(basis, ik)
    fn = wfc_filename(prefix, ik, fmt)
    kx, ky, kz = (float(v) for v in kvec_c)
    if fmt == 2:
        with open(fn, "wb") as f:
            f.write(struct.pack("<iii3ddiidddi", 72, ik + 1, nkstot, kx, ky, kz, float(wk), ng, nb,
                                float(ecutwfc), float(basis.lat0), tpiba, 72))
            f.write(struct.pack("<i9di", 72, *[float(v) for v in G.reshape(9)], 72))
            mill = np.stack([ix, iy, iz], axis=1).astype("<i4")
            f.write(struct.pack("<i", ng * 12) + mill.tobytes() + struct.pack("<i", ng * 12))
            rec = struct.pack("<i", ng * 16)
            for ib in range(nb):
                f.write(rec + np.ascontiguousarray(psi[ib, :ng], dtype="<c16").tobytes() + rec)
    elif fmt == 1:
        lines = ["".join(f"{s:>10}" for s in ("Kpoint", "nKpoint", "kv.x", "kv.y", "kv.z", "weight", "ngtot",
                                              "nband", "ecut", "lat0", "2pi/lat0")) + "\n"]
        lines.append(f"{ik + 1:10d}{nkstot:10d}" + "".join(_cxx_g(v) for v in (kx, ky, kz, float(wk)))
                     + f"{ng:10d}{nb:10d}" + "".join(_cxx_g(v) for v in (float(ecutwfc), basis.lat0, tpiba))
                     + "\n")
        lines.append("\n<Reciprocal Lattice Vector>\n")
        for r in range(3):
            lines.append("".join(_cxx_g(float(v)) for v in G[r]) + "\n")
        lines.append("<Reciprocal Lattice Vector>\n\n")
        lines.append("<G vectors>\n")
        lines.extend(f"{a:10d}{b:10d}{c:10d}\n" for a, b, c in zip(ix, iy, iz))
        lines.append("<G vectors>\n\n")
        for ib in range(nb):
            lines.append(f"\n< Band {ib + 1} >\n")
            v = np.empty(2 * ng)
            v[0::2], v[1::2] = psi[ib, :ng].real, psi[ib, :ng].imag
            cells = [f"{x:15.6e}" for x in v]
            rows = ["".join(cells[i:i + 8]) for i in range(0, len(cells), 8)]  # 4 complex numbers per row
            lines.append("\n".join(rows))
            lines.append(f"\n< Band {ib + 1} >\n")
        with open(fn, "w") as f:
            f.write("".join(lines))
    else:
        raise ValueError("fmt must be 1 (txt) or 2 (dat)")
    return fn


def read_wfc_pw_header(filename) -> WfcHeader:
    """The two header records of a binary wavefunction file."""
    with open(filename, "rb") as f:
        raw = f.read(160)
    if len(raw) < 160:
        raise ValueError(f"{filename}: truncated header")
    h = struct.unpack_from("<iii3ddiidddi", raw, 0)
    g = struct.unpack_from("<i9di", raw, 80)
    if h[0] != 72 or h[-1] != 72 or g[0] != 72 or g[-1] != 72:
        raise ValueError(f"{filename}: not a plane-wave wavefunction file (record markers)")
    return WfcHeader(ikstot=h[1], nkstot=h[2], kvec_c=np.array(h[3:6]), weight=h[6], npwtot=h[7], nbands=h[8],
                     ecutwfc=h[9], lat0=h[10], tpiba=h[11], G=np.array(g[1:10]).reshape(3, 3))


def read_wfc_pw(filename, basis, ik, nkstot, nbands, latvec):
    """ModuleIO::read_wfc_pw for one process per pool, npol = 1: the (nbands, npwk[ik]) coefficients of k-point
    ik in the basis's plane-wave order.  The reference's checks are kept (read_wfc_pw.cpp:96-160): file type,
    k index, number of k-points, plane waves and bands, the k vector, lat0, 2 pi / lat0 and G, all exact;
    a failed check raises ValueError with the reference's message."""
    filename = str(filename)
    ftype = filename[-3:]
    if ftype not in ("txt", "dat"):
        raise ValueError(f"Unknown file type {ftype}")
    if not Path(filename).exists():
        raise ValueError(f"Can't open file {filename}")
    if ftype == "txt":
        # the reference reads nothing from a text file (read_wfc_pw.cpp:96-101, 148-152, 171-176)
        raise ValueError("text wavefunction files carry no readable coefficients: use the binary (.dat) format")
    hd = read_wfc_pw_header(filename)
    npwtot = int(basis.npwk[ik])
    if hd.ikstot != ik + 1 or hd.nkstot != nkstot or hd.npwtot != npwtot or hd.nbands != nbands:
        raise ValueError(f"ikstot_in = {hd.ikstot}, ikstot = {ik + 1}, nkstot_in = {hd.nkstot}, nkstot = {nkstot}, "
                         f"npwtot_in = {hd.npwtot}, npwtot = {npwtot}, nbands_in = {hd.nbands}, nbands = {nbands}: "
                         "ikstot_in != ikstot || nkstot_in != nkstot || npwtot_in != npwtot || nbands_in != NBANDS")
    if not np.array_equal(hd.kvec_c, basis.kvec_c(ik)):
        raise ValueError("k vector in file is not the same as the one in memory")
    if hd.lat0 != basis.lat0 or hd.tpiba != TWO_PI / basis.lat0:
        raise ValueError("lat0_in != pw_wfc->lat0 || tpiba_in != pw_wfc->tpiba")
    if not np.array_equal(hd.G, reciprocal_lattice(latvec)):
        raise ValueError("G_in != G")
    nx, ny, nz = basis.nx, basis.ny, basis.nz
    with open(filename, "rb") as f:
        f.seek(160)
        (size,) = struct.unpack("<i", f.read(4))
        mill = np.frombuffer(f.read(12 * npwtot), dtype="<i4").reshape(npwtot, 3)
        f.read(4)
        # map global index to the file's ordering (read_wfc_pw.cpp:162-190)
        glo_order = np.full(nx * ny * nz, -1, dtype=np.int64)
        glo_order[(mill[:, 0] * ny + mill[:, 1]) * nz + mill[:, 2]] = np.arange(npwtot)
        order = glo_order[basis.ig2ixyz(ik)]
        if np.any(order < 0):
            raise ValueError("a plane wave of the basis is missing from the file")
        out = np.zeros((nbands, npwtot), dtype=np.complex128)
        for ib in range(nbands):
            f.read(4)
            wfc_in = np.frombuffer(f.read(16 * npwtot), dtype="<c16")
            f.read(4)
            out[ib] = wfc_in[order]
    return out


# ------------------------------------------------------------------ cube files
@dataclass
class CubeAtom:
    z: int            # atomic number (0 when the label is not an element)
    zv: float         # valence charge
    tau: tuple        # cartesian position in bohr (the reference writes lat0 * tau of its unit cell)


def _cxx_fixed6(x: float) -> str:
    return f"{x:.6f}"


def write_cube(fn, data, nx, ny, nz, lat0, latvec, atoms, nspin=1, is_=0, iter_=0, ef=0.0, precision=11,
               out_fermi=1, two_fermi=False, append=False):
    """ModuleIO::write_cube (write_cube.cpp:5-136, the one-file data block of write_cube_core :138-282):
    data is in r order (z fastest); six values per line, a new line after every z column."""
    data = np.asarray(data, dtype=np.float64).reshape(nx * ny, nz)
    out = [f"STEP: {iter_}  Cubefile created from ABACUS. Inner loop is z, followed by y and x\n",
           f"{nspin} (nspin) "]
    if out_fermi == 1:
        if two_fermi:
            out.append(f"{_cxx_fixed6(ef)} (fermi energy for spin={is_ + 1}, in Ry)\n")
        else:
            out.append(f"{_cxx_fixed6(ef)} (fermi energy, in Ry)\n")
    else:
        out.append("\n")
    out.append(f"{len(atoms)} 0.0 0.0 0.0 \n")
    lv = np.asarray(latvec, dtype=np.float64).reshape(3, 3)
    for n, row in zip((nx, ny, nz), lv):
        out.append(f"{n} " + " ".join(_cxx_fixed6(lat0 * float(v) / float(n)) for v in row) + "\n")
    for a in atoms:
        out.append(f" {a.z} {_cxx_fixed6(a.zv)} " + " ".join(_cxx_fixed6(float(t)) for t in a.tau) + "\n")
    cells = np.char.mod(f" %.{precision}e", data)
    per = 6
    for row in cells:
        chunks = ["".join(row[i:i + per]) for i in range(0, nz, per)]
        out.append("\n".join(chunks) + "\n")
    with open(fn, "a" if append else "w") as f:
        f.write("".join(out))


@dataclass
class Cube:
    nspin: int
    ef: float
    nat: int
    grid: tuple
    axes: np.ndarray      # (3, 3) voxel vectors in bohr
    atoms: list
    data: np.ndarray      # r order, file grid (or the requested grid after interpolation)


def _read_cube_text(text: str):
    lines = text.split("\n")
    l1 = lines[1]
    nspin = int(l1.split()[0])
    ef = 0.0
    rest = l1[l1.index(")") + 1:].split() if ")" in l1 else []
    if rest:
        ef = float(rest[0])
    nat = int(lines[2].split()[0])
    grid, axes = [], []
    for k in range(3):
        p = lines[3 + k].split()
        grid.append(int(p[0]))
        axes.append([float(x) for x in p[1:4]])
    atoms = []
    for k in range(nat):
        p = lines[6 + k].split()
        atoms.append(CubeAtom(z=int(float(p[0])), zv=float(p[1]), tau=tuple(float(x) for x in p[2:5])))
    vals = np.array(" ".join(lines[6 + nat:]).split(), dtype=np.float64)
    return nspin, ef, nat, tuple(grid), np.array(axes), atoms, vals


def trilinear_interpolate(values, nx_read, ny_read, nz_read, nx, ny, nz):
    """ModuleIO::trilinear_interpolate (read_cube.cpp:198-275): values of an (nx_read, ny_read, nz_read) grid
    in file order onto (nx, ny, nz), periodic; returned in r order (z fastest)."""
    src = np.asarray(values, dtype=np.float64).reshape(nx_read, ny_read, nz_read)

    def axis(n_read, n):
        frac = np.fmod(0.5 * (float(n_read) / n * (1.0 + 2.0 * np.arange(n)) - 1.0), n_read)
        low = frac.astype(np.int64)
        d = frac - low
        high = np.where(low == n_read - 1, 0, low + 1)
        return low, high, d

    lx, hx, dx = axis(nx_read, nx)
    ly, hy, dy = axis(ny_read, ny)
    lz, hz, dz = axis(nz_read, nz)
    X, Y, Z = np.ix_(np.arange(nx), np.arange(ny), np.arange(nz))
    ddx, ddy, ddz = dx[X], dy[Y], dz[Z]
    # the reference's order of the eight terms
    r = (src[lx[X], ly[Y], lz[Z]] * (1 - ddx) * (1 - ddy) * (1 - ddz)
         + src[hx[X], ly[Y], lz[Z]] * ddx * (1 - ddy) * (1 - ddz)
         + src[lx[X], hy[Y], lz[Z]] * (1 - ddx) * ddy * (1 - ddz)
         + src[lx[X], ly[Y], hz[Z]] * (1 - ddx) * (1 - ddy) * ddz
         + src[hx[X], hy[Y], lz[Z]] * ddx * ddy * (1 - ddz)
         + src[hx[X], ly[Y], hz[Z]] * ddx * (1 - ddy) * ddz
         + src[lx[X], hy[Y], hz[Z]] * (1 - ddx) * ddy * ddz
         + src[hx[X], hy[Y], hz[Z]] * ddx * ddy * ddz)
    return r.reshape(-1)


def read_cube(fn, nx=None, ny=None, nz=None, nspin=None, nat=None) -> Cube:
    """ModuleIO::read_cube (read_cube.cpp:3-120) for one process: the header (nspin, Fermi energy, atoms,
    grid) and the values in r order; a file whose grid differs from (nx, ny, nz) is interpolated
    trilinearly (read_cube_core_mismatch).  nspin / nat, when given, are checked as the reference does."""
    nspin_f, ef, nat_f, grid, axes, atoms, vals = _read_cube_text(Path(fn).read_text())
    if nspin is not None and nspin != 4 and nspin_f != nspin:
        raise ValueError(f"nspin mismatch: {nspin} in INPUT parameters but {nspin_f} in {fn}")
    if nat is not None and nat_f != nat:
        raise ValueError(f"number of atoms in {fn} is {nat_f}, expected {nat}")
    nxr, nyr, nzr = grid
    if vals.size != nxr * nyr * nzr:
        raise ValueError(f"{fn}: {vals.size} values for a {nxr}x{nyr}x{nzr} grid")
    want = (nx or nxr, ny or nyr, nz or nzr)
    data = vals if want == grid else trilinear_interpolate(vals, nxr, nyr, nzr, *want)
    return Cube(nspin=nspin_f, ef=ef, nat=nat_f, grid=want, axes=axes, atoms=atoms, data=data)


# ------------------------------------------------------------------ NSCF outputs
def nscf_diag_thr(pw_diag_thr, scf_thr, nelec):
    """The threshold ESolver_KS_PW::nscf gives the band solver (pw_nscf.cpp:63-68)."""
    if pw_diag_thr - 1e-2 > -1e-5:
        return max(1e-13, 0.1 * min(1e-2, scf_thr / nelec))
    return pw_diag_thr


def _cfmt(x: float, precision: int) -> str:
    return f" {x:.{precision}f}"


def nscf_band(fn, ekb, kvec_c, kl_segids, fermie=0.0, precision=8, is_=0, isk=None):
    """ModuleIO::nscf_band (nscf_band.cpp:9-124) for one pool: per k-point of spin is_ its 1-based index, the
    path length (|dk| summed within a segment, units of 2 pi / lat0) and (e - E_F) in eV."""
    ekb = np.asarray(ekb, dtype=np.float64)
    kv = np.asarray(kvec_c, dtype=np.float64)
    nks = len(kv)
    klen = np.zeros(nks)
    for ik in range(1, nks):
        d = kv[ik] - kv[ik - 1]
        klen[ik] = klen[ik - 1] + (math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
                                   if kl_segids[ik] == kl_segids[ik - 1] else 0.0)
    lines = []
    for ik in range(nks):
        if isk is not None and isk[ik] != is_:
            continue
        s = f"{ik + 1:4d}" + _cfmt(klen[ik], precision)
        s += "".join(_cfmt((e - fermie) * RY_TO_EV, precision) for e in ekb[ik])
        lines.append(s + "\n")
    with open(fn, "w") as f:
        f.write("".join(lines))
    return lines


def running_band_lines(ekb, wg, kvec_c, nkstot, isk=None):
    """The eigenvalue block ESolver_KS_PW::nscf writes to the running log (pw_nscf.cpp:80-101), nspin 1:
    ' k-points<ik>(<nkstot>): kx ky kz' then ' spin<is>_final_band <ib> <e in eV> <wg * nks>' per band."""
    nks = len(ekb)
    out = []
    for ik in range(nks):
        kx, ky, kz = (float(v) for v in kvec_c[ik])
        out.append(f" k-points{ik + 1}({nkstot}): {_cxx_g(kx, 0)} {_cxx_g(ky, 0)} {_cxx_g(kz, 0)}\n")
        s = 1 if isk is None else int(isk[ik]) + 1
        for ib in range(len(ekb[ik])):
            out.append(f" spin{s}_final_band {ib + 1} {_cxx_g(float(ekb[ik][ib]) * RY_TO_EV, 0)} "
                       f"{_cxx_g(float(wg[ik][ib]) * nks, 0)}\n")
        out.append("\n")
    return out
