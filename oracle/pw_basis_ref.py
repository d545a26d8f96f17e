"""CPU oracle (test infrastructure only): plane-wave basis set-up of ABACUS.

This file is a numpy restatement of the reference's G-sphere, FFT-grid and
index-map construction.  It is used by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the *checker*; nothing in the
product imports it.

Followed reference code (paths inside abacus-develop v3.8.0):
  * grid sizing ............ source/module_basis/module_pw/pw_init.cpp:24-140
  * k-dependent cut-offs ... source/module_basis/module_pw/pw_basis_k.cpp:53-116
  * sticks / G ordering .... source/module_basis/module_pw/pw_distributeg.cpp:44-200
                             (count_pw_st, get_ig2isz_is2fftixy; serial
                             stick order of pw_distributeg_method1.cpp:84-97)
  * k sphere ............... source/module_basis/module_pw/pw_basis_k.cpp:118-168
  * |k+G|^2, gcar .......... source/module_basis/module_pw/pw_basis_k.cpp:189-265
  * ig2ixyz_k ............... source/module_basis/module_pw/pw_basis_k.cpp:319-344
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TWO_PI = 2.0 * math.pi


def _smooth235(n: int) -> int:
    """Smallest m >= n whose only prime factors are 2, 3, 5 (pw_init.cpp:95-135)."""
    m = n
    while True:
        b = m
        for p in (2, 3, 5):
            while b % p == 0:
                b //= p
        if b == 1:
            return m
        m += 1


def init_grids(lat0: float, latvec: np.ndarray, gridecut: float):
    """Restates PW_Basis::initgrids(lat0, latvec, gridecut) (pw_init.cpp:24-140).

    Returns (nx, ny, nz, tpiba2, G, GGT, gridecut_lat, omega)."""
    latvec = np.asarray(latvec, dtype=np.float64)
    tpiba = TWO_PI / lat0
    tpiba2 = tpiba * tpiba
    GT = np.linalg.inv(latvec)
    G = GT.T
    GGT = G @ GT
    gridecut_lat = gridecut / tpiba2
    ibox = [int(math.sqrt(gridecut_lat) * math.sqrt(float(latvec[i] @ latvec[i]))) + 1 for i in range(3)]
    n = [0, 0, 0]
    rz = np.arange(-ibox[2], ibox[2] + 1)
    ry = np.arange(-ibox[1], ibox[1] + 1)
    rx = np.arange(-ibox[0], ibox[0] + 1)
    fz, fy, fx = np.meshgrid(rz, ry, rx, indexing="ij")
    f = np.stack([fx, fy, fz], -1).reshape(-1, 3).astype(np.float64)
    mod = np.einsum("ni,ij,nj->n", f, GGT, f)
    sel = f[mod <= gridecut_lat]
    for d in range(3):
        n[d] = int(np.max(np.abs(sel[:, d]))) if len(sel) else 0
    ib = [2 * n[d] + 1 for d in range(3)]
    nx, ny, nz = (_smooth235(v) for v in ib)
    omega = abs(np.linalg.det(latvec)) * lat0 ** 3
    return nx, ny, nz, tpiba2, G, GGT, gridecut_lat, omega


@dataclass
class PWBasisKRef:
    """Oracle mirror of ModulePW::PW_Basis_K for one pool (1 process)."""

    lat0: float
    latvec: np.ndarray
    ecutwfc: float
    kvec_d: np.ndarray  # (nks, 3) direct coordinates
    ecutrho: float | None = None
    grid: tuple | None = None  # explicit (nx, ny, nz), pw_init.cpp:146-170 overload
    # outputs
    nx: int = 0
    ny: int = 0
    nz: int = 0
    tpiba2: float = 0.0
    omega: float = 0.0
    npwk: np.ndarray = field(default=None)
    npwk_max: int = 0
    nst: int = 0
    is2fftixy: np.ndarray = field(default=None)
    ig2isz: np.ndarray = field(default=None)
    igl2isz_k: np.ndarray = field(default=None)
    ig2ixyz_k: np.ndarray = field(default=None)
    gk2: np.ndarray = field(default=None)
    gcar: np.ndarray = field(default=None)
    kvec_c: np.ndarray = field(default=None)
    miller_k: list = field(default=None)

    def __post_init__(self):
        latvec = np.asarray(self.latvec, dtype=np.float64)
        self.latvec = latvec
        ecutrho = 4.0 * self.ecutwfc if self.ecutrho is None else self.ecutrho
        nx, ny, nz, tpiba2, G, GGT, gridecut_lat, omega = init_grids(self.lat0, latvec, ecutrho)
        if self.grid is not None:
            nx, ny, nz = self.grid
        self.nx, self.ny, self.nz = nx, ny, nz
        self.tpiba2 = tpiba2
        self.omega = omega
        self.G, self.GGT = G, GGT
        kvec_d = np.atleast_2d(np.asarray(self.kvec_d, dtype=np.float64))
        self.kvec_d = kvec_d
        nks = len(kvec_d)
        # pw_basis_k.cpp:66-81
        kvec_c = kvec_d @ G
        kmaxmod = float(np.max(np.sqrt(np.sum(kvec_c * kvec_c, axis=1)))) if nks else 0.0
        gk_ecut = self.ecutwfc / tpiba2
        ggecut = (math.sqrt(gk_ecut) + kmaxmod) ** 2
        if ggecut > gridecut_lat:
            ggecut = gridecut_lat
            gk_ecut = (math.sqrt(ggecut) - kmaxmod) ** 2
        self.kvec_c = kvec_c
        self.gk_ecut = gk_ecut
        self.ggecut = ggecut
        # count_pw_st + get_ig2isz_is2fftixy (pw_distributeg.cpp:44-200), serial order = ixy ascending
        ix_end = nx // 2 + 1
        iy_end = ny // 2 + 1
        iz_end = nz // 2 + 1
        fftny = ny
        st_len = np.zeros(nx * ny, dtype=np.int64)
        st_bot = np.zeros(nx * ny, dtype=np.int64)
        izs = np.arange(-iz_end, iz_end + 1, dtype=np.float64)
        for ix in range(-ix_end, ix_end + 1):
            for iy in range(-iy_end, iy_end + 1):
                x = ix + nx if ix < 0 else ix
                y = iy + ny if iy < 0 else iy
                f = np.stack([np.full_like(izs, ix), np.full_like(izs, iy), izs], -1)
                mod = np.einsum("ni,ij,nj->n", f, GGT, f)
                ok = np.nonzero(mod <= ggecut)[0]
                if len(ok):
                    idx = x * fftny + y
                    st_len[idx] = len(ok)
                    st_bot[idx] = int(izs[ok[0]])
        sticks = np.nonzero(st_len > 0)[0]
        self.nst = len(sticks)
        self.is2fftixy = sticks.astype(np.int64)
        ig2isz = []
        for s, ixy in enumerate(sticks):
            z0 = st_bot[ixy]
            for iz in range(z0, z0 + st_len[ixy]):
                z = iz + nz if iz < 0 else iz
                ig2isz.append(s * nz + z)
        self.ig2isz = np.asarray(ig2isz, dtype=np.int64)
        self.npw = len(self.ig2isz)
        # Miller indices of the ggecut sphere in basis order (cal_GplusK_cartesian, pw_basis_k.cpp:291-306)
        isz = self.ig2isz
        iz = isz % nz
        st = isz // nz
        ixy = self.is2fftixy[st]
        ix = ixy // fftny
        iy = ixy % fftny
        ix = np.where(ix >= nx // 2 + 1, ix - nx, ix)
        iy = np.where(iy >= ny // 2 + 1, iy - ny, iy)
        iz = np.where(iz >= nz // 2 + 1, iz - nz, iz)
        miller = np.stack([ix, iy, iz], -1).astype(np.float64)
        # setupIndGk (pw_basis_k.cpp:118-168)
        npwk = np.zeros(nks, dtype=np.int64)
        sel_k = []
        for ik in range(nks):
            q = kvec_c[ik] + miller @ G
            gk2 = np.sum(q * q, axis=1)
            sel = np.nonzero(gk2 <= gk_ecut)[0]
            npwk[ik] = len(sel)
            sel_k.append(sel)
        self.npwk = npwk
        self.npwk_max = int(np.max(npwk)) if nks else 0
        L = self.npwk_max
        self.igl2isz_k = np.zeros(nks * L, dtype=np.int64)
        self.ig2ixyz_k = np.zeros(nks * L, dtype=np.int64)
        self.gk2 = np.zeros(nks * L, dtype=np.float64)
        self.gcar = np.zeros((nks * L, 3), dtype=np.float64)
        self.miller_k = []
        for ik in range(nks):
            sel = sel_k[ik]
            n = len(sel)
            self.igl2isz_k[ik * L: ik * L + n] = isz[sel]
            f = miller[sel]
            # collect_local_pw (pw_basis_k.cpp:209-231): gk2 = (f+k)·GGT·(f+k), kv in direct coords
            fk = f + kvec_d[ik]
            self.gk2[ik * L: ik * L + n] = np.einsum("ni,ij,nj->n", fk, GGT, fk)
            self.gcar[ik * L: ik * L + n] = f @ G
            # get_ig2ixyz_k (pw_basis_k.cpp:319-344)
            s_ = isz[sel] // nz
            z_ = isz[sel] % nz
            ixy_ = self.is2fftixy[s_]
            self.ig2ixyz_k[ik * L: ik * L + n] = z_ + (ixy_ % ny) * nz + (ixy_ // ny) * ny * nz
            self.miller_k.append(f.astype(np.int64))

    @property
    def nxyz(self) -> int:
        return self.nx * self.ny * self.nz

    def ig2ixyz(self, ik: int) -> np.ndarray:
        L = self.npwk_max
        return self.ig2ixyz_k[ik * L: ik * L + self.npwk[ik]]

    def gk2_k(self, ik: int) -> np.ndarray:
        L = self.npwk_max
        return self.gk2[ik * L: ik * L + self.npwk[ik]]

    def gplusk_cart(self, ik: int) -> np.ndarray:
        """|k+G| cartesian vectors in bohr^-1 (getgpluskcar, pw_basis_k.cpp:280-284, times tpiba)."""
        L = self.npwk_max
        n = self.npwk[ik]
        return (self.gcar[ik * L: ik * L + n] + self.kvec_c[ik]) * math.sqrt(self.tpiba2)
