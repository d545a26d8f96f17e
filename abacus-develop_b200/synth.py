"""Seeded synthetic inputs for the plane-wave H|psi> / Davidson workloads.

A workload is a cell (lattice, displaced diamond-lattice atoms), a wavefunction
cut-off, a k-point set and a band count.  From a seed it yields:

  * V_eff(r) = -sum_atoms 2 Ry * exp(-|r - R|^2 / 2) on the FFT grid, minimum
    image, laid out r = (ix*ny + iy)*nz + iz (ABACUS's real-space order);
  * 8 Kleinman-Bylander projectors per atom, (l = 0, 1) x (r_c = 0.8, 1.2 bohr):
    beta(q) = c * (-i)^l |q|^l exp(-|q|^2 r_c^2 / 2) Y_lm(q^) exp(-i q.R),
    q = k + G in bohr^-1, c the continuum normalisation, stored like ABACUS's
    ``vkb`` (nkb x npwx, row-major);
  * a diagonal D (``deeq`` shaped (nspin, nat, nh, nh)), uniform in [-3, 3] Ry;
  * psi_0 = complex normal / (1 + |q|^2) on the sphere.

The G-sphere, grid and ordering come from the product's own PW_Basis_K set-up
(``basis.PWBasisK``), which reproduces the reference's ordering.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# fractional coordinates of the 8 atoms of the cubic diamond cell
_DIAMOND8 = np.array([
    [0.00, 0.00, 0.00], [0.00, 0.50, 0.50], [0.50, 0.00, 0.50], [0.50, 0.50, 0.00],
    [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25],
])

NH = 8  # projectors per atom
_PROJ = [(rc, l, m) for rc in (0.8, 1.2) for (l, m) in ((0, 0), (1, 0), (1, 1), (1, -1))]


@dataclass
class CellSpec:
    name: str
    a: float                       # lat0 (bohr)
    latvec: tuple                  # diagonal of the lattice matrix in units of a
    reps: tuple                    # diamond supercell repetitions (x, y, z); (0,0,0) => 2-atom cell
    ecut: float                    # ecutwfc (Ry)
    nbands: int
    grid: tuple | None = None      # explicit FFT grid (None => reference rule)
    kpts: np.ndarray | None = None # direct coordinates, default Gamma
    seed: int = 20250


def diamond_positions(spec: CellSpec) -> np.ndarray:
    """Cartesian positions (bohr) before displacement."""
    lv = np.diag(spec.latvec) * spec.a
    if spec.reps == (0, 0, 0):
        frac = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]])
        return frac @ lv
    rx, ry, rz = spec.reps
    pts = []
    for i in range(rx):
        for j in range(ry):
            for k in range(rz):
                for f in _DIAMOND8:
                    pts.append([(f[0] + i) / rx, (f[1] + j) / ry, (f[2] + k) / rz])
    return np.asarray(pts) @ lv


def mp_grid(n: int, shifted: bool = True) -> np.ndarray:
    """n x n x n Monkhorst-Pack k-points (direct coordinates)."""
    off = 0.5 if shifted else 0.0
    u = (np.arange(n) + off) / n
    u = np.where(u >= 0.5, u - 1.0, u)
    kk = np.array([[x, y, z] for x in u for y in u for z in u])
    return kk


def config(idx: int) -> CellSpec:
    """The five standard workloads (8/64/216-atom diamond cells, k-batched, serving cells)."""
    if idx == 0:
        return CellSpec("diamond8_ecut30", 10.26, (1, 1, 1), (1, 1, 1), 30.0, 32, seed=20250)
    if idx == 1:
        return CellSpec("diamond64_ecut50", 20.52, (1, 1, 1), (2, 2, 2), 50.0, 160, seed=20251)
    if idx == 2:
        return CellSpec("diamond8_mp444", 10.26, (1, 1, 1), (1, 1, 1), 30.0, 32,
                        kpts=mp_grid(4, True), seed=20252)
    if idx == 4:
        return CellSpec("diamond216_ecut40", 30.78, (1, 1, 1), (3, 3, 3), 40.0, 480,
                        grid=(128, 128, 128), seed=20254)
    raise ValueError(f"no single-cell workload {idx}")


def serving_cells() -> list[CellSpec]:
    """The four resident cells of the serving workload."""
    return [
        CellSpec("si2_ecut30", 5.13, (1, 1, 1), (0, 0, 0), 30.0, 8, seed=20253),
        CellSpec("diamond8_ecut30", 10.26, (1, 1, 1), (1, 1, 1), 30.0, 32, seed=20250),
        CellSpec("diamond16_ecut40", 10.26, (1, 1, 2), (1, 1, 2), 40.0, 64, seed=20256),
        CellSpec("diamond64_ecut50", 20.52, (1, 1, 1), (2, 2, 2), 50.0, 160, seed=20251),
    ]


def _ylm_real(l: int, m: int, q: np.ndarray) -> np.ndarray:
    qn = np.linalg.norm(q, axis=1)
    safe = np.where(qn > 1e-12, qn, 1.0)
    if l == 0:
        return np.full(len(q), 1.0 / math.sqrt(4 * math.pi))
    c = math.sqrt(3.0 / (4 * math.pi))
    comp = {0: 2, 1: 0, -1: 1}[m]
    return np.where(qn > 1e-12, c * q[:, comp] / safe, 0.0)


@dataclass
class SynthCell:
    spec: CellSpec
    lat0: float
    latvec: np.ndarray
    tau: np.ndarray              # (nat, 3) cartesian bohr, displaced
    dvals: np.ndarray            # (nkb,) D diagonal (Ry)
    rng_state: dict = field(default=None)

    @property
    def nat(self) -> int:
        return len(self.tau)

    @property
    def nkb(self) -> int:
        return NH * self.nat

    def deeq(self) -> np.ndarray:
        """deeq(nspin=1, nat, nh, nh) with D on the diagonal."""
        d = np.zeros((1, self.nat, NH, NH))
        for ia in range(self.nat):
            d[0, ia][np.diag_indices(NH)] = self.dvals[ia * NH:(ia + 1) * NH]
        return d

    def veff(self, nx: int, ny: int, nz: int) -> np.ndarray:
        """V_eff(r) in the reference layout r = (ix*ny + iy)*nz + iz (float64, Ry)."""
        L = np.diag(self.latvec) * self.lat0
        if not np.allclose(self.latvec, np.diag(np.diag(self.latvec))):
            raise ValueError("synthetic V_eff supports orthorhombic cells")
        gx = np.arange(nx) / nx * L[0]
        gy = np.arange(ny) / ny * L[1]
        gz = np.arange(nz) / nz * L[2]
        v = np.zeros((nx, ny, nz))
        for R in self.tau:
            dx = gx - R[0]
            dx -= L[0] * np.round(dx / L[0])
            dy = gy - R[1]
            dy -= L[1] * np.round(dy / L[1])
            dz = gz - R[2]
            dz -= L[2] * np.round(dz / L[2])
            ex = np.exp(-0.5 * dx * dx)
            ey = np.exp(-0.5 * dy * dy)
            ez = np.exp(-0.5 * dz * dz)
            v -= 2.0 * ex[:, None, None] * ey[None, :, None] * ez[None, None, :]
        return v.reshape(-1)

    def vkb(self, q: np.ndarray, npwx: int, omega: float) -> np.ndarray:
        """Projectors at q = k+G (npw x 3, bohr^-1), returned as (nkb, npwx) row-major complex128."""
        npw = len(q)
        out = np.zeros((self.nkb, npwx), dtype=np.complex128)
        qn2 = np.sum(q * q, axis=1)
        qn = np.sqrt(qn2)
        radial = {}
        for rc in (0.8, 1.2):
            for l in (0, 1):
                # continuum normalisation: sum_G |beta|^2 ~ Omega/(2pi)^3 * Gamma(l+3/2)/(2 rc^(2l+3))
                integ = math.gamma(l + 1.5) / (2.0 * rc ** (2 * l + 3))
                c = math.sqrt((2 * math.pi) ** 3 / omega / integ)
                radial[(rc, l)] = c * qn ** l * np.exp(-0.5 * qn2 * rc * rc)
        for ia, R in enumerate(self.tau):
            sk = np.exp(-1j * (q @ R))
            for j, (rc, l, m) in enumerate(_PROJ):
                out[ia * NH + j, :npw] = ((-1j) ** l) * radial[(rc, l)] * _ylm_real(l, m, q) * sk
        return out

    def projector_tables(self, omega: float, ecut: float, dq: float = 0.01):
        """The same projectors as ``vkb`` as getvnl tables: one atom type, 4 radial functions (r_c, l) on a q
        grid of step dq reaching past sqrt(ecut), 8 (beta, l, lm) channels per atom in the order of ``vkb``.
        getvnl's real Y_lm differ from ``vkb``'s by a sign for (l, m) = (1, +-1); D is diagonal, so the
        Hamiltonian is the same."""
        from .pwdft import ProjectorSet
        nq = int(math.sqrt(ecut) / dq + 4) + 1
        q = np.arange(nq) * dq
        betas = [(0.8, 0), (0.8, 1), (1.2, 0), (1.2, 1)]
        tab = np.zeros((1, len(betas), nq))
        for ib, (rc, l) in enumerate(betas):
            integ = math.gamma(l + 1.5) / (2.0 * rc ** (2 * l + 3))
            c = math.sqrt((2 * math.pi) ** 3 / omega / integ)
            tab[0, ib] = c * q ** l * np.exp(-0.5 * q * q * rc * rc)
        indv = np.array([[0, 1, 1, 1, 2, 3, 3, 3]])
        nhtol = np.array([[0, 1, 1, 1, 0, 1, 1, 1]])
        nhtolm = np.array([[0, 1, 2, 3, 0, 1, 2, 3]])
        return ProjectorSet(ntype=1, na=[self.nat], nbeta=[len(betas)], nh=[NH], nhm=NH, lmax=1, indv=indv,
                            nhtol=nhtol, nhtolm=nhtolm, tab=tab, dq=dq)

    def psi0(self, q: np.ndarray, nbands: int, npwx: int, seed_offset: int = 0) -> np.ndarray:
        """Start vectors, (nbands, npwx) row-major complex128 (band b at b*npwx)."""
        rng = np.random.Generator(np.random.PCG64(self.spec.seed * 7919 + 17 + seed_offset))
        npw = len(q)
        w = 1.0 / (1.0 + np.sum(q * q, axis=1))
        re = rng.standard_normal((nbands, npw))
        im = rng.standard_normal((nbands, npw))
        out = np.zeros((nbands, npwx), dtype=np.complex128)
        out[:, :npw] = (re + 1j * im) * w[None, :]
        return out


def make_cell(spec: CellSpec) -> SynthCell:
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    pos = diamond_positions(spec)
    tau = pos + rng.normal(0.0, 0.05, size=pos.shape)
    dvals = rng.uniform(-3.0, 3.0, size=NH * len(pos))
    return SynthCell(spec=spec, lat0=spec.a, latvec=np.diag(np.asarray(spec.latvec, dtype=np.float64)),
                     tau=tau, dvals=dvals)
