"""Non-self-consistent band solve on the device: ESolver_KS_PW::nscf (module_esolver/pw_nscf.cpp:54-200) for one
pool, norm-conserving pseudopotentials, nspin = 1.

  1. V_eff from a cube file (``out_pot``; interpolated when its grid differs, read_cube.cpp) or an array;
  2. the solver threshold from pw_diag_thr / scf_thr / nelec (pw_nscf.cpp:63-68);
  3. Davidson solves of all k-points on the device (HSolverPW::solve's k loop, the k-points concurrent;
     NSCF exit rule: every band converged, up to 5 retries, hsolver_pw.cpp:580-593), start vectors from
     wavefunction files (``init_wfc file``, read_wfc_pw.cpp) or given arrays;
  4. occupations and the Fermi energy: fixed for an insulator (Occupy::iweights, occupy.cpp:132-186) or
     smeared (Occupy::gweights / efermig, occupy.cpp:203-366: Gaussian, Methfessel-Paxton 1-2, cold,
     Fermi-Dirac);
  5. outputs: the eigenvalue block of the running log, the band-structure file (nscf_band.cpp) and, on
     request, the wavefunction files (write_wfc_pw.cpp).
The band solve is the library's (b200_solve_kpoints); this module is the host-side driver around it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import nscf_io
from . import pwdft as P


def occupation_weights(ekb, wk, nelec):
    """Occupy::iweights for nspin = 1 (is = -1): the lowest nelec / 2 bands of every k-point carry the k
    weight, the rest none; E_F is the highest occupied eigenvalue.  Metals (nelec / 2 not an integer) are
    refused, as the reference refuses fixed occupations for them."""
    ekb = np.asarray(ekb, dtype=np.float64)
    ib_mind = nelec / 2.0
    ib_min = math.ceil(ib_mind)
    if ib_min != int(ib_mind):
        raise ValueError("It is not a semiconductor or insulator. Please do not set 'smearing_method=fixed', "
                         "and try other options.")
    wg = np.zeros_like(ekb)
    wg[:, :ib_min] = np.asarray(wk, dtype=np.float64)[:, None]
    ef = float(np.max(ekb[:, :ib_min])) if ib_min > 0 else -1e10
    return wg, ef


SMEARING_TYPES = {"gaussian": 0, "gauss": 0, "methfessel-paxton": 1, "mp": 1, "mp2": 2,
                  "marzari-vanderbilt": -1, "cold": -1, "mv": -1, "fermi-dirac": -99, "fd": -99}


def smearing_type(method: str) -> int:
    """Occupy::decision's smearing_method -> ngauss (occupy.cpp:27-107)."""
    if method == "mp3":
        raise ValueError("Some refactor of smearing shoule be done before supporting any order of "
                         "Methfessel-Paxton method!")
    if method not in SMEARING_TYPES:
        raise ValueError(f"unknown smearing_method {method!r}")
    return SMEARING_TYPES[method]


_SQRT2 = math.sqrt(2.0)


def wgauss(x: float, n: int) -> float:
    """Occupy::wgauss (occupy.cpp:428-500): the smeared step function of order n at x."""
    maxarg = 200.0
    if n == -99:
        if x < -maxarg:
            return 0.0
        if x > maxarg:
            return 1.0
        return 1.0 / (1.0 + math.exp(-x))
    if n == -1:
        xp = x - 1.0 / _SQRT2
        arg = min(maxarg, xp * xp)
        return 0.5 * math.erf(xp) + 1.0 / math.sqrt(2.0 * math.pi) * math.exp(-arg) + 0.5
    wga = 0.5 * (1 - math.erf(-x))
    if n == 0:
        return wga
    ni = 0
    arg = min(maxarg, x * x)
    hp = math.exp(-arg)
    h0, h1 = 1.0, -2.0 * x
    a = 1.0 / math.sqrt(math.pi)
    for i in range(n):
        a = -a / (float(i + 1) * 4.0)
        wga = wga + a * h1 * hp
        ni += 1
        h0 = 2.0 * (-x) * h1 - 2.0 * float(ni) * h0
        ni += 1
        h1 = 2.0 * (-x) * h0 - 2.0 * float(ni) * h1
    return wga


def w1gauss(x: float, n: int) -> float:
    """Occupy::w1gauss (occupy.cpp:502-611): the integral of y delta(y) up to x (for Fermi-Dirac the negative
    of the entropy term)."""
    if n == -99:
        if abs(x) <= 36.0:
            f = 1.0 / (1.0 + math.exp(-x))
            onemf = 1.0 - f
            return f * math.log(f) + onemf * math.log(onemf)
        return 0.0
    if n == -1:
        xp = x - 1.0 / _SQRT2
        arg = min(200.0, xp * xp)
        return 1.0 / math.sqrt(2.0 * math.pi) * xp * math.exp(-arg)
    arg = min(200.0, x * x)
    w1 = -0.5 * math.exp(-arg) / math.sqrt(math.pi)
    if n == 0:
        return w1
    ni = 0
    hp = math.exp(-arg)
    h0, h1 = 1.0, 2.0 * x
    a = 1.0 / math.sqrt(math.pi)
    for i in range(n):
        a = -a / (float(i + 1) * 4.0)
        ni += 1
        h0m1 = h0
        h0 = 2.0 * x * h1 - 2.0 * float(ni) * h0
        ni += 1
        h1 = 2.0 * x * h0 - 2.0 * float(ni) * h1
        w1 = w1 - a * (0.5 * h0 + float(ni) * h0m1) * hp
    return w1


def _sumkg(ekb, wk, sigma, ngauss, e):
    """Occupy::sumkg (occupy.cpp:399-426): the number of states below e."""
    s2 = 0.0
    for ik in range(ekb.shape[0]):
        s1 = 0.0
        for ib in range(ekb.shape[1]):
            s1 += wgauss((e - ekb[ik, ib]) / sigma, ngauss)
        s2 += wk[ik] * s1
    return s2


def fermi_energy(ekb, wk, nelec, sigma, ngauss):
    """Occupy::efermig (occupy.cpp:263-366): bisection for the Fermi energy between bounds widened by 2 sigma
    until they bracket nelec, to 1e-10 electrons or 300 steps."""
    ekb = np.asarray(ekb, dtype=np.float64)
    eps, maxiter = 1.0e-10, 300
    elw = float(np.min(ekb[:, 0])) - 2 * sigma
    eup = float(np.max(ekb[:, -1])) + 2 * sigma
    changes = 0
    while True:
        sumkup = _sumkg(ekb, wk, sigma, ngauss, eup)
        sumklw = _sumkg(ekb, wk, sigma, ngauss, elw)
        if changes > 1000:
            raise ValueError("ERROS in SMEARING")
        if (sumkup - nelec) < -eps:
            eup += 2 * sigma
        elif (sumklw - nelec) > eps:
            elw -= 2 * sigma
        else:
            break
        changes += 1
    ef = 0.5 * (eup + elw)
    for _ in range(maxiter):
        ef = (eup + elw) / 2.0
        s = _sumkg(ekb, wk, sigma, ngauss, ef)
        if abs(s - nelec) < eps:
            return ef
        if (s - nelec) < -eps:
            elw = ef
        else:
            eup = ef
    return ef


def smearing_weights(ekb, wk, nelec, sigma, method="gaussian"):
    """Occupy::gweights (occupy.cpp:203-246), nspin = 1: (wg, E_F, demet) for a smeared occupation of
    method ('gaussian', 'mp', 'mp2', 'mv' / 'cold', 'fd', and the reference's long names) and width sigma
    (Ry); demet is the correction to the band-energy sum."""
    if sigma == 0.0:
        raise ValueError("Smearing requires gaussian broadening,but gaussian_parameter = 0(default value = 0.01)")
    n = smearing_type(method)
    ekb = np.asarray(ekb, dtype=np.float64)
    wk = np.asarray(wk, dtype=np.float64)
    ef = fermi_energy(ekb, wk, nelec, sigma, n)
    wg = np.zeros_like(ekb)
    demet = 0.0
    for ik in range(ekb.shape[0]):
        for ib in range(ekb.shape[1]):
            x = (ef - ekb[ik, ib]) / sigma
            wg[ik, ib] = wk[ik] * wgauss(x, n)
            demet += wk[ik] * sigma * w1gauss(x, n)
    return wg, ef, demet


def load_veff_cube(fn, basis):
    """V_eff(r) of a cube file on the basis's grid (r order), interpolated when the grids differ."""
    return nscf_io.read_cube(fn, basis.nx, basis.ny, basis.nz).data


def read_start_wavefunctions(prefix, basis, nbands, nkstot, latvec):
    """The start vectors of every k-point from ``<prefix><ik+1>.dat`` (init_wfc file)."""
    return [nscf_io.read_wfc_pw(f"{prefix}{ik + 1}.dat", basis, ik, nkstot, nbands, latvec) for ik in range(basis.nks)]


@dataclass
class NscfResult:
    ekb: np.ndarray            # (nks, nbands) Ry
    wg: np.ndarray             # (nks, nbands) occupation weights
    ef: float                  # Ry
    iters: np.ndarray          # Davidson iterations per k-point
    diag_thr: float
    psis: list = field(default_factory=list)       # host eigenvectors of this rank's k-points, (nbands, npwk)
    files: dict = field(default_factory=dict)      # written outputs
    running_lines: list = field(default_factory=list)
    iks: list = field(default_factory=list)        # the k-points this rank solved (psis follow this order)


def device_solve(hamilt, *, precision=P.PREC_FP64, david_ndim=4, maxiter=50, nworkers=4):
    """The band solve of run_nscf_pool on this rank's GPU: b200_solve_kpoints over the rank's k-points, NSCF
    exit rule (ntry_max 5, notconv_max 0, hsolver_pw.cpp:580-593)."""
    def solve(iks, psi_init, nbands, thr):
        import torch
        basis = hamilt.basis
        ld = basis.npwk_max
        if not iks:
            return np.zeros((0, nbands)), np.zeros(0, dtype=np.int32), []
        psis_d, pcs = [], []
        for q, ik in enumerate(iks):
            npw = int(basis.npwk[ik])
            x = np.zeros((nbands, ld), dtype=np.complex128)
            x[:, :npw] = np.asarray(psi_init[q])[:nbands, :npw]
            psis_d.append(torch.from_numpy(x.reshape(-1)).cuda())
            pcs.append(P.precondition_d(basis, ik))
        ekb, its = hamilt.solve_kpoints(list(iks), pcs, psis_d, ld, nbands, thr, maxiter, david_ndim=david_ndim,
                                        precision=precision, nworkers=nworkers, ntry_max=5, notconv_max=0)
        torch.cuda.synchronize()
        psis = [p.cpu().numpy().reshape(nbands, ld)[:, :int(basis.npwk[ik])].copy() for ik, p in zip(iks, psis_d)]
        return ekb, its, psis
    return solve


def run_nscf_pool(basis, nbands, psi_init, solve, *, wk, nelec, latvec, ecutwfc, pw_diag_thr=1e-2, scf_thr=1e-9,
                  out_dir=None, out_wfc_pw=0, kl_segids=None, band_precision=8, group=None, smearing=None):
    """The NSCF run of one rank of a k-point pool split (one pool per GPU, module_base/module_device/
    device.cpp:195-217): this rank solves its share of the k-points (kpool.partition, cost npwk * nbands^2)
    with solve(iks, psi_init_of_those, nbands, thr) -> (ekb, iters, eigenvectors); the eigenvalues are
    all-gathered (the only collective); occupations, the Fermi energy and the band / running-log files come
    from the gathered eigenvalues (files on rank 0), each rank writes the wavefunction files of its own
    k-points.  psi_init[ik] is indexed by global k-point (entries of other ranks' k-points are not read).
    smearing: None for fixed occupations, else (method, sigma in Ry)."""
    from . import kpool
    ws, rank = 1, 0
    try:
        import torch.distributed as dist
        if dist.is_initialized():
            ws, rank = dist.get_world_size(group), dist.get_rank(group)
    except ImportError:
        pass
    nks = basis.nks
    thr = nscf_io.nscf_diag_thr(pw_diag_thr, scf_thr, nelec)
    mine = kpool.partition(basis.npwk, nbands, ws)[rank]
    ekb_l, its_l, psis_l = solve(mine, [psi_init[ik] for ik in mine], nbands, thr)
    ekb = kpool.gather_eigenvalues({ik: ekb_l[q] for q, ik in enumerate(mine)}, nks, nbands, group)
    its = kpool.gather_eigenvalues({ik: [float(its_l[q])] for q, ik in enumerate(mine)}, nks, 1, group)[:, 0]
    if smearing is None:
        wg, ef = occupation_weights(ekb, wk, nelec)
    else:
        wg, ef, _ = smearing_weights(ekb, wk, nelec, smearing[1], smearing[0])
    kvec_c = np.array([basis.kvec_c(ik) for ik in range(nks)])
    res = NscfResult(ekb=ekb, wg=wg, ef=ef, iters=its.astype(np.int64), diag_thr=thr, psis=psis_l, iks=list(mine))
    res.running_lines = [f" PW_DIAG_THR  = {thr:g}\n"] + nscf_io.running_band_lines(ekb, wg, kvec_c, nks)
    if out_dir is not None:
        d = Path(out_dir)
        d.mkdir(parents=True, exist_ok=True)
        if rank == 0:
            seg = np.zeros(nks, dtype=int) if kl_segids is None else kl_segids
            nscf_io.nscf_band(d / "BANDS_1.dat", ekb, kvec_c, seg, ef, band_precision)
            (d / "running_nscf.log").write_text("".join(res.running_lines))
            res.files["band"] = str(d / "BANDS_1.dat")
            res.files["running"] = str(d / "running_nscf.log")
        if out_wfc_pw in (1, 2):
            res.files["wfc"] = []
            for q, ik in enumerate(mine):
                res.files["wfc"].append(nscf_io.write_wfc_pw_k(str(d / "WAVEFUNC"), basis, ik, psis_l[q],
                                                               kvec_c[ik], wk[ik], ecutwfc, latvec, nbands,
                                                               out_wfc_pw, nks))
    return res


def run_nscf(hamilt, nbands, psi_init, *, wk, nelec, latvec, ecutwfc, pw_diag_thr=1e-2, scf_thr=1e-9,
             precision=P.PREC_FP64, david_ndim=4, maxiter=50, nworkers=4, out_dir=None, out_wfc_pw=0,
             kl_segids=None, band_precision=8, group=None, smearing=None):
    """Solve nbands bands at every k-point of hamilt's basis (V_eff, D and the projectors already set) from the
    start vectors psi_init[ik] ((nbands, npwk) arrays in the basis's order), on this GPU or, under
    torch.distributed, on this rank's share of a k-point pool split.  Outputs go to out_dir when it is
    given: BANDS_1.dat (nscf_band.cpp), running_nscf.log (the eigenvalue block), WAVEFUNC<ik>.dat / .txt
    (out_wfc_pw 2 / 1)."""
    solve = device_solve(hamilt, precision=precision, david_ndim=david_ndim, maxiter=maxiter, nworkers=nworkers)
    return run_nscf_pool(hamilt.basis, nbands, psi_init, solve, wk=wk, nelec=nelec, latvec=latvec,
                         ecutwfc=ecutwfc, pw_diag_thr=pw_diag_thr, scf_thr=scf_thr, out_dir=out_dir,
                         out_wfc_pw=out_wfc_pw, kl_segids=kl_segids, band_precision=band_precision, group=group,
                         smearing=smearing)
