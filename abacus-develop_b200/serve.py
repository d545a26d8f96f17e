"""Serving loop for non-self-consistent band solves: resident cells, requests admitted as they arrive.

``Server`` wraps the native server (include/abacus_b200.h, ``b200_server_*``): worker threads with one
non-blocking stream each; an idle worker takes the oldest queued request whose cell is under its in-flight
cap and whose solver slot fits in the HBM budget (first come, first served within a cell); pooled solver
slots are re-targeted to each request's k-point.

``build_serving_cells`` makes the resident cells of the serving workload (the 2-, 8-, 16- and 64-atom
diamond-lattice cells, each with a high-symmetry k-path whose projectors are built on the device by
getvnl); ``poisson_load`` replays Poisson arrivals against a server and reports latency percentiles and
throughput.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import call
from .pwdft import PREC_FP64, PREC_MIXED, HamiltPW, PWBasisK, _torch  # noqa: F401

STATUS_OK = 0
STATUS_SHED = 9  # waited past the cell's admission bound (server policy with shedding)


@dataclass
class Result:
    id: int
    status: int
    t_submit: float
    t_admit: float
    t_done: float
    iters: int
    iters_low: int
    eig: np.ndarray
    tag: object = None

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class Server:
    def __init__(self, hbm_budget_bytes: int = 40 << 30, nworkers: int = 8, david_ndim: int = 4):
        h = _lib.vp()
        call("b200_server_create", int(hbm_budget_bytes), int(nworkers), int(david_ndim), C.byref(h))
        self._h = h
        self._lib = _lib.load()
        self._cells = []
        self._pending = {}
        self._mu = threading.Lock()

    def set_policy(self, policy: int = 0, shed_factor: float = 0.0):
        """Admission: policy 0 oldest first, 1 highest response ratio (wait + S_c) / S_c first; shed_factor > 0
        completes requests that waited past shed_factor * S_c with STATUS_SHED (S_c: the cell's mean service)."""
        call("b200_server_set_policy", self._h, int(policy), float(shed_factor))

    def set_express(self, nworkers: int = 0, max_service_s: float = 0.0):
        """Workers 0..nworkers-1 take only requests of cells whose mean service time is at most max_service_s
        (cells not yet timed included); 0 turns it off."""
        call("b200_server_set_express", self._h, int(nworkers), float(max_service_s))

    def add_cell(self, hamilt: HamiltPW, max_inflight: int = 2) -> int:
        """Register a resident cell; at most max_inflight of its requests run at once."""
        cid = C.c_int()
        call("b200_server_add_cell", self._h, hamilt.handle, int(max_inflight), C.byref(cid))
        self._cells.append(hamilt)
        return cid.value

    def submit(self, cell: int, ik: int, nbands: int, thr: float = 1e-9, precision: int = PREC_MIXED,
               seed: int | None = None, maxiter: int = 300, tag=None) -> int:
        if seed is None:
            seed = request_seed(cell, ik, nbands)
        eig = np.zeros(nbands)
        rid = C.c_longlong()
        with self._mu:
            call("b200_server_submit", self._h, cell, ik, nbands, precision, float(thr), int(maxiter),
                 int(seed) & 0xFFFFFFFFFFFFFFFF, eig.ctypes.data_as(_lib.pf64), C.byref(rid))
            self._pending[rid.value] = (eig, tag)
        return rid.value

    def poll(self, wait: bool = False, max_out: int = 256) -> list:
        ids = (C.c_longlong * max_out)()
        st = (C.c_int * max_out)()
        ts, ta, td = (C.c_double * max_out)(), (C.c_double * max_out)(), (C.c_double * max_out)()
        it, itl = (C.c_int * max_out)(), (C.c_int * max_out)()
        n = C.c_int()
        call("b200_server_poll", self._h, max_out, int(wait), ids, st, ts, ta, td, it, itl, C.byref(n))
        out = []
        with self._mu:
            for i in range(n.value):
                eig, tag = self._pending.pop(ids[i])
                out.append(Result(ids[i], st[i], ts[i], ta[i], td[i], it[i], itl[i], eig, tag))
        return out

    def drain(self) -> list:
        call("b200_server_drain", self._h)
        res = []
        while True:
            r = self.poll(wait=False)
            if not r:
                return res
            res.extend(r)

    def stats(self) -> dict:
        a = (C.c_double * 6)()
        call("b200_server_stats", self._h, a)
        return {"pool_bytes": a[0], "peak_pool_bytes": a[1], "peak_in_flight": int(a[2]),
                "slots_created": int(a[3]), "slots_evicted": int(a[4]), "clock_s": a[5]}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.b200_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def request_seed(cell: int, ik: int, nbands: int) -> int:
    """Start-vector seed of a request: a function of what is asked only, so that a request gives the same
    result alone and among others."""
    return ((cell * 1000003 + ik) * 1009 + nbands) * 0x9E3779B1 + 12345


def high_symmetry_path(npts: int = 16) -> np.ndarray:
    """Gamma - X - M - Gamma - R of a simple-cubic / tetragonal Brillouin zone, npts points (direct coords)."""
    corners = np.array([[0, 0, 0], [0.5, 0, 0], [0.5, 0.5, 0], [0, 0, 0], [0.5, 0.5, 0.5]], dtype=np.float64)
    seg = np.linalg.norm(np.diff(corners, axis=0), axis=1)
    s = np.linspace(0.0, seg.sum(), npts)
    cum = np.concatenate([[0.0], np.cumsum(seg)])
    pts = []
    for x in s:
        i = min(int(np.searchsorted(cum, x, side="right")) - 1, len(seg) - 1)
        t = (x - cum[i]) / seg[i]
        pts.append(corners[i] + t * (corners[i + 1] - corners[i]))
    return np.array(pts)


@dataclass
class ServingCell:
    spec: object
    cell: object
    basis: PWBasisK
    hamilt: HamiltPW
    kpath: np.ndarray
    nbands: int
    keep: list = field(default_factory=list)


def build_serving_cells(specs=None, npath: int = 16) -> list:
    """Resident cells: V_eff, D and the projectors of every k-point of the path on the device."""
    from . import synth
    torch = _torch()
    specs = synth.serving_cells() if specs is None else specs
    out = []
    for spec in specs:
        cell = synth.make_cell(spec)
        kp = high_symmetry_path(npath)
        basis = PWBasisK(spec.a, cell.latvec, spec.ecut, kp, grid=spec.grid)
        h = HamiltPW(basis, PREC_FP64)
        veff = torch.from_numpy(cell.veff(basis.nx, basis.ny, basis.nz)).cuda()
        h.set_veff(veff)
        deeq = torch.from_numpy(cell.deeq()).cuda()
        h.set_deeq([cell.nat], [synth.NH], deeq)
        h.set_projectors(cell.projector_tables(basis.omega, spec.ecut), cell.tau / spec.a)
        for ik in range(basis.nks):
            h.build_vkb(ik)
        torch.cuda.synchronize()
        out.append(ServingCell(spec, cell, basis, h, kp, spec.nbands, keep=[veff, deeq]))
    return out


def percentile(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else float("nan")


def summarize(results, cells) -> dict:
    ok = [r for r in results if r.status == STATUS_OK]
    lat = [r.latency for r in ok]
    first = min(r.t_submit for r in results)
    last = max(r.t_done for r in results)
    per_cell = {}
    for c in range(len(cells)):
        rc = [r for r in ok if r.tag[0] == c]
        lc = [r.latency for r in rc]
        per_cell[cells[c].spec.name] = {
            "n": len(lc), "p50_ms": 1e3 * percentile(lc, 50), "p99_ms": 1e3 * percentile(lc, 99),
            "service_p50_ms": 1e3 * percentile([r.t_done - r.t_admit for r in rc], 50)}
    shed = sum(1 for r in results if r.status == STATUS_SHED)
    return {"n": len(results), "n_ok": len(ok), "n_shed": shed, "throughput_rps": len(ok) / (last - first),
            "p50_ms": 1e3 * percentile(lat, 50), "p99_ms": 1e3 * percentile(lat, 99), "per_cell": per_cell}


def poisson_load(server: Server, cell_ids: list, cells: list, rate: float, nreq: int, seed: int = 7,
                 thr: float = 1e-9, precision: int = PREC_MIXED) -> dict:
    """Open-loop Poisson arrivals (mean `rate` per second) of `nreq` requests, cell uniform, k-point uniform
    on the cell's path, nbands the cell's; returns the results with latency / throughput figures."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=nreq)
    which = rng.integers(0, len(cells), size=nreq)
    ks = [int(rng.integers(0, cells[c].basis.nks)) for c in which]
    t0 = time.perf_counter()
    arrive = np.cumsum(gaps)
    for i in range(nreq):
        dt = arrive[i] - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        c = int(which[i])
        server.submit(cell_ids[c], ks[i], cells[c].nbands, thr=thr, precision=precision, tag=(c, ks[i]))
    res = server.drain()
    out = summarize(res, cells)
    out["offered_rate"] = rate
    out["wall_s"] = time.perf_counter() - t0
    out["results"] = res
    return out
