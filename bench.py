"""Benchmark: plane-wave H|psi> bands/s (FP64 and mixed) and Davidson time-to-1e-8 Ry on one B200.

Workload (default): 64-atom diamond supercell, a = 20.52 bohr, ecut 50 Ry,
96^3 FFT grid, npw = 51 627, 160 bands, 512 Kleinman-Bylander projectors,
Gamma point, seeded synthetic V_eff / projectors / D / psi (no dataset).

One step = one H|psi> (kinetic + local V_eff via the stick/plane FFT +
nonlocal projectors, whose FP64 products run on the int8 tensor cores as an
exact modular emulation) on the whole 160-band block, inputs resident in HBM.
psi + hpsi + projectors (about 690 MB) exceed the 126 MB L2, so no flush is
needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--skip-david] [--skip-216] [--skip-kbatch] [--skip-serve] [--skip-cpu] [--gemm-only]
                  [--solvers-only]

Besides the headline line, the same JSON line carries:
  e2e           the same H|psi> from pinned host psi to pinned host hpsi through b200_hamilt_hpsi_host
                (uploads, H|psi> pieces and downloads overlapped);
  psi_to_rho    rho(r) += w|psi(r)|^2 over the 160 bands (ElecStatePW::psiToRho);
  nonlocal      the projector part of the FP64 step, with the int8 tensor-core products and with cuBLAS;
  tc_gemm       the 3xTF32 tensor-core complex GEMM on the 216-atom subspace shapes and the projector
                shapes (--gemm-only runs only this, for profiling);
  fp64_gemm     FP64 complex GEMM (gemm_op) on the projector and 216-atom subspace shapes: cuBLAS ZGEMM
                against the FP64 tensor peak, and the int8 tensor-core emulation (b200_zgemm_i8);
  davidson      FP64 vs mixed Davidson on the 64-atom cell: wall time to thr 1e-9 and the time after which
                every eigenvalue stays within 1e-8 Ry of an FP64 solve to 1e-11 (per-iteration traces);
  davidson_216  the same on the 216-atom cell (128^3 grid, 480 bands, 1728 projectors);
  dav_subspace  Davidson with subspace rotation (Diago_DavSubspace, FP64) on the 64-atom cell next to
                DiagoDavid FP64, and on the 8-atom cell next to the reference's compiled CPU solver;
  bpcg          band-parallel CG (DiagoBPCG, FP64) on the 64-atom cell: a first- and a later-SCF-step call;
                on the 8-atom cell a later-step call next to the reference's compiled CPU solver;
  kbatch        64 uneven k-points of the 8-atom cell: batched H|psi>, per-k calls, CUDA-graph replay,
                concurrent Davidson of all k-points;
  serving       Poisson arrivals on four resident cells: p50 / p99 latency and throughput at the offered
                200 requests/s and at 70 % of the measured capacity.

Multi-GPU (torchrun): every rank runs an independent replica of the workload
(k-points / requests are independent units: weak scaling, no collective in the
data path); the step time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
WORKLOAD_NAME = ("64-atom diamond supercell a=20.52 bohr, ecut 50 Ry, 96^3 grid, npw 51627, "
                 "160 bands, 512 projectors, Gamma")
METRIC = "H|psi> bands/s (FP64) + Davidson time-to-1e-8 Ry, mixed vs FP64"
# band pieces of the end-to-end H|psi> pipeline, timed at set-up (the pipeline halves the first and last
# piece: 6 pieces of 160 bands are 16, 32, 32, 32, 32, 16)
E2E_PIECES = (4, 5, 6, 7, 8, 10)
# dram__bytes_read.sum + dram__bytes_write.sum of the fused local H|psi> kernels (3 launches: one band chunk
# of all 160 bands, the autotuner's choice, x 3 passes) for one 160-band FP64 application, from an ncu
# capture without cache flush (the local-pass traffic summary under profiles/)
NCU_TRAFFIC_LOCAL_FP64 = 2030089984


def load_package():
    name = "abacus_develop_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = ROOT / "abacus-develop_b200"
    spec = importlib.util.spec_from_file_location(name, pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms while running.  Entering waits (up to 3 s) for the
    sampler's first line, so that it is live when the timed region starts; only lines that arrive inside the
    region are summarised."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "50"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.n0 = len(self.lines)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.n1 = len(self.lines)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[getattr(self, "n0", 0):getattr(self, "n1", len(self.lines))]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def time_steps(fn, steps, stream):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def local_flops_per_band(basis):
    """Algorithmic flops of the local part of H|psi> per band: two pruned 3-D transforms,
    2*[5*S*log2(nz) + 5*nx_act*nz*ny*log2(ny) + 5*N*log2(nx)] with S = nst*nz sticks x z and nx_act the
    occupied x-columns (the reference's own pruning, fft.cpp:583-591)."""
    import math
    S = basis.nst * basis.nz
    return 2.0 * (5 * S * math.log2(basis.nz) + 5 * basis.nxc * basis.nz * basis.ny * math.log2(basis.ny)
                  + 5 * basis.nxyz * math.log2(basis.nx))


def local_bytes_per_band(basis, b, r):
    """Algorithmic HBM bytes of the local part of H|psi> per band:
    b*(3*npw + 4*nst*nz) + r*N (psi read, hpsi write + psi re-read for the kinetic term,
    two stick-buffer round trips, one V_eff read)."""
    npw = int(basis.npwk[0])
    S = basis.nst * basis.nz
    return b * (3 * npw + 4 * S) + r * basis.nxyz


# ---- the CPU arm: the oracle's H|psi> (numpy/scipy restatement of the reference CPU functors and
# PW_Basis_K transforms) on the host cores, band-parallel: one single-threaded process per core, each
# holding the cell's Hamiltonian; a step hands every process its share of the bands ----
_CPU_HAM = None


def _cpu_worker_init(cfg):
    global _CPU_HAM
    from threadpoolctl import threadpool_limits
    threadpool_limits(1)  # one BLAS thread per process; the oracle's FFTs run with one worker
    sys.path.insert(0, str(ROOT))
    from oracle import hamilt_ref as H
    from oracle.pw_basis_ref import PWBasisKRef
    spec_s = importlib.util.spec_from_file_location("_bench_synth", ROOT / "abacus-develop_b200" / "synth.py")
    synth = importlib.util.module_from_spec(spec_s)
    sys.modules["_bench_synth"] = synth  # dataclasses look their module up there
    spec_s.loader.exec_module(synth)
    H.FFT_WORKERS = 1
    spec = synth.config(cfg)
    cell = synth.make_cell(spec)
    b = PWBasisKRef(spec.a, cell.latvec, spec.ecut, np.zeros((1, 3)), grid=spec.grid)
    ld = int(b.npwk_max)
    ham = H.HamiltPWRef(b, 0, cell.veff(b.nx, b.ny, b.nz), cell.vkb(b.gplusk_cart(0), ld, b.omega), cell.deeq(),
                        [8], [cell.nat])
    psi = cell.psi0(b.gplusk_cart(0), spec.nbands, ld).reshape(-1)
    _CPU_HAM = (ham, psi, ld)


def _cpu_worker_hpsi(b0, nb):
    ham, psi, ld = _CPU_HAM
    ham.hpsi(psi[b0 * ld:(b0 + nb) * ld], nb, ld)
    return nb


class CpuArm:
    """The oracle's H|psi> of the 64-atom cell on `procs` host processes (spawned, so that a pool started
    after GPU work is safe).  step(nb) applies H to nb bands, split evenly over the processes."""

    TIMEOUT_S = 600  # a step that takes longer than this means a broken pool: fail instead of waiting

    def __init__(self, procs, cfg=1):
        import multiprocessing as mp
        self.procs = procs
        # maxtasksperchild=None and a bounded wait: a worker whose set-up fails would otherwise be respawned
        # forever while the parent waits
        self.pool = mp.get_context("spawn").Pool(procs, initializer=_cpu_worker_init, initargs=(cfg,))
        try:
            self.pool.starmap_async(_cpu_worker_hpsi, [(0, 1)] * procs).get(self.TIMEOUT_S)  # all set up and warm
        except BaseException:
            self.pool.terminate()
            raise

    def step(self, nb):
        share = [nb // self.procs + (1 if i < nb % self.procs else 0) for i in range(self.procs)]
        tasks, b0 = [], 0
        for n in share:
            if n:
                tasks.append((b0, n))
                b0 += n
        t0 = time.perf_counter()
        done = sum(self.pool.starmap_async(_cpu_worker_hpsi, tasks).get(self.TIMEOUT_S))
        return done, time.perf_counter() - t0

    def close(self):
        self.pool.terminate()
        self.pool.join()


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_bands_per_s(procs, budget_s=10.0, nb_step=None):
    """Bands/s of the CPU arm over steps of nb_step bands (default 2 per process, at least 16) until
    budget_s has passed; returns (bands/s, bands done, seconds, per-step seconds)."""
    arm = CpuArm(procs)
    try:
        nb = nb_step or max(16, 2 * procs)
        done, el, steps = 0, 0.0, []
        while el < budget_s:
            d, t = arm.step(nb)
            done += d
            el += t
            steps.append(t)
        return done / el, done, el, steps
    finally:
        arm.close()


def run_reference(args, ws, rank):
    """CPU reference arm: the reference's algorithm for this path on all the host cores (band-parallel)."""
    if rank != 0:
        return
    cores = host_cores()
    nb = max(16, 2 * cores)
    arm = CpuArm(cores)
    try:
        for _ in range(args.warmup):
            arm.step(nb)
        times = [arm.step(nb)[1] for _ in range(args.steps)]
    finally:
        arm.close()
    per_step = float(np.median(times))
    val = nb / per_step
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "bands/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "sample": f"{nb} of 160 bands per step"},
        "cpu_baseline": {"value": val, "unit": "bands/s", "cores": cores, "kind": "port",
                         "sample": f"{nb} bands of the 160-band block per step (median of {args.steps} steps), "
                                   f"numpy/scipy restatement of the reference CPU functors and PW_Basis_K "
                                   f"transforms, {cores} single-threaded processes, bands split evenly"},
        "e2e": {"value": val, "unit": "bands/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    ref = guarded_section(cpu_reference_davidson_8atom, load_package())
    if isinstance(ref, dict):
        ref.pop("eig", None)
        line["davidson_8atom"] = ref
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import torch
    pkg = load_package()
    P = pkg.pwdft
    lib = pkg._lib.load()
    spec = pkg.synth.config(1)
    wl = P.build_workload(spec)
    basis = wl.basis
    nb = spec.nbands
    ld = basis.npwk_max
    npw = int(basis.npwk[0])
    stream = torch.cuda.current_stream()
    h64 = P.device_hamilt(wl, P.PREC_FP64)
    h32 = P.device_hamilt(wl, P.PREC_MIXED)
    psi_h = wl.psi0_h[0][:nb].reshape(-1)
    psi = torch.from_numpy(psi_h).cuda()
    hpsi = torch.zeros_like(psi)
    psi32 = psi.to(torch.complex64)
    hpsi32 = torch.zeros_like(psi32)

    # set-up: the autotuner picks the band chunk and the plane-pass variant of each precision on this workload
    # (--tune C64:V64,C32:V32 sets them instead, e.g. to profile exactly what an earlier run chose)
    if args.tune == "auto":
        tuned64 = h64.autotune(0, psi, hpsi, nb, ld, with_variant=True)
        tuned32 = h32.autotune(0, psi32, hpsi32, nb, ld, with_variant=True)
    else:
        (c64, v64), (c32, v32) = [tuple(int(x) for x in part.split(":")) for part in args.tune.split(",")]
        h64.set_chunk(c64)
        h64.set_plane_variant(v64)
        h32.set_chunk(c32)
        h32.set_plane_variant(v32)
        tuned64, tuned32 = (c64, v64), (c32, v32)
    step64 = lambda: h64.hpsi(0, psi, hpsi, nb, ld)  # noqa: E731
    step32 = lambda: h32.hpsi(0, psi32, hpsi32, nb, ld)  # noqa: E731
    local64 = lambda: h64.hpsi_part(0, psi, hpsi, nb, ld, 1)  # noqa: E731
    local32 = lambda: h32.hpsi_part(0, psi32, hpsi32, nb, ld, 1)  # noqa: E731
    for _ in range(args.warmup):
        step64()
        step32()
    torch.cuda.synchronize()

    gpu_index = local
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES")
    if cvd:
        try:
            gpu_index = int(cvd.split(",")[local])
        except ValueError:
            pass
    barrier(ws)
    l0 = lib.b200_kernel_launches()
    with ClockSampler(gpu_index) as clk:
        ms64 = time_steps(step64, args.steps, stream)
    launches = int(lib.b200_kernel_launches() - l0)
    barrier(ws)
    ms64 = max_over_ranks(ms64, ws)
    ms32 = max_over_ranks(time_steps(step32, args.steps, stream), ws)
    ms_loc64 = time_steps(local64, args.steps, stream)
    # the same FP64 step with the projector products on cuBLAS ZGEMM instead of the int8 tensor cores
    h64.set_fp64_gemm(0)
    for _ in range(2):
        step64()
    ms64_cublas = time_steps(step64, args.steps, stream)
    h64.set_fp64_gemm(1)
    for _ in range(2):
        step64()
    ms_loc32 = time_steps(local32, args.steps, stream)

    # end to end through the public API: pinned host psi -> H|psi> -> pinned host hpsi, every step; the
    # uploads, H|psi> pieces and downloads overlap on three streams (b200_hamilt_hpsi_host)
    psi_pin = torch.from_numpy(psi_h).pin_memory()
    out_pin = torch.empty_like(psi_pin).pin_memory()

    pieces = E2E_PIECES[0]

    def e2e_step():
        h64.hpsi_host(0, psi_pin, out_pin, psi, hpsi, nb, ld, pieces=pieces)

    # set-up: the piece count with the shortest time of a few pipelined steps (the same choice on every rank)
    e2e_tune = {}
    for pieces in E2E_PIECES:
        for _ in range(2):
            e2e_step()
        e2e_tune[pieces] = max_over_ranks(time_steps(e2e_step, 5, stream), ws)
    pieces = min(e2e_tune, key=e2e_tune.get)
    for _ in range(2):
        e2e_step()
    barrier(ws)
    ms_e2e = max_over_ranks(time_steps(e2e_step, args.steps, stream), ws)
    # the link alone: the same bytes copied one way (pinned host -> device, device -> host) and both ways at
    # once on two streams, no compute; the pipelined step cannot beat the slower direction
    up_s = torch.cuda.Stream()

    def copy_up():
        psi.copy_(psi_pin, non_blocking=True)

    def copy_down():
        out_pin.copy_(hpsi, non_blocking=True)

    def copy_both():
        up_s.wait_stream(stream)
        with torch.cuda.stream(up_s):
            psi.copy_(psi_pin, non_blocking=True)
        out_pin.copy_(hpsi, non_blocking=True)
        stream.wait_stream(up_s)

    link_ms = {name: time_steps(fn, 5, stream) for name, fn in
               (("h2d", copy_up), ("d2h", copy_down), ("both", copy_both))}

    hbm_peak, _, peak_kind = peaks()
    fp_peaks = P.measure_peaks()
    b_local64 = local_bytes_per_band(basis, 16, 8) * nb
    b_local32 = local_bytes_per_band(basis, 8, 4) * nb
    f_local = local_flops_per_band(basis) * nb
    ach64 = b_local64 / (ms_loc64 * 1e-3) / 1e9
    ach32 = b_local32 / (ms_loc32 * 1e-3) / 1e9
    # the roofline time of the pass: the slower of its bytes at the HBM peak and its flops at the CUDA-core
    # peak of its precision (both measured); frac = that time / the measured time
    t_roof64 = max(b_local64 / (hbm_peak * 1e9), f_local / (fp_peaks["fp64_tflops"] * 1e12))
    t_roof32 = max(b_local32 / (hbm_peak * 1e9), f_local / (fp_peaks["fp32_tflops"] * 1e12))
    nkb = wl.nkb
    nl_flops = 16.0 * npw * nkb * nb

    line = {
        "metric": METRIC,
        "value": ws * nb / (ms64 * 1e-3),
        "unit": "bands/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms64,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "parallelism": f"replicas{ws}",
                   "l2": "inputs larger than L2 (psi+hpsi+projectors ~690 MB), no flush",
                   "autotuned_chunk_variant": {"fp64": list(tuned64), "mixed": list(tuned32)}},
        "mixed": {"value": ws * nb / (ms32 * 1e-3), "unit": "bands/s", "ms_per_step": ms32,
                  "dtype": "f32 FFT + f32 projector GEMM"},
        "roofline": {"kernel": "fused local H|psi> FP64 (z pass, plane pass, z pass per band chunk)",
                     "bound": "hbm", "achieved": ach64, "peak": hbm_peak, "unit": "GB/s",
                     "frac": ach64 / hbm_peak, "peak_kind": peak_kind,
                     "traffic": NCU_TRAFFIC_LOCAL_FP64,
                     "traffic_note": "DRAM bytes of one 160-band local pass, ncu without cache flush; "
                                     "achieved and algorithmic_bytes are per the same pass",
                     "algorithmic_bytes": b_local64, "algorithmic_flops": f_local, "ms": ms_loc64,
                     "t_roof_ms": t_roof64 * 1e3, "frac_of_t_roof": t_roof64 / (ms_loc64 * 1e-3),
                     "compute_peaks_measured": fp_peaks,
                     "mixed": {"achieved": ach32, "frac": ach32 / hbm_peak, "ms": ms_loc32,
                               "algorithmic_bytes": b_local32, "t_roof_ms": t_roof32 * 1e3,
                               "frac_of_t_roof": t_roof32 / (ms_loc32 * 1e-3)}},
        "nonlocal": {"flops": nl_flops, "ms_fp64": ms64 - ms_loc64,
                     "tflops_fp64": nl_flops / ((ms64 - ms_loc64) * 1e-3) / 1e12,
                     "path": "int8 tensor cores, exact modular emulation of the FP64 products (16 moduli)",
                     "ms_fp64_cublas": ms64_cublas - ms_loc64,
                     "bands_s_with_cublas": ws * nb / (ms64_cublas * 1e-3)},
        "e2e": {"value": ws * nb / (ms_e2e * 1e-3), "unit": "bands/s",
                "h2d_bytes_per_step": psi.numel() * 16, "d2h_bytes_per_step": hpsi.numel() * 16,
                "pieces": pieces, "ms_by_pieces": {str(k): round(v, 3) for k, v in e2e_tune.items()},
                "link_ms": {k: round(v, 3) for k, v in link_ms.items()},
                "link_gbs": {k: round(psi.numel() * 16 / (v * 1e-3) / 1e9 * (2 if k == "both" else 1), 1)
                             for k, v in link_ms.items()}},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }

    line["psi_to_rho"] = rho_bench(P, wl, psi, args.steps, stream)
    line["tc_gemm"] = gemm_bench(P)
    line["fp64_gemm"] = guarded_section(gemm64_bench, pkg, fp_peaks)
    if not args.skip_david:
        line["davidson"] = davidson_bench(P, wl, h64)
        line["dav_subspace"] = dav_subspace_bench(pkg, P, wl, h64, rank == 0 and ws == 1 and not args.skip_cpu)
        line["bpcg"] = bpcg_bench(pkg, P, wl, h64, rank == 0 and ws == 1 and not args.skip_cpu)
    del h32, psi32, hpsi32
    if not args.skip_216:
        del h64, psi, hpsi
        torch.cuda.empty_cache()
        line["davidson_216"] = davidson_216(pkg)
        torch.cuda.empty_cache()
    if not args.skip_kbatch:
        line["kbatch"] = kbatch_bench(pkg, args.steps)
        torch.cuda.empty_cache()
    if not args.skip_serve:
        line["serving"] = serving_bench(pkg)
        torch.cuda.empty_cache()

    if rank == 0 and ws == 1 and not args.skip_cpu:
        line["davidson_8atom"] = guarded_section(davidson_8atom, pkg)
        cores = host_cores()
        bps, done, el, _ = cpu_bands_per_s(cores, budget_s=args.cpu_budget)
        bps1, done1, el1, _ = cpu_bands_per_s(1, budget_s=args.cpu_budget / 2, nb_step=4)
        line["cpu_baseline"] = {"value": bps, "unit": "bands/s", "cores": cores, "kind": "port",
                                "sample": f"{done} bands of the 160-band block in {el:.1f} s on {cores} single-threaded "
                                          f"processes (bands split evenly), numpy restatement of the reference CPU "
                                          f"functors + PW_Basis_K transforms",
                                "one_core": {"value": bps1, "sample": f"{done1} bands in {el1:.1f} s, 1 process"}}
    line["summary"] = summary_of(line)
    if rank == 0:
        print(json.dumps(line), flush=True)


def _r(x, nd=3):
    """A number rounded for the compact summary (None stays None)."""
    if x is None:
        return None
    return float(f"{x:.{nd}g}")


def summary_of(line):
    """The figures the headline metric names, compact, as the line's last key (a reader that keeps only the
    end of the output still sees them): FP64 / mixed H|psi>, the roofline fraction, the Davidson solves
    (median times, speed-ups, errors against the oracle), serving latency."""
    out = {"hpsi_fp64_bands_s": _r(line.get("value"), 4), "hpsi_mixed_bands_s": _r(line.get("mixed", {}).get("value"), 4),
           "e2e_bands_s": _r(line.get("e2e", {}).get("value"), 4),
           "local_frac": _r(line.get("roofline", {}).get("frac")),
           "local_frac_mixed": _r(line.get("roofline", {}).get("mixed", {}).get("frac"))}
    nl = line.get("nonlocal") or {}
    if "ms_fp64_cublas" in nl:
        out["nonlocal_ms_int8_vs_cublas"] = [_r(nl.get("ms_fp64")), _r(nl.get("ms_fp64_cublas"))]
    for key in ("davidson", "davidson_216"):
        d = line.get(key)
        if isinstance(d, dict) and "fp64_s" in d:
            out[key] = {k: _r(d.get(k)) for k in ("fp64_s", "mixed_s", "speedup", "fp64_to_1e-8_s", "mixed_to_1e-8_s",
                                                   "speedup_to_1e-8", "fp64_err_ry", "mixed_err_ry")}
            out[key]["err_vs"] = d.get("err_vs")
            if "fp64_int8_s" in d:
                out[key].update({k: _r(d.get(k)) for k in ("fp64_int8_to_1e-8_s", "speedup_to_1e-8_vs_fp64_int8")})
    sv = line.get("serving")
    if isinstance(sv, dict):
        def lat(x):
            out = {"rps": _r(x.get("throughput_rps")), "p50_ms": _r(x.get("p50_ms")), "p99_ms": _r(x.get("p99_ms")),
                   "p99_over_p50": _r(x.get("p99_ms") / x["p50_ms"]) if x.get("p50_ms") else None}
            if x.get("n_shed"):
                out["shed"] = x["n_shed"]
            pc = x.get("per_cell") or {}
            ratios = [c["p99_ms"] / c["p50_ms"] for c in pc.values() if c.get("p50_ms")]
            if ratios:
                out["worst_cell_p99_over_p50"] = _r(max(ratios))
            return out
        out["serving"] = {k: lat(v) for k, v in sv.items() if isinstance(v, dict) and "p50_ms" in v}
    cb = line.get("cpu_baseline")
    if isinstance(cb, dict):
        out["cpu_bands_s"] = _r(cb.get("value"))
        out["cpu_cores"] = cb.get("cores")
    return out


def guarded_section(fn, *args):
    """A section beside the headline whose failure (e.g. the compiled CPU reference missing or unloadable on
    this host) is reported in its own entry instead of losing the whole line."""
    try:
        return fn(*args)
    except Exception as exc:  # noqa: BLE001
        return {"error": f"{type(exc).__name__}: {exc}"[:300]}


def rho_bench(P, wl, psi, steps, stream):
    """psiToRho's band loop on the 64-atom cell (160 bands, FP64): bands/s and bytes moved per band by the
    drop-in transform path (sphere read, three full-box sweeps of the transform, rho read + write)."""
    import torch
    b = wl.basis
    nb, ld = wl.spec.nbands, b.npwk_max
    N = b.nx * b.ny * b.nz
    rho = torch.zeros(N, dtype=torch.float64, device="cuda")
    w1 = np.full(nb, 2.0 / b.omega)
    step = lambda: b.psi_to_rho(0, psi, nb, ld, w1, rho)  # noqa: E731
    for _ in range(2):
        step()
    ms = time_steps(step, max(3, steps // 4), stream)
    return {"bands_per_s": nb / (ms * 1e-3), "ms_per_160_bands": ms,
            "path": "register transforms: inverse z pass per band chunk, then per z plane inverse y and x transforms with w|psi|^2 summed in registers, partial planes reduced once (96^3 grid; other grids: recip_to_real per band + elecstate_pw_op, the reference's loop)"}


def cpu_reference_davidson_8atom(pkg):
    """The reference's own CPU DiagoDavid (compiled from its sources, oracle/_ref) on the 8-atom cell
    (32 bands, npw 2945, thr 1e-9), H|psi> by the oracle port on all host cores.  None if not built."""
    sys.path.insert(0, str(ROOT))
    from oracle import hamilt_ref as H
    from oracle import ref_david
    from oracle.pw_basis_ref import PWBasisKRef
    if not ref_david.available():
        return None
    cores = os.cpu_count() or 1
    H.FFT_WORKERS = cores
    spec = pkg.synth.config(0)
    cell = pkg.synth.make_cell(spec)
    b = PWBasisKRef(spec.a, cell.latvec, spec.ecut, np.zeros((1, 3)))
    ld = int(b.npwk_max)
    ham = H.HamiltPWRef(b, 0, cell.veff(b.nx, b.ny, b.nz), cell.vkb(b.gplusk_cart(0), ld, b.omega), cell.deeq(), [8],
                        [cell.nat])
    psi = cell.psi0(b.gplusk_cart(0), spec.nbands, ld).reshape(-1).copy()
    e = np.zeros(spec.nbands)
    t0 = time.perf_counter()
    it = ref_david.diag(lambda x, nv, dim, i0, i1: ham.hpsi(x[i0:i1 + 1].reshape(-1), i1 - i0 + 1, dim)
                        .reshape(i1 - i0 + 1, dim), H.precondition(b, 0), spec.nbands, ld, 4, ld, psi, e, 1e-9, 200)
    return {"seconds": time.perf_counter() - t0, "iters": it, "eig": e, "cores": cores,
            "kind": "reference", "what": "DiagoDavid<complex<double>, CPU> compiled from the reference sources "
                                        "(diago_david.cpp, math_kernel_op.cpp, dngvd_op.cpp; scipy OpenBLAS), "
                                        "H|psi> by the numpy port of the reference functors"}


def davidson_8atom(pkg):
    """8-atom cell (a = 10.26 bohr, ecut 30 Ry, 36^3, npw 2945, 32 bands, thr 1e-9): GPU FP64 and mixed solves
    next to the reference's CPU DiagoDavid on the same inputs."""
    import torch
    P = pkg.pwdft
    spec = pkg.synth.config(0)
    wl = P.build_workload(spec)
    h = P.device_hamilt(wl, P.PREC_FP64)
    ld, nb = wl.basis.npwk_max, spec.nbands
    pc = P.precondition_d(wl.basis, 0)
    out = {"workload": "8-atom diamond a=10.26 bohr, ecut 30 Ry, 36^3 grid, npw 2945, 32 bands, Gamma, thr 1e-9"}
    for name, prec in (("gpu_fp64", P.PREC_FP64), ("gpu_mixed", P.PREC_MIXED)):
        runs = []
        for _ in range(4):  # the first run warms the kernels and handles; the median of the other three
            dav = P.DiagoDavid(pc, nb, ld, 4, prec)
            x = torch.from_numpy(wl.psi0_h[0].reshape(-1).copy()).cuda()
            e = np.zeros(nb)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            it = dav.diag_hamilt(h, 0, ld, x, e, 1e-9, 200)
            torch.cuda.synchronize()
            runs.append(time.perf_counter() - t0)
        out[name + "_s"] = float(np.median(runs[1:]))
        out[name + "_runs_s"] = runs[1:]
        out[name + "_iters"] = it
        out[name + "_eig"] = e
    ref = cpu_reference_davidson_8atom(pkg)
    if ref is not None:
        out["cpu_reference_s"] = ref["seconds"]
        out["cpu_reference_iters"] = ref["iters"]
        out["cpu_reference_cores"] = ref["cores"]
        out["cpu_reference"] = ref["what"]
        out["max_abs_diff_fp64_vs_reference_ry"] = float(np.max(np.abs(out["gpu_fp64_eig"] - ref["eig"])))
        out["max_abs_diff_mixed_vs_reference_ry"] = float(np.max(np.abs(out["gpu_mixed_eig"] - ref["eig"])))
        out["gpu_fp64_speedup_vs_cpu_reference"] = ref["seconds"] / out["gpu_fp64_s"]
    out.pop("gpu_fp64_eig")
    out.pop("gpu_mixed_eig")
    return out


def settle_time(trace, ref, tol=1e-8):
    """Seconds until the Ritz values come within tol of ref and stay there (None if they never do)."""
    t, _, e = trace
    if len(t) == 0:
        return None
    ok = np.max(np.abs(e - ref[None, :]), axis=1) < tol
    if not ok[-1]:
        return None
    i = len(ok) - 1
    while i > 0 and ok[i - 1]:
        i -= 1
    return float(t[i])


def residual_norms(P, h, x, e, nb, ld):
    """|H x_m - e_m x_m| of returned vectors through the FP64 H|psi> (which the tests pin to the oracle at
    1e-12 on this cell): for orthonormal x_m each e_m is within that norm of an eigenvalue of H."""
    import torch
    hx = torch.zeros_like(x)
    h.hpsi(0, x, hx, nb, ld)
    X = x.view(nb, ld)
    r = hx.view(nb, ld) - torch.from_numpy(e).to(x.device)[:, None] * X
    norms = torch.linalg.vector_norm(r, dim=1).cpu().numpy()
    ortho = (X.conj() @ X.T - torch.eye(nb, dtype=x.dtype, device=x.device)).abs().max().item()
    del hx, r
    return float(norms.max()), ortho


def solve_pair(P, h, pc, nb, ld, psi0_h, thr_ref=1e-11, thr=1e-9, repeats=3, e_oracle=None, oracle_what=None,
               int8_repeats=0):
    """FP64 and mixed solves to thr, alternating, `repeats` each, with per-iteration eigenvalue traces.
    The reference eigenvalues are the oracle's (e_oracle, a fixture) when given, else an FP64 device solve
    to thr_ref; each arm reports the median wall time and time to 1e-8 Ry over its repeats (with min / max),
    its largest eigenvalue error against the reference, and the residual norms of its returned vectors
    through the pinned FP64 H|psi>.  int8_repeats > 0 adds an FP64 arm whose subspace products run on the
    int8 tensor-core emulation where it is faster (b200_david_set_fp64_gemm mode 2; one solver reused, its
    workspaces grown by an untimed solve first)."""
    import torch

    def solve(prec, t_thr, keep=False):
        dav = P.DiagoDavid(pc, nb, ld, 4, prec)
        dav.set_trace(True)
        x = torch.from_numpy(psi0_h.copy()).cuda()
        e = np.zeros(nb)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dav.diag_hamilt(h, 0, ld, x, e, t_thr, 300)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        res = residual_norms(P, h, x, e, nb, ld) if keep else None
        out = (wall, e, dav.stats(), dav.trace(), res)
        del dav, x
        torch.cuda.empty_cache()
        return out

    # warm-up, one untimed solve of each arm at the timed threshold: the first use of every kernel (modules load
    # lazily), handle and workspace shape happens here (a first mixed solve took up to 1.5x its repeats)
    solve(P.PREC_MIXED, thr)
    if e_oracle is not None:
        solve(P.PREC_FP64, thr)
        e_ref, st_ref = np.asarray(e_oracle, dtype=np.float64), None
        err_vs = oracle_what
    else:
        _, e_ref, st_ref, _, _ = solve(P.PREC_FP64, thr_ref)
        err_vs = f"FP64 device solve to thr {thr_ref}"
    runs64, runsmx = [], []
    for i in range(repeats):
        runs64.append(solve(P.PREC_FP64, thr, keep=(i == 0)))
        runsmx.append(solve(P.PREC_MIXED, thr, keep=(i == 0)))

    def arm(runs):
        walls = [r[0] for r in runs]
        settles = [settle_time(r[3], e_ref) for r in runs]
        ok = [t for t in settles if t is not None]
        return {"median_s": float(np.median(walls)), "runs_s": walls,
                "to_1e-8_s": float(np.median(ok)) if len(ok) == len(runs) else None, "to_1e-8_runs_s": settles,
                "err_ry": float(max(np.max(np.abs(r[1] - e_ref)) for r in runs)),
                "max_residual": runs[0][4][0], "orthonormality": runs[0][4][1], "stats": runs[0][2]}

    a64, amx = arm(runs64), arm(runsmx)
    extra = {}
    if int8_repeats > 0:
        dav = P.DiagoDavid(pc, nb, ld, 4, P.PREC_FP64)
        dav.set_fp64_gemm(2)
        x = torch.from_numpy(psi0_h.copy()).cuda()
        dav.diag_hamilt(h, 0, ld, x, np.zeros(nb), 1e-4, 300)
        runs8 = []
        for _ in range(int8_repeats):
            dav.set_trace(True)
            x.copy_(torch.from_numpy(psi0_h))
            e = np.zeros(nb)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            dav.diag_hamilt(h, 0, ld, x, e, thr, 300)
            torch.cuda.synchronize()
            runs8.append((time.perf_counter() - t0, e, dav.stats(), dav.trace(), (None, None)))
        del dav, x
        torch.cuda.empty_cache()
        a8 = arm(runs8)
        extra = {"fp64_int8_s": a8["median_s"], "fp64_int8_runs_s": a8["runs_s"],
                 "fp64_int8_to_1e-8_s": a8["to_1e-8_s"], "fp64_int8_err_ry": a8["err_ry"],
                 "speedup_to_1e-8_vs_fp64_int8": (a8["to_1e-8_s"] / amx["to_1e-8_s"])
                 if (a8["to_1e-8_s"] and amx["to_1e-8_s"]) else None,
                 "fp64_int8": "the FP64 solve with its subspace products on the int8 tensor-core emulation of the "
                              "FP64 products where that is faster (cuBLAS ZGEMM elsewhere)"}
    out = {"fp64_s": a64["median_s"], "mixed_s": amx["median_s"], "speedup": a64["median_s"] / amx["median_s"],
           "fp64_runs_s": a64["runs_s"], "mixed_runs_s": amx["runs_s"],
           "fp64_to_1e-8_s": a64["to_1e-8_s"], "mixed_to_1e-8_s": amx["to_1e-8_s"],
           "fp64_to_1e-8_runs_s": a64["to_1e-8_runs_s"], "mixed_to_1e-8_runs_s": amx["to_1e-8_runs_s"],
           "speedup_to_1e-8": (a64["to_1e-8_s"] / amx["to_1e-8_s"]) if (a64["to_1e-8_s"] and amx["to_1e-8_s"]) else None,
           "fp64_err_ry": a64["err_ry"], "mixed_err_ry": amx["err_ry"], "err_vs": err_vs,
           "fp64_max_residual": a64["max_residual"], "mixed_max_residual": amx["max_residual"],
           "fp64_orthonormality": a64["orthonormality"], "mixed_orthonormality": amx["orthonormality"],
           "fp64_iters": a64["stats"][1], "mixed_iters_fp32": amx["stats"][0], "mixed_iters_fp64": amx["stats"][1],
           "fp64_hpsi_bands": a64["stats"][2], "mixed_hpsi_bands": amx["stats"][2],
           "ref_iters": st_ref[1] if st_ref else None, "thr": thr, "repeats": repeats,
           "timing": "medians over alternating repeats (runs listed); to_1e-8: time after which every Ritz value "
                     "stays within 1e-8 Ry of the reference eigenvalues, from the per-iteration trace; residuals "
                     "|Hx - ex| of the first repeat's vectors through the FP64 H|psi>", **extra}
    return out


EIG_FIXTURE_64 = ROOT / "tests" / "golden" / "eig_diamond64.npz"
EIG_FIXTURE_216 = ROOT / "tests" / "golden" / "eig_diamond216.npz"


def davidson_bench(P, wl, h64):
    """64-atom cell: errors and time to 1e-8 Ry against the oracle's eigenvalues (tests/golden/eig_diamond64.npz:
    the reference's DiagoDavid on the oracle's H|psi> to thr 1e-11)."""
    nb = wl.spec.nbands
    ld = wl.basis.npwk_max
    pc = P.precondition_d(wl.basis, 0)
    fx = np.load(EIG_FIXTURE_64)
    out = solve_pair(P, h64, pc, nb, ld, wl.psi0_h[0][:nb].reshape(-1), e_oracle=fx["eig"],
                     oracle_what=f"oracle fixture eig_diamond64.npz ({fx['solver']}, thr {float(fx['thr'])})")
    out["workload"] = WORKLOAD_NAME
    return out


def dav_subspace_bench(pkg, P, wl, h64, with_cpu):
    """Diago_DavSubspace (FP64) on the 64-atom cell next to DiagoDavid FP64 from the same orthonormal start
    (160 bands, david_ndim 4, thr 1e-9, NSCF exit rule), and on the 8-atom cell next to the reference's own
    CPU Diago_DavSubspace (compiled from its sources, oracle/_ref) on the same inputs."""
    import torch
    nb, ld = wl.spec.nbands, wl.basis.npwk_max
    npw = int(wl.basis.npwk[0])
    q, _ = np.linalg.qr(wl.psi0_h[0][:nb, :npw].T)
    psi0 = np.zeros((nb, ld), complex)
    psi0[:, :npw] = q.T
    pc_ds = P.precondition_dav_subspace_d(wl.basis, 0)
    pc_dav = P.precondition_d(wl.basis, 0)

    def run_ds():
        ds = P.DiagoDavSubspace(pc_ds, nb, npw, 4, 1e-9, 300)
        x = torch.from_numpy(psi0.reshape(-1).copy()).cuda()
        e = np.zeros(nb)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it = ds.diag_hamilt(h64, 0, x, ld, e)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, it, e, ds.stats()

    def run_dav():
        dav = P.DiagoDavid(pc_dav, nb, ld, 4, P.PREC_FP64)
        x = torch.from_numpy(psi0.reshape(-1).copy()).cuda()
        e = np.zeros(nb)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it = dav.diag_hamilt(h64, 0, ld, x, e, 1e-9, 300)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, it, e, dav.stats()

    run_ds()  # warm-up
    ds_runs = [run_ds() for _ in range(3)]
    dav_runs = [run_dav() for _ in range(3)]
    ds, dv = ds_runs[0], dav_runs[0]
    out = {"workload": WORKLOAD_NAME + ", thr 1e-9", "dav_subspace_s": float(np.median([r[0] for r in ds_runs])),
           "dav_subspace_runs_s": [r[0] for r in ds_runs], "dav_subspace_iters": ds[1],
           "dav_subspace_hpsi_bands": ds[3][1], "david_fp64_s": float(np.median([r[0] for r in dav_runs])),
           "david_fp64_runs_s": [r[0] for r in dav_runs], "david_fp64_iters": dv[1],
           "david_fp64_hpsi_bands": dv[3][2], "max_abs_diff_vs_david_ry": float(np.max(np.abs(ds[2] - dv[2])))}
    if with_cpu:
        out["8atom"] = guarded_section(dav_subspace_8atom, pkg)
    return out


def dav_subspace_8atom(pkg):
    """8-atom cell (npw 2945, 32 bands, thr 1e-9): the device solver against the reference's CPU
    Diago_DavSubspace on the same orthonormal start, H|psi> of the CPU arm by the numpy port on all cores."""
    import torch
    sys.path.insert(0, str(ROOT))
    from oracle import hamilt_ref as H
    from oracle import ref_david
    from oracle.pw_basis_ref import PWBasisKRef
    P = pkg.pwdft
    spec = pkg.synth.config(0)
    wl = P.build_workload(spec)
    h = P.device_hamilt(wl, P.PREC_FP64)
    ld, nb = wl.basis.npwk_max, spec.nbands
    npw = int(wl.basis.npwk[0])
    q, _ = np.linalg.qr(wl.psi0_h[0][:nb, :npw].T)
    psi0 = np.zeros((nb, ld), complex)
    psi0[:, :npw] = q.T
    pc = P.precondition_dav_subspace_d(wl.basis, 0)
    runs = []
    for _ in range(4):  # the first run warms the kernels and handles; the median of the other three
        ds = P.DiagoDavSubspace(pc, nb, npw, 4, 1e-9, 200)
        x = torch.from_numpy(psi0.reshape(-1).copy()).cuda()
        e = np.zeros(nb)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it = ds.diag_hamilt(h, 0, x, ld, e)
        torch.cuda.synchronize()
        runs.append(time.perf_counter() - t0)
    best = float(np.median(runs[1:]))
    out = {"gpu_s": best, "gpu_runs_s": runs[1:], "gpu_iters": it}
    if not ref_david.available():
        return out
    H.FFT_WORKERS = os.cpu_count() or 1
    b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, np.zeros((1, 3)))
    ham = H.HamiltPWRef(b, 0, wl.veff_h, wl.vkb_h[0][:, :ld], wl.deeq_h, [8], [wl.cell.nat])

    def hp(x, nv, d, i0, i1):
        m = i1 - i0 + 1
        y = np.zeros((m, ld), complex)
        y[:, :npw] = x[i0:i1 + 1, :npw]
        return ham.hpsi(y.reshape(-1), m, ld).reshape(m, ld)[:, :npw]

    e_r, p_r = np.zeros(nb), psi0.copy()
    t0 = time.perf_counter()
    it_r = ref_david.dav_subspace(hp, H.precondition_dav_subspace(b, 0), nb, npw, 4, ld, p_r, e_r, 1e-9, 200)
    cpu_s = time.perf_counter() - t0
    out.update({"cpu_reference_s": cpu_s, "cpu_reference_iters": it_r,
                "cpu_reference_cores": H.FFT_WORKERS, "max_abs_diff_vs_reference_ry": float(np.max(np.abs(e - e_r))),
                "gpu_speedup_vs_cpu_reference": cpu_s / best,
                "cpu_reference": "Diago_DavSubspace<complex<double>, CPU> compiled from the reference sources "
                                 "(diago_dav_subspace.cpp, dngvd_op.cpp; scipy OpenBLAS), H|psi> by the numpy port "
                                 "of the reference functors"})
    return out


def bpcg_bench(pkg, P, wl, h64, with_cpu):
    """DiagoBPCG (FP64) on the 64-atom cell from an orthonormal start: a first-SCF-step call (24 iterations,
    Rayleigh-Ritz every 4) and a later-step call (4 iterations) after it; on the 8-atom cell a later-step
    call next to the reference's own CPU DiagoBPCG (compiled from its sources) on the same start."""
    import torch
    nb, ld = wl.spec.nbands, wl.basis.npwk_max
    npw = int(wl.basis.npwk[0])
    q, _ = np.linalg.qr(wl.psi0_h[0][:nb, :npw].T)
    psi0 = np.zeros((nb, ld), complex)
    psi0[:, :npw] = q.T
    pc = P.precondition_d(wl.basis, 0)

    def run(x, scf_iter, bp):
        e = np.zeros(nb)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it = bp.diag_hamilt(h64, 0, x, e, scf_iter)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, it, e, bp.stats()

    pairs = []
    for _ in range(4):  # the first repeat warms every kernel and handle; medians of the other three
        bp = P.DiagoBPCG(pc, nb, ld)
        x = torch.from_numpy(psi0.reshape(-1).copy()).cuda()
        first = run(x, 1, bp)
        later = run(x, 2, bp)
        pairs.append((first, later))
    pairs = pairs[1:]
    first, later = pairs[0]
    t_first = float(np.median([p[0][0] for p in pairs]))
    t_later = float(np.median([p[1][0] for p in pairs]))
    out = {"workload": WORKLOAD_NAME, "first_step_s": t_first, "first_step_runs_s": [p[0][0] for p in pairs],
           "first_step_iters": first[1], "first_step_max_residual": first[3][0], "first_step_hpsi_bands": first[3][1],
           "later_step_s": t_later, "later_step_runs_s": [p[1][0] for p in pairs], "later_step_iters": later[1],
           "later_step_max_residual": later[3][0], "ms_per_iteration_later_step": 1e3 * t_later / max(1, later[1])}
    if with_cpu:
        out["8atom"] = guarded_section(bpcg_8atom, pkg)
    return out


def bpcg_8atom(pkg):
    """8-atom cell (npw 2945, 32 bands): one later-SCF-step DiagoBPCG call (4 iterations) on the device and by
    the reference's CPU DiagoBPCG from the same orthonormal start, H|psi> of the CPU arm by the numpy port on
    all cores."""
    import torch
    sys.path.insert(0, str(ROOT))
    from oracle import hamilt_ref as H
    from oracle import ref_david
    from oracle.pw_basis_ref import PWBasisKRef
    P = pkg.pwdft
    spec = pkg.synth.config(0)
    wl = P.build_workload(spec)
    h = P.device_hamilt(wl, P.PREC_FP64)
    ld, nb = wl.basis.npwk_max, spec.nbands
    npw = int(wl.basis.npwk[0])
    q, _ = np.linalg.qr(wl.psi0_h[0][:nb, :npw].T)
    psi0 = np.ascontiguousarray(q.T)
    pc = P.precondition_d(wl.basis, 0)
    runs = []
    for _ in range(4):  # the first run warms the kernels and handles; the median of the other three
        bp = P.DiagoBPCG(pc, nb, npw)
        x = torch.from_numpy(psi0.reshape(-1).copy()).cuda()
        e = np.zeros(nb)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it = bp.diag_hamilt(h, 0, x, e, 2)
        torch.cuda.synchronize()
        runs.append(time.perf_counter() - t0)
    best = float(np.median(runs[1:]))
    out = {"gpu_s": best, "gpu_runs_s": runs[1:], "gpu_iters": it}
    if not ref_david.available() or ld != npw:
        return out
    H.FFT_WORKERS = os.cpu_count() or 1
    b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, np.zeros((1, 3)))
    ham = H.HamiltPWRef(b, 0, wl.veff_h, wl.vkb_h[0][:, :ld], wl.deeq_h, [8], [wl.cell.nat])
    e_r, p_r = np.zeros(nb), psi0.copy()
    t0 = time.perf_counter()
    ref_david.bpcg(lambda x, nv, d, i0, i1: ham.hpsi(x[i0:i1 + 1].reshape(-1), i1 - i0 + 1, d).reshape(i1 - i0 + 1, d),
                   H.precondition(b, 0), nb, npw, p_r, e_r, 2, 1)
    cpu_s = time.perf_counter() - t0
    out.update({"cpu_reference_s": cpu_s, "cpu_reference_cores": H.FFT_WORKERS,
                "max_abs_diff_vs_reference_ry": float(np.max(np.abs(e - e_r))),
                "gpu_speedup_vs_cpu_reference": cpu_s / best,
                "cpu_reference": "DiagoBPCG<complex<double>, CPU> compiled from the reference sources with its "
                                 "container tensor library (diago_bpcg.cpp, math_kernel_op.cpp, ATen einsum/"
                                 "lapack; scipy OpenBLAS), H|psi> by the numpy port of the reference functors"})
    return out


def device_cell(pkg, spec, kpts=None):
    """A cell's Hamiltonian with V_eff, D and the projectors built on the device by getvnl (same synthetic
    generators as the host path, through a radial table of step 0.01 bohr^-1)."""
    import torch
    P, S = pkg.pwdft, pkg.synth
    cell = S.make_cell(spec)
    k = np.zeros((1, 3)) if kpts is None else kpts
    basis = P.PWBasisK(spec.a, cell.latvec, spec.ecut, k, grid=spec.grid)
    h = P.HamiltPW(basis, P.PREC_FP64)
    veff = torch.from_numpy(cell.veff(basis.nx, basis.ny, basis.nz)).cuda()
    h.set_veff(veff)
    deeq = torch.from_numpy(cell.deeq()).cuda()
    h.set_deeq([cell.nat], [S.NH], deeq)
    h.set_projectors(cell.projector_tables(basis.omega, spec.ecut), cell.tau / spec.a)
    for ik in range(basis.nks):
        h.build_vkb(ik)
    torch.cuda.synchronize()
    h._keep += [veff, deeq]
    return cell, basis, h


def davidson_216(pkg):
    """216-atom cell (a = 30.78 bohr, ecut 40 Ry, 128^3 grid, npw 124 289, 480 bands, 1728 projectors):
    FP64 vs mixed Davidson, time to 1e-8 Ry."""
    P = pkg.pwdft
    spec = pkg.synth.config(4)
    t0 = time.perf_counter()
    cell, basis, h = device_cell(pkg, spec)
    ld = basis.npwk_max
    psi0 = cell.psi0(basis.gplusk_cart(0), spec.nbands, ld).reshape(-1)
    # the autotuner picks the local pass's band chunk and plane variant on this cell: the chunk of the FP64
    # handle (used by both precisions of its solves) and the FP64 variant on it, the FP32 variant on an FP32
    # handle of the same basis (plane variants are kept per basis and precision)
    import torch
    x = torch.from_numpy(psi0).cuda()
    hx = torch.zeros_like(x)
    tuned64 = h.autotune(0, x, hx, spec.nbands, ld, with_variant=True)
    h32 = P.HamiltPW(basis, P.PREC_MIXED)
    h32.set_veff(h._keep[-2])
    x32, hx32 = x.to(torch.complex64), hx.to(torch.complex64)
    tuned32 = h32.autotune(0, x32, hx32, spec.nbands, ld, with_variant=True)
    del x, hx, x32, hx32, h32
    torch.cuda.empty_cache()
    setup = time.perf_counter() - t0
    pc = P.precondition_d(basis, 0)
    # five alternating repeats, medians reported with every run listed: a solve synchronises with the host
    # every iteration, and a stall of the shared host cores shows up in single repeats.  The errors are
    # against the oracle's eigenvalues (tests/golden/eig_diamond216.npz: the reference's DiagoDavid on the
    # oracle's H|psi>) where that fixture exists, else against an FP64 device solve to 1e-10; the residual norms through the FP64 H|psi> (pinned to the oracle at
    # 1e-12 on this cell by the tests) bound every returned eigenvalue's distance to the spectrum
    if EIG_FIXTURE_216.exists():
        fx = np.load(EIG_FIXTURE_216)
        out = solve_pair(P, h, pc, spec.nbands, ld, psi0, repeats=5, e_oracle=fx["eig"], int8_repeats=3,
                         oracle_what=f"oracle fixture eig_diamond216.npz ({fx['solver']}, thr {float(fx['thr'])})")
    else:
        out = solve_pair(P, h, pc, spec.nbands, ld, psi0, thr_ref=1e-10, repeats=5, int8_repeats=3)
    out["workload"] = (f"216-atom diamond supercell a=30.78 bohr, ecut 40 Ry, 128^3 grid, npw {int(basis.npwk[0])}, "
                       f"480 bands, 1728 projectors (device getvnl), Gamma")
    out["setup_s"] = setup
    out["autotuned_chunk_variant"] = {"fp64": list(tuned64), "fp32_variant": tuned32[1]}
    return out


# complex64 3xTF32 tensor-core GEMM shapes: the subspace products of the 216-atom Davidson (dim 124289,
# nband 480, subspace up to 1920) and the projector products of the 64-atom H|psi> (512 projectors, npw
# 51627, 160 bands)
GEMM_SHAPES = [("N", 124289, 480, 1300), ("N", 124289, 480, 480), ("C", 480, 1920, 124289),
               ("C", 1920, 480, 124289), ("C", 480, 480, 124289), ("N", 51627, 160, 512), ("C", 512, 160, 51627)]


def gemm_bench(P, reps=5):
    """tc_cgemm (gemm_op<complex<float>, GPU> on tcgen05) on the shapes above: CUDA-event time per call and
    complex-equivalent TFLOP/s (8 M N K flop per call)."""
    import torch
    out = []
    for ta, M, N, K in GEMM_SHAPES:
        rows_a, cols_a = (M, K) if ta == "N" else (K, M)
        lda, ldb = rows_a + rows_a % 2, K + K % 2
        g = torch.Generator(device="cuda").manual_seed(7)
        a = torch.randn(cols_a, lda, dtype=torch.complex64, device="cuda", generator=g)
        b = torch.randn(N, ldb, dtype=torch.complex64, device="cuda", generator=g)
        c = torch.zeros(N, M, dtype=torch.complex64, device="cuda")
        for _ in range(3):
            P.tc_cgemm(ta, M, N, K, 1.0, a, lda, b, ldb, 0.0, c, M)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            P.tc_cgemm(ta, M, N, K, 1.0, a, lda, b, ldb, 0.0, c, M)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out.append({"op": ta, "M": M, "N": N, "K": K, "ms": ms, "tflops": 8.0 * M * N * K / (ms * 1e-3) / 1e12})
        del a, b, c
        torch.cuda.empty_cache()
    assert P.tc_cgemm_error() == 0
    return out


# FP64 complex GEMM shapes of the plain path: the 64-atom projector products and the 216-atom subspace
# products (transa, transb, M, N, K)
GEMM64_SHAPES = [("C", "N", 512, 160, 51627), ("N", "N", 51627, 160, 512), ("N", "N", 124289, 480, 480),
                 ("C", "N", 480, 1920, 124289)]


def gemm64_bench(pkg, peaks_tf, reps=5):
    """The FP64 complex GEMM of gemm_op<complex<double>, GPU> on the shapes above: cuBLAS ZGEMM through
    b200_gemm_op_f64 against the measured FP64 tensor-core peak (a complex product is four real products on
    the FP64 tensor pipe, so 8 M N K flop at the DMMA rate is its ceiling), and the int8 tensor-core
    emulation b200_zgemm_i8 (with both operands' residues built in every call)."""
    import ctypes as C
    import torch
    lib = pkg._lib.load()
    one = (C.c_double * 2)(1.0, 0.0)
    zero = (C.c_double * 2)(0.0, 0.0)
    out = []
    for ta, tb, M, N, K in GEMM64_SHAPES:
        rows_a = M if ta == "N" else K
        cols_a = K if ta == "N" else M
        a = torch.randn(cols_a, rows_a, dtype=torch.complex128, device="cuda")
        b = torch.randn(N, K, dtype=torch.complex128, device="cuda")
        c = torch.zeros(N, M, dtype=torch.complex128, device="cuda")

        def call():
            rc = lib.b200_gemm_op_f64(ta.encode(), tb.encode(), M, N, K, one, a.data_ptr(), rows_a, b.data_ptr(), K, zero,
                                      c.data_ptr(), M, None)
            assert rc == 0

        for _ in range(2):
            call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            call()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        tf = 8.0 * M * N * K / (ms * 1e-3) / 1e12

        # the same product on the int8 tensor cores (b200_zgemm_i8: residues of both operands every call)
        def call_i8():
            rc = lib.b200_zgemm_i8(ta.encode(), tb.encode(), M, N, K, one, a.data_ptr(), rows_a, b.data_ptr(), K, zero,
                                   c.data_ptr(), M, 16, None)
            assert rc == 0

        for _ in range(2):
            call_i8()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            call_i8()
        e1.record()
        torch.cuda.synchronize()
        ms8 = e0.elapsed_time(e1) / reps
        out.append({"op": ta + tb, "M": M, "N": N, "K": K, "ms": ms, "tflops": tf,
                    "frac_of_dmma_peak": tf / peaks_tf["dmma_fp64_tflops"], "int8_ms": ms8,
                    "int8_equiv_tflops": 8.0 * M * N * K / (ms8 * 1e-3) / 1e12})
        del a, b, c
        torch.cuda.empty_cache()
    return out


def kbatch_bench(pkg, steps):
    """8-atom cell, shifted 4x4x4 Monkhorst-Pack grid (64 k-points, uneven npw), 32 bands: H|psi> of all
    k-points per call (one launch per FFT pass), per-k-point calls, CUDA-graph replay; concurrent Davidson
    solves of all k-points."""
    import torch
    P = pkg.pwdft
    spec = pkg.synth.config(2)
    wl = P.build_workload(spec)
    nk, nb, ld = wl.basis.nks, spec.nbands, wl.basis.npwk_max
    iks = list(range(nk))
    res = {"workload": f"8-atom diamond a=10.26 bohr, ecut 30 Ry, 36^3 grid, 64 k-points (shifted 4x4x4 MP), "
                       f"npwk {int(min(wl.basis.npwk))}-{int(max(wl.basis.npwk))}, 32 bands"}
    stream = torch.cuda.Stream()
    for name, prec, dt in (("fp64", P.PREC_FP64, np.complex128), ("mixed", P.PREC_MIXED, np.complex64)):
        h = P.device_hamilt(wl, prec)
        psis = [torch.from_numpy(wl.psi0_h[ik][:nb].reshape(-1).astype(dt)).cuda() for ik in iks]
        outs = [torch.zeros_like(x) for x in psis]
        with torch.cuda.stream(stream):
            batch = lambda: h.hpsi_kbatch(iks, psis, outs, nb, ld, stream=stream)  # noqa: E731

            def perk():
                for ik in iks:
                    h.hpsi(ik, psis[ik], outs[ik], nb, ld, stream=stream)
            for _ in range(3):
                batch()
                perk()
            ms_b = time_steps(batch, steps, stream)
            ms_k = time_steps(perk, steps, stream)
            g = h.capture_hpsi_kbatch(iks, psis, outs, nb, ld, stream=stream)
            for _ in range(3):
                g.launch(stream)
            ms_g = time_steps(lambda: g.launch(stream), steps, stream)
        del g
        res[name] = {"batched_bands_per_s": nk * nb / (ms_b * 1e-3), "per_k_bands_per_s": nk * nb / (ms_k * 1e-3),
                     "graph_bands_per_s": nk * nb / (ms_g * 1e-3), "ms_batched": ms_b, "ms_per_k": ms_k,
                     "ms_graph": ms_g}
        del h, psis, outs
    h = P.device_hamilt(wl, P.PREC_FP64)
    pcs = [P.precondition_d(wl.basis, ik) for ik in iks]
    for name, prec in (("fp64", P.PREC_FP64), ("mixed", P.PREC_MIXED)):
        # three calls, the median reported (all listed): each call builds its 8 workers' solvers (handles,
        # buffers) and drives 8 host threads that synchronise every iteration, so calls vary with the host cores
        runs = []
        for _ in range(3):
            psis = [torch.from_numpy(wl.psi0_h[ik].reshape(-1).copy()).cuda() for ik in iks]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eig, its = h.solve_kpoints(iks, pcs, psis, ld, nb, 1e-9, 200, precision=prec, nworkers=8)
            torch.cuda.synchronize()
            runs.append(time.perf_counter() - t0)
        res[name]["solve_all_k_s"] = float(np.median(runs))
        res[name]["solve_all_k_runs_s"] = runs
        res[name]["solve_iters_mean"] = float(np.mean(its))
        if name == "fp64":
            e64 = eig
        else:
            res["mixed"]["solve_max_err_vs_fp64_ry"] = float(np.max(np.abs(eig - e64)))
    # all 64 k-points in lock-step: one batched call per phase for all k, FP64 and mixed
    for name, prec in (("fp64", P.PREC_FP64), ("mixed", P.PREC_MIXED)):
        runs = []
        for _ in range(4):
            psis = [torch.from_numpy(wl.psi0_h[ik].reshape(-1).copy()).cuda() for ik in iks]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eig_b, its_b = h.solve_kpoints_batched(iks, pcs, psis, ld, nb, 1e-9, 200, precision=prec)
            torch.cuda.synchronize()
            runs.append(time.perf_counter() - t0)
        res[name]["solve_all_k_batched_s"] = float(np.median(runs[1:]))
        res[name]["solve_all_k_batched_runs_s"] = runs[1:]
        res[name]["solve_batched_iters_max"] = int(np.max(its_b))
        res[name]["solve_batched_max_diff_vs_per_k_fp64_ry"] = float(np.max(np.abs(eig_b - e64)))
    res["solve"] = ("Davidson of all 64 k-points, thr 1e-9: 8 concurrent solves on separate streams (solve_all_k), "
                    "or all k-points in lock-step with batched calls (solve_all_k_batched; the first of 4 runs, which "
                    "makes the solver's buffers, excluded)")
    return res


def serving_bench(pkg, npath=8, nreq=200, rate=200.0):
    """Serving: Poisson arrivals of band solves on the four resident cells (2, 8, 16 and 64 atoms, 8, 32, 64
    and 160 bands, mixed precision, thr 1e-9, k uniform on an 8-point high-symmetry path per cell)."""
    S = pkg.serve
    cells = S.build_serving_cells(npath=npath)
    srv = S.Server(hbm_budget_bytes=64 << 30, nworkers=8)
    ids = [srv.add_cell(c.hamilt) for c in cells]
    for i, c in enumerate(cells):  # warm-up: creates the solver slots
        for w in range(2):
            srv.submit(ids[i], w, c.nbands, thr=1e-9)
    srv.drain()
    alone = {}
    for i, c in enumerate(cells):
        srv.submit(ids[i], 3, c.nbands, thr=1e-9)
        r = srv.drain()[0]
        alone[c.spec.name] = 1e3 * (r.t_done - r.t_admit)
    full = S.poisson_load(srv, ids, cells, rate, nreq, seed=11)
    full.pop("results")
    cap = full["throughput_rps"]
    sustained = S.poisson_load(srv, ids, cells, 0.7 * cap, max(20, int(0.7 * cap * 8)), seed=12)
    sustained.pop("results")
    # at the measured capacity (offered = capacity): the highest response ratio first, without and with
    # shedding of requests that waited past their cell's mean service time
    srv.set_policy(1, 0.0)
    at_cap_rr = S.poisson_load(srv, ids, cells, cap, max(40, int(cap * 10)), seed=13)
    at_cap_rr.pop("results")
    srv.set_policy(1, 1.0)
    at_cap_shed = S.poisson_load(srv, ids, cells, cap, max(40, int(cap * 10)), seed=13)
    at_cap_shed.pop("results")
    # the same with one express worker for the cells whose solves take under 30 ms (the 2-atom cell)
    srv.set_express(1, 0.03)
    at_cap_express = S.poisson_load(srv, ids, cells, cap, max(40, int(cap * 10)), seed=13)
    at_cap_express.pop("results")
    srv.set_express(0, 0.0)
    srv.set_policy(0, 0.0)
    st = srv.stats()
    srv.close()
    return {"offered": full, "at_70pct_capacity": sustained, "at_capacity_response_ratio": at_cap_rr,
            "at_capacity_response_ratio_shed1": at_cap_shed, "at_capacity_response_ratio_shed1_express1": at_cap_express,
            "alone_service_ms": alone,
            "pool": {"peak_bytes": st["peak_pool_bytes"], "peak_in_flight": st["peak_in_flight"],
                     "slots": st["slots_created"], "budget_bytes": 64 << 30},
            "workers": 8, "workload": "4 resident cells, 8 k-points each, mixed precision, thr 1e-9",
            "policies": "offered / at_70pct_capacity: oldest first; at_capacity_*: offered = the measured capacity, "
                        "highest response ratio first, without / with shedding past 1x the cell's mean service; "
                        "express1: one of the 8 workers reserved for cells of under 30 ms mean service"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)  # 0.38 s of FP64 H|psi>: several clock samples
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-david", action="store_true")
    ap.add_argument("--skip-216", action="store_true")
    ap.add_argument("--skip-kbatch", action="store_true")
    ap.add_argument("--skip-serve", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--tune", default="auto",
                    help="'auto' (autotune at set-up) or C64:V64,C32:V32 band chunk and plane variant per precision")
    ap.add_argument("--gemm-only", action="store_true", help="only the tensor-core GEMM shapes (for profiling)")
    ap.add_argument("--solvers-only", action="store_true",
                    help="only the Diago_DavSubspace and DiagoBPCG sections on the 64-atom cell (for profiling)")
    args = ap.parse_args()
    if args.gemm_only:
        pkg = load_package()
        print(json.dumps({"tc_gemm": gemm_bench(pkg.pwdft, reps=1)}), flush=True)
        return
    if args.solvers_only:
        pkg = load_package()
        P = pkg.pwdft
        wl = P.build_workload(pkg.synth.config(1))
        h64 = P.device_hamilt(wl, P.PREC_FP64)
        print(json.dumps({"dav_subspace": dav_subspace_bench(pkg, P, wl, h64, False),
                          "bpcg": bpcg_bench(pkg, P, wl, h64, False)}, default=float), flush=True)
        return
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), rank)
        return
    ws, rank, local = dist_setup()
    try:
        run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
