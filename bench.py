"""Benchmark: plane-wave H|psi> bands/s (FP64 and mixed) and Davidson time-to-1e-8 Ry on one B200.

Workload (default): 64-atom diamond supercell, a = 20.52 bohr, ecut 50 Ry,
96^3 FFT grid, npw = 51 627, 160 bands, 512 Kleinman-Bylander projectors,
Gamma point, seeded synthetic V_eff / projectors / D / psi (no dataset).

One step = one H|psi> (kinetic + local V_eff via the stick/plane FFT +
nonlocal projectors) on the whole 160-band block, inputs resident in HBM.
psi + hpsi + projectors (about 690 MB) exceed the 126 MB L2, so no flush is
needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

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
# dram__bytes_read.sum + dram__bytes_write.sum of the fused local H|psi> kernels for one 160-band
# application, from the ncu capture summarised in profiles/hpsi_local_diamond64.md (None until captured)
NCU_TRAFFIC_LOCAL_FP64 = None


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
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

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
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
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


def local_bytes_per_band(basis, b, r):
    """Algorithmic HBM bytes of the local part of H|psi> per band:
    b*(3*npw + 4*nst*nz) + r*N (psi read, hpsi write + psi re-read for the kinetic term,
    two stick-buffer round trips, one V_eff read)."""
    npw = int(basis.npwk[0])
    S = basis.nst * basis.nz
    return b * (3 * npw + 4 * S) + r * basis.nxyz


def cpu_port_bands_per_s(wl, budget_s=10.0, sample_bands=8, workers=1):
    """The oracle's H|psi> on the host cores over a bounded sample of bands."""
    sys.path.insert(0, str(ROOT))
    from oracle import hamilt_ref as H
    from oracle.pw_basis_ref import PWBasisKRef
    H.FFT_WORKERS = workers
    spec = wl.spec
    ref_b = PWBasisKRef(spec.a, wl.cell.latvec, spec.ecut, np.zeros((1, 3)), grid=spec.grid)
    ld = wl.basis.npwk_max
    ref = H.HamiltPWRef(ref_b, 0, wl.veff_h, wl.vkb_h[0][:, :ld], wl.deeq_h, [8], [wl.cell.nat])
    psi = wl.psi0_h[0][:sample_bands].reshape(-1)
    done = 0
    t0 = time.perf_counter()
    while True:
        ref.hpsi(psi, sample_bands, ld)
        done += sample_bands
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    return done / el, done, el


def run_reference(args, ws, rank):
    """CPU reference arm: the reference's algorithm for this path on the host cores."""
    if rank != 0:
        return
    load_package()
    sys.path.insert(0, str(ROOT))
    from oracle import hamilt_ref as H
    from oracle.pw_basis_ref import PWBasisKRef
    from importlib import import_module
    synth = import_module("abacus_develop_b200.synth")
    spec = synth.config(1)
    cell = synth.make_cell(spec)
    b = PWBasisKRef(spec.a, cell.latvec, spec.ecut, np.zeros((1, 3)))
    ld = int(b.npwk_max)
    veff = cell.veff(b.nx, b.ny, b.nz)
    vkb = cell.vkb(b.gplusk_cart(0), ld, b.omega)
    psi = cell.psi0(b.gplusk_cart(0), 8, ld).reshape(-1)
    cores = os.cpu_count() or 1
    H.FFT_WORKERS = cores
    ref = H.HamiltPWRef(b, 0, veff, vkb, cell.deeq(), [8], [cell.nat])
    sample = 4
    for _ in range(args.warmup):
        ref.hpsi(psi[:sample * ld], sample, ld)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.hpsi(psi[:sample * ld], sample, ld)
        times.append(time.perf_counter() - t0)
    per_step = float(np.mean(times))
    val = sample / per_step
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "bands/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "sample": f"{sample} of 160 bands per step"},
        "cpu_baseline": {"value": val, "unit": "bands/s", "cores": cores, "kind": "port",
                         "sample": f"{sample} bands of the 160-band block per step, numpy/scipy restatement of the "
                                   f"reference CPU functors and PW_Basis_K transforms, {cores} FFT/BLAS threads"},
        "e2e": {"value": val, "unit": "bands/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
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
    ms_loc32 = time_steps(local32, args.steps, stream)

    # end to end through the public API: pinned host psi -> device, H|psi>, hpsi -> pinned host
    psi_pin = torch.from_numpy(psi_h).pin_memory()
    out_pin = torch.empty_like(psi_pin).pin_memory()

    def e2e_step():
        psi.copy_(psi_pin, non_blocking=True)
        step64()
        out_pin.copy_(hpsi, non_blocking=True)

    for _ in range(2):
        e2e_step()
    barrier(ws)
    ms_e2e = max_over_ranks(time_steps(e2e_step, args.steps, stream), ws)

    hbm_peak, _, peak_kind = peaks()
    b_local64 = local_bytes_per_band(basis, 16, 8) * nb
    b_local32 = local_bytes_per_band(basis, 8, 4) * nb
    ach64 = b_local64 / (ms_loc64 * 1e-3) / 1e9
    ach32 = b_local32 / (ms_loc32 * 1e-3) / 1e9
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
                   "l2": "inputs larger than L2 (psi+hpsi+projectors ~690 MB), no flush"},
        "mixed": {"value": ws * nb / (ms32 * 1e-3), "unit": "bands/s", "ms_per_step": ms32,
                  "dtype": "f32 FFT + f32 projector GEMM"},
        "roofline": {"kernel": "fused local H|psi> FP64 (k_zpass_inv + k_plane + k_zpass_fwd)",
                     "bound": "hbm", "achieved": ach64, "peak": hbm_peak, "unit": "GB/s",
                     "frac": ach64 / hbm_peak, "peak_kind": peak_kind,
                     "traffic": NCU_TRAFFIC_LOCAL_FP64,
                     "algorithmic_bytes": b_local64, "ms": ms_loc64,
                     "mixed": {"achieved": ach32, "frac": ach32 / hbm_peak, "ms": ms_loc32,
                               "algorithmic_bytes": b_local32}},
        "nonlocal": {"flops": nl_flops, "ms_fp64": ms64 - ms_loc64, "tflops_fp64": nl_flops / ((ms64 - ms_loc64) * 1e-3) / 1e12},
        "e2e": {"value": ws * nb / (ms_e2e * 1e-3), "unit": "bands/s",
                "h2d_bytes_per_step": psi.numel() * 16, "d2h_bytes_per_step": hpsi.numel() * 16},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }

    if not args.skip_david:
        line["davidson"] = davidson_bench(P, wl, h64, h32)

    if rank == 0 and ws == 1 and not args.skip_cpu:
        bps, done, el = cpu_port_bands_per_s(wl, budget_s=args.cpu_budget)
        line["cpu_baseline"] = {"value": bps, "unit": "bands/s", "cores": 1, "kind": "port",
                                "sample": f"{done} bands of the 160-band block in {el:.1f} s, numpy restatement "
                                          f"of the reference CPU functors + PW_Basis_K transforms, 1 thread"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def davidson_bench(P, wl, h64, h32):
    """Time to eigenvalues within 1e-8 Ry of a tightly converged FP64 solve, FP64 vs mixed."""
    import torch
    nb = wl.spec.nbands
    ld = wl.basis.npwk_max
    pc = P.precondition_d(wl.basis, 0)
    psi0 = wl.psi0_h[0][:nb].reshape(-1)

    def solve(h, prec, thr):
        dav = P.DiagoDavid(pc, nb, ld, 4, prec)
        x = torch.from_numpy(psi0.copy()).cuda()
        e = np.zeros(nb)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it = dav.diag_hamilt(h, 0, ld, x, e, thr, 200)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, e, dav.stats()

    _, e_ref, it_ref = solve(h64, P.PREC_FP64, 1e-11)
    t64, e64, it64 = solve(h64, P.PREC_FP64, 1e-9)
    tmx, emx, itmx = solve(h64, P.PREC_MIXED, 1e-9)
    return {"fp64_s": t64, "mixed_s": tmx, "speedup": t64 / tmx,
            "fp64_iters": it64[1], "mixed_iters_fp32": itmx[0], "mixed_iters_fp64": itmx[1],
            "fp64_hpsi_bands": it64[2], "mixed_hpsi_bands": itmx[2], "ref_iters": it_ref[1],
            "fp64_max_err_ry": float(np.max(np.abs(e64 - e_ref))),
            "mixed_max_err_ry": float(np.max(np.abs(emx - e_ref))),
            "reference_solve": "FP64 Davidson to thr 1e-11 on the same device",
            "thr": 1e-9}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-david", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    args = ap.parse_args()
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
