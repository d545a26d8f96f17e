"""k-point pools across GPUs: which rank solves which k-point, and the gather of eigenvalues.

ABACUS on GPUs parallelises only over k-points (one pool per process, each pool
binds one GPU: module_base/module_device/device.cpp:195-217, the k-point
division of module_base/parallel_global.cpp:239-302).  Here the same split is
cost-balanced: a k-point's cost is taken as npw_k * nbands^2 (the Davidson
subspace products dominate), and k-points are handed out largest first to the
least loaded rank.  Ranks never exchange wavefunctions; the only collective is
the final all-gather of the (nks x nbands) eigenvalues.
"""
from __future__ import annotations

import numpy as np


def partition(npwk, nbands: int, nranks: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment of k-points to ranks (deterministic)."""
    npwk = np.asarray(npwk, dtype=np.int64)
    cost = npwk.astype(np.float64) * float(nbands) ** 2
    order = sorted(range(len(npwk)), key=lambda i: (-cost[i], i))
    load = [0.0] * nranks
    out: list[list[int]] = [[] for _ in range(nranks)]
    for ik in order:
        r = min(range(nranks), key=lambda j: (load[j], j))
        out[r].append(ik)
        load[r] += cost[ik]
    return [sorted(v) for v in out]


def gather_eigenvalues(local: dict, nks: int, nbands: int, group=None) -> np.ndarray:
    """All-gather {ik: eigenvalues} from every rank into an (nks, nbands) array on every rank."""
    import torch
    import torch.distributed as dist
    ws = dist.get_world_size(group) if dist.is_initialized() else 1
    buf = torch.full((nks, nbands), float("nan"), dtype=torch.float64)
    for ik, e in local.items():
        buf[ik] = torch.as_tensor(np.asarray(e, dtype=np.float64))
    if ws == 1:
        return buf.numpy()
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    parts = [torch.empty_like(buf, device=dev) for _ in range(ws)]
    dist.all_gather(parts, buf.to(dev), group=group)
    full = parts[0].cpu().clone()
    for p in parts[1:]:
        p = p.cpu()
        mask = ~torch.isnan(p)
        full[mask] = p[mask]
    return full.numpy()
