"""CPU (gloo, world size 2) tests of the multi-GPU host logic: k-point pools and the eigenvalue gather."""
from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_balanced_and_complete(pkg):
    part = pkg.kpool.partition
    npwk = [2984, 3022, 3001, 2990, 3010, 2999, 3020, 2985] * 8
    for nr in (1, 2, 3, 4, 8):
        p = part(npwk, 32, nr)
        flat = sorted(i for v in p for i in v)
        assert flat == list(range(len(npwk)))
        loads = [sum(npwk[i] for i in v) for v in p]
        assert max(loads) - min(loads) <= max(npwk)
    assert part(npwk, 32, 4) == part(npwk, 32, 4)  # deterministic


def _worker(rank, ws, port, out_q):
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_package
    pkg = load_package()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        nks, nb = 6, 4
        mine = pkg.kpool.partition([100 + i for i in range(nks)], nb, ws)[rank]
        local = {ik: np.arange(nb) + 10.0 * ik for ik in mine}
        full = pkg.kpool.gather_eigenvalues(local, nks, nb)
        out_q.put((rank, mine, full.tolist()))
    finally:
        dist.destroy_process_group()


def test_gather_eigenvalues_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = np.array([np.arange(4) + 10.0 * ik for ik in range(6)])
    owned = set()
    for rank, mine, full in res:
        assert np.array_equal(np.array(full), expect)
        owned |= set(mine)
    assert owned == set(range(6))


def test_rank_failure_is_reported(tmp_path):
    """A rank that dies before the gather makes the other rank fail with an error (short timeout), not hang."""
    ctx = mp.get_context("spawn")
    port = _free_port()
    p0 = ctx.Process(target=_dying_worker, args=(0, port, str(tmp_path)))
    p1 = ctx.Process(target=_dying_worker, args=(1, port, str(tmp_path)))
    p0.start()
    p1.start()
    p0.join(timeout=120)
    p1.join(timeout=120)
    assert p1.exitcode == 3  # the rank that "crashed" between steps
    assert (tmp_path / "rank0_error").exists()


def _dying_worker(rank, port, outdir):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(3)  # leaves between steps, nothing in flight
    try:
        t = torch.zeros(4)
        dist.all_reduce(t)
    except Exception as e:  # noqa: BLE001
        open(os.path.join(outdir, "rank0_error"), "w").write(str(e)[:200])
    os._exit(0)
