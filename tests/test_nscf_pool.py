"""The NSCF driver's k-point pool split on CPU (gloo, world size 2): each k-point solved by exactly one rank,
the eigenvalues gathered on every rank, the band file written once (rank 0) with every k-point, the
wavefunction files written by their owners and readable bit for bit, smeared occupations from the gathered
eigenvalues.  The band solve is injected: a small
dense stand-in (exact eigenpairs of a per-k Hermitian matrix), since this test is about the host logic."""
from __future__ import annotations

import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KD = [[0.0, 0.0, 0.0], [0.25, 0.0, 0.0], [0.25, 0.25, 0.0], [0.5, 0.25, 0.0], [0.5, 0.5, 0.5]]
LATVEC = np.eye(3)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _basis(pkg):
    return pkg.pwdft.PWBasisK(10.26, LATVEC, 8.0, np.array(KD))


def _stand_in_solve(basis):
    def solve(iks, psi_init, nbands, thr):
        ekb, psis = [], []
        for ik, x0 in zip(iks, psi_init):
            n = int(basis.npwk[ik])
            g2 = basis.gk2_k(ik) * basis.tpiba2
            h = np.diag(g2).astype(complex) + 0.05 * np.exp(1j * np.add.outer(np.arange(n), -np.arange(n)) / n)
            h = 0.5 * (h + h.conj().T)
            w, v = np.linalg.eigh(h)
            ekb.append(w[:nbands])
            psis.append(np.ascontiguousarray(v[:, :nbands].T))
        return np.array(ekb).reshape(len(iks), nbands), np.full(len(iks), 7, dtype=np.int32), psis
    return solve


def _worker(rank, ws, port, outdir, q):
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_package
    pkg = load_package()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        b = _basis(pkg)
        nb = 6
        psi0 = [np.zeros((nb, int(b.npwk[ik])), complex) for ik in range(b.nks)]
        res = pkg.nscf.run_nscf_pool(b, nb, psi0, _stand_in_solve(b), wk=[0.4] * b.nks, nelec=8.0, latvec=LATVEC,
                                     ecutwfc=8.0, pw_diag_thr=1e-9, out_dir=outdir, out_wfc_pw=2)
        sm = pkg.nscf.run_nscf_pool(b, nb, psi0, _stand_in_solve(b), wk=[0.4] * b.nks, nelec=7.0, latvec=LATVEC,
                                    ecutwfc=8.0, pw_diag_thr=1e-9, smearing=("mp", 0.01))
        q.put((rank, res.iks, res.ekb.tolist(), res.ef, res.iters.tolist(), res.files.get("wfc", []), sm.ef,
               sm.wg.tolist(), [np.asarray(x) for x in res.psis]))
    finally:
        dist.destroy_process_group()


def test_nscf_pool_two_ranks(pkg, tmp_path, monkeypatch):
    # one BLAS thread per rank: two ranks whose BLAS pools each span every core spend the test spinning
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        monkeypatch.setenv(var, "1")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path), q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=180) for _ in range(2)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    b = _basis(pkg)
    nb = 6
    ekb_ref = _stand_in_solve(b)(list(range(b.nks)), [None] * b.nks, nb, 0.0)[0]
    gathered = np.array(res[0][2])
    assert np.max(np.abs(gathered - ekb_ref)) < 1e-12     # the ranks' BLAS threads differ from this process's
    wg_s, ef_s, _ = pkg.nscf.smearing_weights(gathered, [0.4] * b.nks, 7.0, 0.01, "mp")
    owned, psi_by_k = [], {}
    for rank, iks, ekb, ef, iters, wfc, sm_ef, sm_wg, psis in res:
        owned += iks
        assert np.array_equal(np.array(ekb), gathered)         # the same gathered array on every rank
        assert ef == float(np.max(gathered[:, :4])) and iters == [7] * b.nks
        assert len(wfc) == len(iks)
        assert sm_ef == ef_s and np.array_equal(np.array(sm_wg), wg_s)  # smeared occupations from the gather
        psi_by_k.update(zip(iks, psis))
    assert sorted(owned) == list(range(b.nks))
    band = (tmp_path / "BANDS_1.dat").read_text().rstrip("\n").split("\n")
    assert len(band) == b.nks and band[0].startswith("   1 0.00000000")
    io = pkg.nscf_io
    for ik in range(b.nks):
        back = io.read_wfc_pw(tmp_path / f"WAVEFUNC{ik + 1}.dat", b, ik, b.nks, nb, LATVEC)
        assert np.array_equal(back, psi_by_k[ik])
