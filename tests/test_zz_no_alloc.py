"""GPU test of the allocation-free local H|psi> entry point.

Some callers cannot allocate device memory at the point of the call: code that
runs inside a CUDA-graph capture (cudaMalloc is not capturable), code whose
device memory belongs to a host framework's pool, and paths that must not
synchronise the device.  b200_hamilt_hpsi_local_noalloc serves them with a
fixed scratch array inside the library.  This test calls it through the C-ABI
twice in a row (the second call sees the first call's leftovers in the shared
scratch) and compares each result with the regular entry point
b200_hamilt_hpsi_part(mode = 1), within the FP64 tolerance of the other H|psi>
tests (1e-12 relative) and the FP32 one (2e-6).  It sits in a file collected
last so that a stop-at-first-failure run has run every other test first, and it
builds everything it needs itself, so it also passes alone in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("cfg,prec,tol", [(0, 0, 1e-12), (1, 0, 1e-12), (0, 1, 2e-6)])
def test_noalloc_matches_regular_entry_point(pkg, cfg, prec, tol):
    P = pkg.pwdft
    lib = pkg._lib.load()
    spec = pkg.synth.config(cfg)
    wl = P.build_workload(spec)
    h = P.device_hamilt(wl, prec)
    ld = wl.basis.npwk_max
    nb = spec.nbands if cfg == 0 else 40  # 40 bands of the 64-atom cell span several scratch chunks
    dt = torch.complex128 if prec == 0 else torch.complex64
    psi = torch.from_numpy(wl.psi0_h[0][:nb].reshape(-1)).to(dt).cuda()
    ref = torch.zeros_like(psi)
    h.hpsi_part(0, psi, ref, nb, ld, 1)
    torch.cuda.synchronize()
    ref_h = ref.cpu().numpy().astype(np.complex128)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = torch.full_like(psi, complex(3.0, -1.0))
        rc = lib.b200_hamilt_hpsi_local_noalloc(h.handle, 0, nb, ld, ctypes.c_void_p(psi.data_ptr()),
                                                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
        assert rc == 0, lib.b200_last_error().decode()
        torch.cuda.synchronize()
        assert rel(out.cpu().numpy().astype(np.complex128), ref_h) < tol, f"call {call}"


def test_noalloc_rejects_bad_arguments(pkg):
    P = pkg.pwdft
    lib = pkg._lib.load()
    wl = P.build_workload(pkg.synth.serving_cells()[0])
    h = P.device_hamilt(wl, 0)
    ld = wl.basis.npwk_max
    x = torch.zeros(8 * ld, dtype=torch.complex128, device="cuda")
    rc = lib.b200_hamilt_hpsi_local_noalloc(h.handle, 0, 8, ld - 1, ctypes.c_void_p(x.data_ptr()),
                                            ctypes.c_void_p(x.data_ptr()), None)
    assert rc == 1 and b"ld" in lib.b200_last_error()
    rc = lib.b200_hamilt_hpsi_local_noalloc(None, 0, 8, ld, None, None, None)
    assert rc == 1
