"""ctypes binding of libabacus_b200.so (the C-ABI in include/abacus_b200.h).

The library is loaded from this directory; a missing library or a failing call
raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libabacus_b200.so"
HEADER = HERE.parent / "include" / "abacus_b200.h"

vp = C.c_void_p
i32 = C.c_int
f64 = C.c_double
f32 = C.c_float
pi32 = C.POINTER(C.c_int)
pf64 = C.POINTER(C.c_double)

HPSI_CB = C.CFUNCTYPE(i32, vp, vp, vp, i32, i32, i32, i32)

_SIGS = {
    "b200_last_error": ([], C.c_char_p),
    "b200_version": ([], C.c_char_p),
    "b200_kernel_launches": ([], C.c_ulonglong),
    "b200_ekinetic_pw_op_f64": ([i32, i32, i32, f64, vp, vp, vp, vp], i32),
    "b200_ekinetic_pw_op_f32": ([i32, i32, i32, f32, vp, vp, vp, vp], i32),
    "b200_veff_pw_op_f64": ([i32, vp, vp, vp], i32),
    "b200_veff_pw_op_f32": ([i32, vp, vp, vp], i32),
    "b200_veff_pw_op_npol2_f64": ([i32, vp, vp, vp, vp, vp, vp, vp], i32),
    "b200_veff_pw_op_npol2_f32": ([i32, vp, vp, vp, vp, vp, vp, vp], i32),
    "b200_nonlocal_pw_op_f64": ([i32, i32, i32, pi32, pi32, i32, i32, i32, i32, i32, vp, vp, vp, vp], i32),
    "b200_nonlocal_pw_op_f32": ([i32, i32, i32, pi32, pi32, i32, i32, i32, i32, i32, vp, vp, vp, vp], i32),
    "b200_nonlocal_pw_op_nc_f64": ([i32, i32, i32, pi32, pi32, i32, i32, i32, i32, vp, vp, vp, vp], i32),
    "b200_nonlocal_pw_op_nc_f32": ([i32, i32, i32, pi32, pi32, i32, i32, i32, i32, vp, vp, vp, vp], i32),
    "b200_set_3d_fft_box_op_f64": ([i32, vp, vp, vp, vp], i32),
    "b200_set_3d_fft_box_op_f32": ([i32, vp, vp, vp, vp], i32),
    "b200_set_recip_to_real_output_op_f64": ([i32, i32, f64, vp, vp, vp], i32),
    "b200_set_recip_to_real_output_op_f32": ([i32, i32, f32, vp, vp, vp], i32),
    "b200_set_real_to_recip_output_op_f64": ([i32, i32, i32, f64, vp, vp, vp, vp], i32),
    "b200_set_real_to_recip_output_op_f32": ([i32, i32, i32, f32, vp, vp, vp, vp], i32),
    "b200_pw_basis_create": ([f64, pf64, f64, f64, i32, i32, i32, i32, pf64, C.POINTER(vp)], i32),
    "b200_pw_basis_destroy": ([vp], i32),
    "b200_pw_basis_dims": ([vp, pi32], i32),
    "b200_pw_basis_scalars": ([vp, pf64], i32),
    "b200_pw_basis_kpoint": ([vp, i32, pi32, vp, vp, vp], i32),
    "b200_pw_basis_kvec_c": ([vp, i32, pf64], i32),
    "b200_pw_basis_device_maps": ([vp, i32, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)], i32),
    "b200_recip_to_real_f64": ([vp, vp, vp, i32, i32, f64, vp], i32),
    "b200_recip_to_real_f32": ([vp, vp, vp, i32, i32, f32, vp], i32),
    "b200_real_to_recip_f64": ([vp, vp, vp, i32, i32, f64, vp], i32),
    "b200_real_to_recip_f32": ([vp, vp, vp, i32, i32, f32, vp], i32),
    "b200_hamilt_create": ([vp, i32, C.POINTER(vp)], i32),
    "b200_hamilt_destroy": ([vp], i32),
    "b200_hamilt_set_veff": ([vp, vp], i32),
    "b200_hamilt_set_vkb": ([vp, i32, i32, i32, vp], i32),
    "b200_hamilt_set_deeq": ([vp, i32, pi32, pi32, i32, i32, i32, i32, vp], i32),
    "b200_hamilt_hpsi": ([vp, i32, i32, i32, i32, vp, vp, vp], i32),
    "b200_hamilt_hpsi_part": ([vp, i32, i32, i32, i32, vp, vp, i32, vp], i32),
    "b200_hamilt_hpsi_host": ([vp, i32, i32, i32, i32, vp, vp, vp, vp, i32, vp], i32),
    "b200_hamilt_hpsi_local_noalloc": ([vp, i32, i32, i32, vp, vp, vp], i32),
    "b200_hamilt_hpsi_kbatch": ([vp, i32, pi32, i32, i32, i32, C.POINTER(vp), C.POINTER(vp), vp], i32),
    "b200_graph_capture_hpsi_kbatch": ([vp, i32, pi32, i32, i32, i32, C.POINTER(vp), C.POINTER(vp), vp,
                                        C.POINTER(vp)], i32),
    "b200_graph_launch": ([vp, vp], i32),
    "b200_graph_destroy": ([vp], i32),
    "b200_hamilt_autotune": ([vp, i32, i32, i32, vp, vp, vp, pi32, pi32], i32),
    "b200_hamilt_set_plane_variant": ([vp, i32], i32),
    "b200_hamilt_set_band_chunk": ([vp, i32], i32),
    "b200_server_set_express": ([vp, i32, f64], i32),
    "b200_server_set_policy": ([vp, i32, f64], i32),
    "b200_elecstate_pw_op_f64": ([i32, i32, f64, C.POINTER(vp), vp, vp], i32),
    "b200_elecstate_pw_op_f32": ([i32, i32, f32, C.POINTER(vp), vp, vp], i32),
    "b200_elecstate_pw_op_nc_f64": ([i32, i32, i32, f64, C.POINTER(vp), vp, vp, vp], i32),
    "b200_elecstate_pw_op_nc_f32": ([i32, i32, i32, f32, C.POINTER(vp), vp, vp, vp], i32),
    "b200_pw_basis_psi_to_rho_f64": ([vp, i32, i32, i32, vp, pf64, vp, vp], i32),
    "b200_pw_basis_psi_to_rho_f32": ([vp, i32, i32, i32, vp, pf64, vp, vp], i32),
    "b200_cal_ylm_real_op_f64": ([i32, i32, vp, vp, vp], i32),
    "b200_cal_ylm_real_op_f32": ([i32, i32, vp, vp, vp], i32),
    "b200_cal_sk_op_f64": ([i32] * 14 + [pi32, vp, vp, f64, vp, vp, vp, vp, vp, vp, vp], i32),
    "b200_cal_sk_op_f32": ([i32] * 14 + [pi32, vp, vp, f32, vp, vp, vp, vp, vp, vp, vp], i32),
    "b200_cal_vnl_op_f64": ([i32] * 6 + [pi32, pi32, pi32, f64, f64] + [vp] * 10, i32),
    "b200_cal_vnl_op_f32": ([i32] * 6 + [pi32, pi32, pi32, f32, f32] + [vp] * 10, i32),
    "b200_hamilt_set_projectors": ([vp, i32, pi32, pi32, pi32, i32, i32, pi32, pi32, pi32, i32, i32, f64, pf64, pf64],
                                   i32),
    "b200_hamilt_build_vkb": ([vp, i32, vp], i32),
    "b200_server_create": ([C.c_ulonglong, i32, i32, C.POINTER(vp)], i32),
    "b200_server_destroy": ([vp], i32),
    "b200_server_add_cell": ([vp, vp, i32, pi32], i32),
    "b200_server_submit": ([vp, i32, i32, i32, i32, f64, i32, C.c_ulonglong, pf64, C.POINTER(C.c_longlong)], i32),
    "b200_server_poll": ([vp, i32, i32, C.POINTER(C.c_longlong), pi32, pf64, pf64, pf64, pi32, pi32, pi32], i32),
    "b200_server_drain": ([vp], i32),
    "b200_server_stats": ([vp, pf64], i32),
    "b200_hamilt_copy_vkb": ([vp, i32, vp, vp], i32),
    "b200_solve_kpoints": ([vp, i32, pi32, i32, i32, i32, i32, C.POINTER(vp), C.POINTER(vp), i32, pf64, f64, i32,
                            i32, i32, i32, pi32], i32),
    "b200_solve_kpoints_batched": ([vp, i32, pi32, i32, i32, i32, i32, C.POINTER(vp), C.POINTER(vp), i32, pf64, f64,
                                    i32, pi32, vp], i32),
    "b200_tc_cgemm": ([C.c_char, C.c_char, i32, i32, i32, f32, f32, vp, i32, vp, i32, f32, f32, vp, i32, vp], i32),
    "b200_tc_cgemm_error": ([pi32], i32),
    "b200_tc_set_wait_limit_ns": ([C.c_ulonglong], i32),
    "b200_measure_peaks": ([pf64, pf64, pf64], i32),
    "b200_gemm_op_f64": ([C.c_char, C.c_char, i32, i32, i32, pf64, vp, i32, vp, i32, pf64, vp, i32, vp], i32),
    "b200_zgemm_i8": ([C.c_char, C.c_char, i32, i32, i32, pf64, vp, i32, vp, i32, pf64, vp, i32, i32, vp], i32),
    "b200_zgemm_i8_error": ([pi32], i32),
    "b200_hamilt_set_fp64_gemm": ([vp, i32, i32], i32),
    "b200_hamilt_set_veff_nc": ([vp, vp], i32),
    "b200_hamilt_set_deeq_nc": ([vp, i32, pi32, pi32, i32, i32, i32, vp], i32),
    "b200_hamilt_hpsi_nc": ([vp, i32, i32, i32, vp, vp, vp], i32),
    "b200_zgemm_i8_constants": ([i32, C.c_longlong, pi32, pf64, pf64, pf64, pi32], i32),
    "b200_gemv_op_f64": ([C.c_char, i32, i32, pf64, vp, i32, vp, i32, pf64, vp, i32, vp], i32),
    "b200_dot_real_op_f64": ([i32, vp, vp, i32, pf64, vp], i32),
    "b200_dot_real_op_f32": ([i32, vp, vp, i32, C.POINTER(C.c_float), vp], i32),
    "b200_david_create": ([i32, i32, i32, i32, vp, C.POINTER(vp)], i32),
    "b200_david_destroy": ([vp], i32),
    "b200_david_diag": ([vp, HPSI_CB, vp, i32, vp, pf64, f64, i32, i32, i32, pi32], i32),
    "b200_david_diag_hamilt": ([vp, vp, i32, i32, i32, vp, pf64, f64, i32, i32, i32, pi32], i32),
    "b200_david_stats": ([vp, pi32, pi32, pi32], i32),
    "b200_david_set_trace": ([vp, i32], i32),
    "b200_david_set_low_ndim": ([vp, i32], i32),
    "b200_david_trace": ([vp, i32, i32, pf64, pi32, pf64, pi32], i32),
    "b200_david_set_verbosity": ([vp, i32], i32),
    "b200_david_set_stream": ([vp, vp], i32),
    "b200_david_set_mixed_threshold": ([vp, f64], i32),
    "b200_david_set_fp64_gemm": ([vp, i32], i32),
    "b200_dav_subspace_create": ([i32, i32, i32, f64, i32, i32, vp, C.POINTER(vp)], i32),
    "b200_dav_subspace_destroy": ([vp], i32),
    "b200_dav_subspace_diag": ([vp, HPSI_CB, vp, vp, i32, pf64, pi32, i32, pi32], i32),
    "b200_dav_subspace_diag_hamilt": ([vp, vp, i32, i32, vp, i32, pf64, pi32, i32, pi32], i32),
    "b200_dav_subspace_set_stream": ([vp, vp], i32),
    "b200_dav_subspace_set_verbosity": ([vp, i32], i32),
    "b200_dav_subspace_stats": ([vp, pi32, pi32], i32),
    "b200_bpcg_create": ([vp, i32, i32, C.POINTER(vp)], i32),
    "b200_bpcg_destroy": ([vp], i32),
    "b200_bpcg_diag": ([vp, HPSI_CB, vp, vp, pf64, i32, pi32], i32),
    "b200_bpcg_diag_hamilt": ([vp, vp, i32, i32, vp, pf64, i32, pi32], i32),
    "b200_bpcg_set_stream": ([vp, vp], i32),
    "b200_bpcg_stats": ([vp, pf64, pi32], i32),
}

_lib = None


class B200Error(RuntimeError):
    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


def header_symbols() -> list[str]:
    """Entry points declared in include/abacus_b200.h."""
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*|unsigned long long)\s+(b200_\w+)\s*\(", txt, re.M)))


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: run abacus-develop_b200/build.py (no CPU fallback exists)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != 0:
        raise B200Error(name, rc, lib.b200_last_error().decode())


class HostCallback:
    """A Python H|psi> function as a b200_hpsi_cb.  ctypes cannot carry an exception out of a callback (it
    prints it and returns to C as if nothing happened), so the exception is kept here, the callback returns
    1 and the solver abandons the solve with B200_STATUS_CALLBACK_ERROR; call_with() then raises the kept
    exception.  After a successful call the current torch stream is synchronised, so the block's writes are
    complete when the solver reads them, whichever stream the function used."""

    def __init__(self, fn):
        self.exc = None

        def cb(user, x, hx, nvec, dim, i0, i1):
            try:
                fn(x, hx, nvec, dim, i0, i1)
                import torch
                torch.cuda.current_stream().synchronize()
                return 0
            except BaseException as exc:  # noqa: BLE001 -- re-raised by call_with on the Python side
                if self.exc is None:
                    self.exc = exc
                return 1

        self.cfn = HPSI_CB(cb)

    def call_with(self, name: str, *args) -> None:
        try:
            call(name, *args)
        except B200Error:
            if self.exc is not None:
                raise self.exc
            raise


def ptr(t) -> int:
    """Device pointer of a torch tensor (or None)."""
    return None if t is None else t.data_ptr()


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
