"""Build oracle/_ref/libref_david.so: the reference's own CPU DiagoDavid, compiled from its sources.

Test infrastructure: only the tests and bench.py's CPU reference arm load the library.  Run in a container
where the reference tree is mounted, given by the ABACUS_REF environment variable or build(ref=...); the result is a
shared library under oracle/_ref/ (git-ignored) that needs only scipy's bundled OpenBLAS at run time.

Compiled from the reference (unchanged, from where they lie):
  source/module_hsolver/diago_david.cpp            the Davidson iteration
  source/module_hsolver/diago_dav_subspace.cpp     the Davidson-subspace iteration (HSolverPW method "dav_subspace")
  source/module_hsolver/diag_const_nums.cpp        its constants (one, zero, minus one)
  source/module_hsolver/kernels/math_kernel_op.cpp the CPU BLAS functors it calls (gemm_op, gemv_op, ...)
  source/module_hsolver/kernels/dngvd_op.cpp       dnevx_op / dngvd_op (LAPACK zheevx, zhegvd, ...)
  source/module_base/module_device/memory_op.cpp   resize / set / sync / delete memory ops
  source/module_base/timer.cpp                     ModuleBase::timer::tick
  source/module_hsolver/diago_bpcg.cpp             the band-parallel CG iteration (HSolverPW method "bpcg")
  source/module_psi/psi.cpp, module_parameter/parameter.cpp, module_hamilt_general/operator.cpp
                                                   the psi / global-parameter / operator layer BPCG calls
  source/module_base/module_container/{ATen/core,ATen/ops,ATen/kernels,base/core}/*.cpp
                                                   the tensor library BPCG is written in (einsum, BLAS, LAPACK)
  source/module_elecstate/occupy.cpp, module_base/matrix.cpp
                                                   occupations (smearing weights, Fermi energy) of an NSCF run
  source/module_basis/module_pw/{pw_basis,pw_basis_k,pw_init,pw_distributeg*,pw_distributer,fft,
  pw_transform_k}.cpp, module_base/matrix3.cpp, module_base/mymath.cpp
                                                   the plane-wave basis and its transforms
  source/module_hamilt_pw/hamilt_pwdft/{operator_pw/{operator_pw,ekinetic_pw,veff_pw},kernels/{ekinetic_op,
  veff_op}}.cpp                                    the kinetic and local operators of H|psi>
  source/module_hamilt_pw/hamilt_pwdft/{operator_pw/nonlocal_pw,kernels/nonlocal_op}.cpp
                                                   the nonlocal operator of H|psi> (Nonlocal::init / act /
                                                   add_nonlocal_pp with its functor), compiled against
                                                   ref/nl_stub/: stand-ins for UnitCell and
                                                   pseudopot_cell_vnl that declare only the members it reads
plus this directory's ref/shim.cpp (process-level services: WARNING_QUIT throws, TITLE is silent, the CPU
device tag, a one-process reduce_pool, NPROC_IN_POOL = 1, diagH_LAPACK on the reference's dngvd_op) and
ref/david_capi.cpp, ref/dav_subspace_capi.cpp, ref/bpcg_capi.cpp (C entry points with a callback H|psi>),
ref/occupy_capi.cpp (the occupation functions), ref/pw_basis_capi.cpp (the basis set-up, its transforms
and the local H|psi> operators), ref/nonlocal_capi.cpp (the nonlocal operator).
ref/include/fftw3.h declares the FFTW API names those sources use and ref/fftw_stub.cpp stands in for them
(FFTW is absent): plans record a batch of 1-D complex transforms that executing runs as mixed-radix FFTs.

The reference calls Fortran BLAS/LAPACK (zgemm_, zheevx_, ...); scipy's OpenBLAS exports the same routines
under a scipy_ prefix, so the object files' references are renamed with objcopy before linking.
No cmake, no reference build system, no network.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
def _ref_source(ref: str | os.PathLike | None) -> Path | None:
    """The reference's source/ tree: the argument, else $ABACUS_REF; None when neither is given."""
    root = ref if ref is not None else os.environ.get("ABACUS_REF")
    return Path(root) / "source" if root else None
SOURCES = [
    "module_hsolver/diago_david.cpp",
    "module_hsolver/diago_dav_subspace.cpp",
    "module_hsolver/diag_const_nums.cpp",
    "module_hsolver/kernels/math_kernel_op.cpp",
    "module_hsolver/kernels/dngvd_op.cpp",
    "module_base/module_device/memory_op.cpp",
    "module_base/timer.cpp",
    # DiagoBPCG and what it stands on: the psi / operator layer and the container tensor library
    "module_hsolver/diago_bpcg.cpp",
    "module_psi/psi.cpp",
    "module_parameter/parameter.cpp",
    "module_hamilt_general/operator.cpp",
    "module_base/module_container/ATen/core/tensor.cpp",
    "module_base/module_container/ATen/core/tensor_map.cpp",
    "module_base/module_container/ATen/core/tensor_shape.cpp",
    "module_base/module_container/ATen/core/tensor_buffer.cpp",
    "module_base/module_container/ATen/core/tensor_types.cpp",
    "module_base/module_container/ATen/ops/einsum_op.cpp",
    "module_base/module_container/ATen/ops/linalg_op.cpp",
    "module_base/module_container/ATen/kernels/blas.cpp",
    "module_base/module_container/ATen/kernels/lapack.cpp",
    "module_base/module_container/ATen/kernels/linalg.cpp",
    "module_base/module_container/ATen/kernels/memory_impl.cpp",
    "module_base/module_container/base/core/cpu_allocator.cpp",
    "module_base/module_container/base/core/refcount.cpp",
    # the occupation code of the NSCF weights and the matrix class it takes
    "module_elecstate/occupy.cpp",
    "module_base/matrix.cpp",
    # the plane-wave basis set-up (spheres, sticks, index maps); its FFT plans go to oracle/ref/fftw_stub.cpp
    "module_basis/module_pw/pw_basis.cpp",
    "module_basis/module_pw/pw_basis_k.cpp",
    "module_basis/module_pw/pw_init.cpp",
    "module_basis/module_pw/pw_distributeg.cpp",
    "module_basis/module_pw/pw_distributeg_method1.cpp",
    "module_basis/module_pw/pw_distributeg_method2.cpp",
    "module_basis/module_pw/pw_distributer.cpp",
    "module_basis/module_pw/fft.cpp",
    "module_basis/module_pw/pw_transform_k.cpp",
    # the kinetic and local operators of H|psi> and their CPU kernels
    "module_hamilt_pw/hamilt_pwdft/operator_pw/operator_pw.cpp",
    "module_hamilt_pw/hamilt_pwdft/operator_pw/ekinetic_pw.cpp",
    "module_hamilt_pw/hamilt_pwdft/operator_pw/veff_pw.cpp",
    "module_hamilt_pw/hamilt_pwdft/kernels/ekinetic_op.cpp",
    "module_hamilt_pw/hamilt_pwdft/kernels/veff_op.cpp",
    "module_hamilt_pw/hamilt_pwdft/operator_pw/nonlocal_pw.cpp",
    "module_hamilt_pw/hamilt_pwdft/kernels/nonlocal_op.cpp",
    "module_base/matrix3.cpp",
    "module_base/mymath.cpp",
]
OWN = [HERE / "ref" / "shim.cpp", HERE / "ref" / "david_capi.cpp", HERE / "ref" / "dav_subspace_capi.cpp",
       HERE / "ref" / "bpcg_capi.cpp", HERE / "ref" / "occupy_capi.cpp", HERE / "ref" / "pw_basis_capi.cpp",
       HERE / "ref" / "fftw_stub.cpp", HERE / "ref" / "nonlocal_capi.cpp"]
# compiled with ref/nl_stub/ ahead of the reference tree on the include path (the cell and projector
# stand-ins the nonlocal operator is built against); every other file sees only the reference's headers
NL_STUB = {"nonlocal_pw.cpp", "nonlocal_op.cpp", "nonlocal_capi.cpp"}


def openblas() -> Path:
    import scipy
    libs = sorted(glob.glob(str(Path(scipy.__file__).resolve().parent.parent / "scipy.libs" / "libscipy_openblas*.so")))
    if not libs:
        raise RuntimeError("scipy's bundled OpenBLAS not found")
    return Path(libs[0])


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(" ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
    return r.stdout


def build(quiet: bool = False, ref: str | os.PathLike | None = None) -> Path | None:
    """Compile the library from the reference checkout at `ref` (or $ABACUS_REF); without either, or when the
    tree is absent, nothing is built and None is returned."""
    REF = _ref_source(ref)
    if REF is None or not REF.exists():
        if not quiet:
            print("reference tree not given (ABACUS_REF unset) or not present: oracle/_ref not rebuilt",
                  file=sys.stderr)
        return None
    OUT.mkdir(exist_ok=True)
    tmp = OUT / "obj"
    tmp.mkdir(exist_ok=True)
    flags = ["-std=c++14", "-O2", "-fPIC", "-fopenmp", f"-I{HERE / 'ref' / 'include'}", f"-I{REF}",
             f"-I{REF / 'module_base/module_container'}"]
    objs = []
    for src in [REF / s for s in SOURCES] + OWN:
        obj = tmp / (src.parent.name + "_" + src.stem + ".o")
        extra = [f"-I{HERE / 'ref' / 'nl_stub'}"] if src.name in NL_STUB else []
        run(["g++", *extra, *flags, "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    # Fortran BLAS / LAPACK references -> scipy_ names
    lib = openblas()
    exported = set(ln.split()[-1] for ln in run(["nm", "-D", "--defined-only", str(lib)]).splitlines() if ln.strip())
    for obj in objs:
        undef = [ln.split()[-1] for ln in run(["nm", "-u", str(obj)]).splitlines() if ln.strip()]
        ren = [f"--redefine-sym={s}=scipy_{s}" for s in undef if s.endswith("_") and ("scipy_" + s) in exported]
        if ren:
            run(["objcopy", *ren, str(obj)])
    so = OUT / "libref_david.so"
    run(["g++", "-shared", "-fopenmp", "-o", str(so), *map(str, objs), str(lib), f"-Wl,-rpath,{lib.parent}"])
    shutil.rmtree(tmp)
    return so


if __name__ == "__main__":
    print(build(ref=sys.argv[1] if len(sys.argv) > 1 else None))
