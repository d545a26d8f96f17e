// Davidson with subspace rotation on the device: hsolver::Diago_DavSubspace<T, DEVICE_GPU>
// (module_hsolver/diago_dav_subspace.h:11-40), the "dav_subspace" method of HSolverPW.
#pragma once
#include <cuda_runtime.h>

#include <memory>

#include "david.h"

namespace b200 {

struct DavSubspaceBase {
    virtual ~DavSubspaceBase() = default;
    // Diago_DavSubspace::diag(hpsi_func, psi_in, psi_in_dmax, eigenvalue_in, is_occupied, scf_type)
    // (diago_dav_subspace.cpp:804-838): psi (complex128, nband vectors at psi + m*ldpsi, ldpsi >= dim) and
    // eig (host, nband) in place; occupied: host array of nband flags or nullptr (all occupied).  Returns the
    // total iteration count of all tries.
    virtual int diag(const HPsiDevice& f, void* psi, int ldpsi, double* eig, const int* occupied, bool scf) = 0;
    virtual void set_stream(cudaStream_t s) = 0;
    virtual void set_verbosity(int level) = 0;
    // unconverged bands after the last solve
    virtual int notconv() const = 0;
    // single-band applications of H in the last solve
    virtual int hpsi_bands() const = 0;
    virtual size_t device_bytes() const = 0;
};

// precond_d: device array of dim (HSolverPW passes |k+G|^2 tpiba2 for this method, hsolver_pw.cpp:573-580)
std::unique_ptr<DavSubspaceBase> make_dav_subspace(int nband, int dim, int david_ndim, double diag_thr, int diag_nmax,
                                                   bool need_subspace, const double* precond_d);

}  // namespace b200
