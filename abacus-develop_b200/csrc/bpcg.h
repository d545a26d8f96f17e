// Band-parallel preconditioned conjugate gradient on the device: hsolver::DiagoBPCG<T, DEVICE_GPU>
// (module_hsolver/diago_bpcg.h:18-337), the "bpcg" method of HSolverPW.
#pragma once
#include <cuda_runtime.h>

#include <memory>

#include "david.h"

namespace b200 {

struct BpcgBase {
    virtual ~BpcgBase() = default;
    // DiagoBPCG::diag(hamilt, psi, eigenvalue) (diago_bpcg.cpp:254-306) with DiagoIterAssist::SCF_ITER =
    // scf_iter: psi (complex128, nband vectors of nbasis entries at psi + m*nbasis) and eig (host, nband)
    // replaced; H applied through f to all nband vectors of a block.  Returns the iterations of the loop.
    virtual int diag(const HPsiDevice& f, void* psi, double* eig, int scf_iter) = 0;
    virtual void set_stream(cudaStream_t s) = 0;
    // largest residual norm |H psi - eps psi| of the last iteration of the last diag (host copy)
    virtual double max_err() const = 0;
    virtual int hpsi_bands() const = 0;
    virtual size_t device_bytes() const = 0;
};

// precond_d: device array of nbasis (HSolverPW passes 1 + g2 + sqrt(1 + (g2 - 1)^2) on the plane waves and
// 1 on the padding, hsolver_pw.cpp:549-584)
std::unique_ptr<BpcgBase> make_bpcg(int nband, int nbasis, const double* precond_d);

}  // namespace b200
