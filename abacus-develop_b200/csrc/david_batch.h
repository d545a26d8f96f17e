// Lock-step Davidson of many k-points of one Hamiltonian (david_batch.cu).
#pragma once
#include <cuda_runtime.h>

#include <memory>

namespace b200 {

struct Hamilt;
class DavidBatchSolver;

// A reusable batched solver for up to `cap` k-points with at most `dim_cap` plane waves each, nband bands,
// subspace david_ndim * nband; precision B200_PREC_FP64 or B200_PREC_MIXED.  Every buffer is made here.
std::unique_ptr<DavidBatchSolver, void (*)(DavidBatchSolver*)> make_david_batch(Hamilt* H, int cap, int nband, int ndim,
                                                                                int dim_cap, int precision,
                                                                                cudaStream_t s);
// Solve nk <= cap k-points; psi_h: host array of nk device pointers (FP64 vectors at m*ldpsi, overwritten with the
// eigenvectors); eig: host nk x nband; iters: host nk (may be NULL).  Returns the iterations run.
int david_batch_solve(DavidBatchSolver& d, int nk, const int* iks, int spin, const double* const* precond_d,
                      void* const* psi_h, int ldpsi, double* eig, double thr, int maxiter, int* iters);

}  // namespace b200
