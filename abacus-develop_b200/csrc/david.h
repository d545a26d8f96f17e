// Block Davidson on the device: hsolver::DiagoDavid<T, DEVICE_GPU> (diago_david.h:19-84).
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <functional>
#include <memory>
#include <vector>

namespace b200 {

// H applied to vectors id_start..id_end of the block starting at x (vectors of length dim, stride dim);
// hx points at the output of vector id_start (the reference's HPsiFunc contract, diago_david.h:40-57).
using HPsiDevice = std::function<void(const void* x, void* hx, int nvec, int dim, int id_start, int id_end, cudaStream_t s)>;

struct DavidStats {
    int iters_low = 0;     // Davidson iterations in the low-precision stage (mixed only)
    int iters_fp64 = 0;    // Davidson iterations in FP64
    int hpsi_bands = 0;    // band applications of H (all stages)
};

// Per-iteration record of a solve: seconds since the solve began (taken when the iteration's eigenvalues
// reach the host, which every iteration does for its convergence test), the stage (0 = FP64, 1 = FP32)
// and the nband Ritz values.
struct DavidTrace {
    bool on = false;
    std::chrono::steady_clock::time_point t0;
    std::vector<double> t, eig;
    std::vector<int> stage;
    void reset() {
        t0 = std::chrono::steady_clock::now();
        t.clear();
        eig.clear();
        stage.clear();
    }
    void record(int st, const double* e, int n) {
        if (!on) return;
        t.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
        stage.push_back(st);
        eig.insert(eig.end(), e, e + n);
    }
};

struct DavidBase {
    virtual ~DavidBase() = default;
    // FP64 solve with a user H|psi> (psi: complex128, nband vectors at psi + m*ldpsi)
    virtual int diag(const HPsiDevice& f64, int ldpsi, void* psi, double* eig, double thr, int maxiter, int ntry_max,
                     int notconv_max) = 0;
    // Solve with built-in H|psi> callbacks for both precisions; precision 0 = FP64, 1 = mixed + FP64 refinement
    virtual int diag_hamilt(const HPsiDevice& f64, const HPsiDevice& f32, int precision, int ldpsi, void* psi,
                            double* eig, double thr, int maxiter, int ntry_max, int notconv_max) = 0;
    virtual const DavidStats& stats() const = 0;
    virtual void set_mixed_thr(double thr) = 0;
    // mixed precision only: subspace size factor (nbase_x = ndim * nband) of the FP32 stage (default: the
    // solver's own david_ndim); a smaller FP32 subspace means smaller FP64 subspace eigensolves there
    virtual void set_low_ndim(int ndim) = 0;
    virtual void set_reference_refresh(bool on) = 0;
    // FP64 subspace products: 0 = cuBLAS ZGEMM; 1 = the int8 tensor-core emulation in the FP64 refinement
    // sweep of a mixed solve; 2 = the int8 emulation in every FP64 stage (1, 2: for the product shapes on
    // which it is faster); 3 = the int8 emulation for every product of every FP64 stage
    virtual void set_fp64_gemm(int mode) = 0;
    virtual int precision() const = 0;
    // 0 = quiet; 1 = one line per Davidson iteration on stderr (iteration, basis size, unconverged bands,
    // largest eigenvalue change), the role of DiagoDavid's test_david levels (diago_david.cpp:53-58)
    virtual void set_verbosity(int level) = 0;
    // stream for all of the solver's work (default: the legacy default stream, as the reference)
    virtual void set_stream(cudaStream_t s) = 0;
    // solve vectors of length dim <= the construction dim next (another k-point of the same cell), with
    // that k-point's preconditioner; reuses every buffer
    virtual void retarget(int dim, const double* precond_d) = 0;
    // device memory held by the solver (bytes)
    virtual size_t device_bytes() const = 0;
    // per-iteration eigenvalue trace of the next solves (off by default)
    virtual DavidTrace& trace() = 0;
};

std::unique_ptr<DavidBase> make_david(int nband, int dim, int david_ndim, int precision, const double* precond_d);

}  // namespace b200
