// Davidson with subspace rotation on the device, restating hsolver::Diago_DavSubspace
// (module_hsolver/diago_dav_subspace.cpp:86-957), FP64.
//
// The iteration, as the reference's CPU branch runs it:
//  * diag (:804-838) tries diag_once up to six times (test_exit_cond :841-857); a try after the first, or
//    every try when need_subspace is set, starts with diagH_subspace (:860-957), a Rayleigh-Ritz of psi
//    with the generalised problem (psi^H H psi, psi^H psi);
//  * diag_once (:86-291): the Rayleigh-Ritz of the nband input vectors as a standard problem; then per
//    iteration the residuals of the unconverged Ritz pairs, divided by the preconditioner
//    0.5 (1 + x + sqrt(1 + (x - 1)^2)), x = |h_diag - lambda|, and normalised -- not orthogonalised
//    (cal_grad :294-428); their H|psi>; the new columns of hcc = B^H H B and scc = B^H B made Hermitian
//    (cal_elem :431-574); the lowest nband pairs of the generalised problem (hcc, scc) (diag_zhegvx
//    :577-706); a band converges when its eigenvalue moved less than thr (max(5 thr, 1e-5) for an empty
//    band); at convergence, when the basis would exceed nbase_x - 1, or at the last iteration, psi becomes
//    the Ritz vectors and the basis restarts from them (refresh :709-801).
//
// On the device: the subspace products are FP64 cuBLAS GEMMs (Zgemm3m), the residual scaling, the
// preconditioner and the normalisation are two fused kernels, the Hermitian fill of the new rows is one
// kernel over both matrices, and the generalised eigenproblem is cuSOLVER's divide-and-conquer Zhegvdx for
// the lowest nband pairs (the CPU branch's dngvx, range 'I').  The reference's GPU branch solves the
// standard problem hcc x = lambda x instead (dnevx_op, :608-626), ignoring scc; this solver follows the CPU
// branch, which is the method as written.  H is applied to the nband input vectors of the first step, not
// to all nbase_x (:127): the others are never read.  One eigenvalue copy to the host per iteration drives
// the convergence test; nothing is allocated inside a solve.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "common.h"
#include "linalg_status.h"
#include "dav_subspace.h"

namespace b200 {

namespace {

constexpr int kT = 256;
inline int grid_of(long n) {
    long b = (n + kT - 1) / kT;
    if (b > 148L * 8) b = 148L * 8;
    return int(b < 1 ? 1 : b);
}

// vc(:, m) = vcc(:nbase, unconv[m]); vcl(:, m) = -lambda vc(:, m); lam[m] = lambda = w[unconv[m]]
// (the compaction of cal_grad, :306-315, into separate arrays)
__global__ void k_ds_gather(int nbase, int nbase_x, int nc, const int* __restrict__ unconv,
                            const double2* __restrict__ vcc, const double* __restrict__ w, double2* __restrict__ vc,
                            double2* __restrict__ vcl, double* __restrict__ lam) {
    const long n = long(nbase) * nc;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int m = int(i / nbase);
        const int r = int(i - long(m) * nbase);
        const int col = unconv[m];
        const double e = w[col];
        const double2 v = vcc[long(col) * nbase_x + r];
        vc[long(m) * nbase_x + r] = v;
        vcl[long(m) * nbase_x + r] = make_double2(-e * v.x, -e * v.y);
        if (r == 0) lam[m] = e;
    }
}

__device__ __forceinline__ double ds_denominator(double h, double e) {
    const double x = fabs(h - e);
    return 0.5 * (1.0 + x + sqrt(1.0 + (x - 1.0) * (x - 1.0)));
}

__device__ double block_sum(double v) {
    __shared__ double part[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) part[0] = v;
    }
    __syncthreads();
    const double r = part[0];
    __syncthreads();
    return r;
}

// Preconditioned, normalised residual of column m (one block per column, :384-421): x / d(lambda_m), then
// divided by its 2-norm.  The first pass only reads (the norm), the second reads and writes.
constexpr int kDsNormThreads = 1024;
__global__ void __launch_bounds__(kDsNormThreads) k_ds_precond_normalise(long dim, double2* __restrict__ X,
                                                                          const double* __restrict__ pc,
                                                                          const double* __restrict__ lam) {
    double2* x = X + long(blockIdx.x) * dim;
    const double e = lam[blockIdx.x];
    double acc = 0.0;
#pragma unroll 4
    for (long g = threadIdx.x; g < dim; g += blockDim.x) {
        const double d = ds_denominator(pc[g], e);
        const double2 v = x[g];
        const double re = v.x / d, im = v.y / d;
        acc += re * re + im * im;
    }
    const double nrm = sqrt(block_sum(acc));
#pragma unroll 4
    for (long g = threadIdx.x; g < dim; g += blockDim.x) {
        const double d = ds_denominator(pc[g], e);
        const double2 v = x[g];
        x[g] = make_double2(v.x / d / nrm, v.y / d / nrm);
    }
}

// Hermitian completion of the rows last..nbase-1 of hcc and scc (:542-556): element (j, i), i < j, from
// (i, j) conjugated; the diagonal made real.  Column-major, leading dimension nbase_x.
__global__ void k_ds_herm_fill(int last, int nbase, int nbase_x, double2* __restrict__ hcc, double2* __restrict__ scc) {
    const long n = long(nbase - last) * nbase;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < n; t += long(gridDim.x) * blockDim.x) {
        const int j = last + int(t / nbase);
        const int i = int(t - long(j - last) * nbase);
        if (i < j) {
            const double2 h = hcc[long(j) * nbase_x + i], s = scc[long(j) * nbase_x + i];
            hcc[long(i) * nbase_x + j] = make_double2(h.x, -h.y);
            scc[long(i) * nbase_x + j] = make_double2(s.x, -s.y);
        } else if (i == j) {
            hcc[long(j) * nbase_x + j].y = 0.0;
            scc[long(j) * nbase_x + j].y = 0.0;
        }
    }
}

// refresh (:709-801): the leading nband block of hcc / scc / vcc becomes diag(e) / I / I
__global__ void k_ds_refresh_diag(int nband, int nbase_x, const double* __restrict__ e, double2* __restrict__ hcc,
                                  double2* __restrict__ scc, double2* __restrict__ vcc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nband; i += gridDim.x * blockDim.x) {
        const long d = long(i) * nbase_x + i;
        hcc[d] = make_double2(e[i], 0.0);
        scc[d] = make_double2(1.0, 0.0);
        vcc[d] = make_double2(1.0, 0.0);
    }
}

// diag_zhegvx with is_subspace on the first step (:688-699): the eigenvalues are the real diagonal of hcc and
// vcc(m, m) = 1 (the rest of its leading block is zero there)
__global__ void k_ds_diag_as_eig(int nband, int nbase_x, const double2* __restrict__ hcc, double* __restrict__ w,
                                 double2* __restrict__ vcc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nband; i += gridDim.x * blockDim.x) {
        w[i] = hcc[long(i) * nbase_x + i].x;
        vcc[long(i) * nbase_x + i] = make_double2(1.0, 0.0);
    }
}

class DavSubspace : public DavSubspaceBase {
  public:
    DavSubspace(int nband, int dim, int ndim, double thr, int maxiter, bool need_subspace, const double* precond_d)
        : nb_(nband), dim_(dim), nx_(ndim * nband), thr_(thr), maxiter_(maxiter), subspace_(need_subspace) {
        B200_CHECK(ndim > 1 && nband > 0 && ndim * nband < dim, kInvalidArgument,
                   "need david_ndim > 1 and david_ndim*nband < dim");
        B200_CHECK(maxiter > 0 && thr > 0.0, kInvalidArgument, "need diag_nmax > 0 and diag_thr > 0");
        B200_CUBLAS(cublasCreate(&cb_));
        B200_CUSOLVER(cusolverDnCreate(&cs_));
        set_handles_stream();
        const size_t nx = size_t(nx_);
        psi_iter_.resize(nx * dim_);
        hphi_.resize(nx * dim_);
        hcc_.resize(nx * nx);
        scc_.resize(nx * nx);
        vcc_.resize(nx * nx);
        a_.resize(nx * nx);
        b_.resize(nx * nx);
        vc_.resize(nx * nb_);
        vcl_.resize(nx * nb_);
        lam_.resize(nb_);
        w_.resize(nx);
        pc_.resize(dim_);
        unconv_d_.resize(nb_);
        info_.resize(2);
        B200_CUDA(cudaMemcpyAsync(pc_.ptr, precond_d, size_t(dim_) * sizeof(double), cudaMemcpyDeviceToDevice, s_));
        B200_CUDA(cudaMemsetAsync(psi_iter_.ptr, 0, psi_iter_.n * sizeof(double2), s_));
        B200_CUDA(cudaMemsetAsync(hphi_.ptr, 0, hphi_.n * sizeof(double2), s_));
        // workspace of every eigensolve a solve makes, so that it allocates nothing
        auto* A = reinterpret_cast<cuDoubleComplex*>(a_.ptr);
        auto* B = reinterpret_cast<cuDoubleComplex*>(b_.ptr);
        int l1 = 0, l2 = 0, l3 = 0, meig = 0;
        B200_CUSOLVER(cusolverDnZheevd_bufferSize(cs_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb_, A, nx_,
                                                     w_.ptr, &l1));
        B200_CUSOLVER(cusolverDnZhegvdx_bufferSize(cs_, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                                      CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_UPPER, nx_, A, nx_, B, nx_,
                                                      0.0, 0.0, 1, nb_, &meig, w_.ptr, &l2));
        B200_CUSOLVER(cusolverDnZhegvd_bufferSize(cs_, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                                     CUBLAS_FILL_MODE_UPPER, nb_, A, nb_, B, nb_, w_.ptr, &l3));
        lwork_ = std::max(1, std::max(l1, std::max(l2, l3)));
        work_.resize(size_t(lwork_));
        e_iter_.assign(nx_, 0.0);
        unconv_.assign(nb_, 0);
        B200_CUDA(cudaStreamSynchronize(s_));
    }
    ~DavSubspace() override {
        if (cb_) cublasDestroy(cb_);
        if (cs_) cusolverDnDestroy(cs_);
    }

    int diag(const HPsiDevice& f, void* psi_v, int ldpsi, double* eig, const int* occupied, bool scf) override {
        B200_CHECK(ldpsi >= dim_, kInvalidArgument, "psi_in_dmax must be >= dim");
        auto* psi = static_cast<double2*>(psi_v);
        occ_.assign(nb_, 1);
        if (occupied)
            for (int m = 0; m < nb_; ++m) occ_[m] = occupied[m] != 0;
        hpsi_bands_ = 0;
        notconv_ = 0;
        // a fresh subspace, as a newly constructed Diago_DavSubspace has (:14-83)
        B200_CUDA(cudaMemsetAsync(hcc_.ptr, 0, hcc_.n * sizeof(double2), s_));
        B200_CUDA(cudaMemsetAsync(scc_.ptr, 0, scc_.n * sizeof(double2), s_));
        B200_CUDA(cudaMemsetAsync(vcc_.ptr, 0, vcc_.n * sizeof(double2), s_));
        int total = 0, ntry = 0;
        while (true) {
            if (subspace_ || ntry > 0) diagh_subspace(f, psi, ldpsi, eig);
            total += diag_once(f, psi, ldpsi, eig);
            ++ntry;
            const bool f1 = ntry <= 5, f2 = !scf && notconv_ > 0, f3 = scf && notconv_ > 5;
            if (!(f1 && (f2 || f3))) break;
        }
        B200_CUDA(cudaStreamSynchronize(s_));
        return total;
    }
    void set_stream(cudaStream_t s) override {
        B200_CUDA(cudaStreamSynchronize(s_));
        s_ = s;
        set_handles_stream();
    }
    void set_verbosity(int level) override { verbosity_ = level; }
    int notconv() const override { return notconv_; }
    int hpsi_bands() const override { return hpsi_bands_; }
    size_t device_bytes() const override {
        return (psi_iter_.n + hphi_.n + hcc_.n + scc_.n + vcc_.n + a_.n + b_.n + vc_.n + vcl_.n + work_.n) *
                   sizeof(double2) +
               (lam_.n + w_.n + pc_.n) * sizeof(double) + (unconv_d_.n + info_.n) * sizeof(int);
    }

  private:
    int nb_, dim_, nx_;
    double thr_;
    int maxiter_;
    bool subspace_;
    int verbosity_ = 0;
    int notconv_ = 0, hpsi_bands_ = 0;
    cudaStream_t s_ = 0;
    cublasHandle_t cb_ = nullptr;
    cusolverDnHandle_t cs_ = nullptr;
    DeviceArray<double2> psi_iter_, hphi_, hcc_, scc_, vcc_, a_, b_, vc_, vcl_, work_;
    DeviceArray<double> lam_, w_, pc_;
    DeviceArray<int> unconv_d_, info_;
    int lwork_ = 0;
    std::vector<double> e_iter_;
    std::vector<int> unconv_, occ_;

    void set_handles_stream() {
        B200_CUBLAS(cublasSetStream(cb_, s_));
        B200_CUSOLVER(cusolverDnSetStream(cs_, s_));
    }
    void check_launch() {
        note_launch();
        B200_CUDA(cudaGetLastError());
    }
    // C = al op(A) B + be C, FP64 complex
    void gemm(cublasOperation_t a, int m, int n, int k, double al_re, const double2* A, int lda, const double2* B,
              int ldb, double be_re, double2* C, int ldc) {
        if (m <= 0 || n <= 0) return;
        const cuDoubleComplex al = make_cuDoubleComplex(al_re, 0.0), be = make_cuDoubleComplex(be_re, 0.0);
        B200_CUBLAS(cublasZgemm3m(cb_, a, CUBLAS_OP_N, m, n, k, &al, reinterpret_cast<const cuDoubleComplex*>(A), lda,
                                     reinterpret_cast<const cuDoubleComplex*>(B), ldb, &be,
                                     reinterpret_cast<cuDoubleComplex*>(C), ldc));
    }
    void apply_h(const HPsiDevice& f, double2* x_base, double2* hx, int i0, int i1) {
        f(x_base, hx, nx_, dim_, i0, i1, s_);
        hpsi_bands_ += i1 - i0 + 1;
    }
    // eigenvalues w[:nband] to the host and the solver's info word checked
    void fetch_eigenvalues(const char* what) {
        int info = 0;
        B200_CUDA(cudaMemcpyAsync(e_iter_.data(), w_.ptr, size_t(nb_) * sizeof(double), cudaMemcpyDeviceToHost, s_));
        B200_CUDA(cudaMemcpyAsync(&info, info_.ptr, sizeof(int), cudaMemcpyDeviceToHost, s_));
        B200_CUDA(cudaStreamSynchronize(s_));
        B200_CHECK(info == 0, kNumericalError,
                   std::string(what) + " failed, info " + std::to_string(info) +
                       (info > 0 ? " (overlap matrix not positive definite: dependent search directions)" : ""));
        for (int m = 0; m < nb_; ++m)
            B200_CHECK(std::isfinite(e_iter_[m]), kNumericalError, "non-finite eigenvalue (NaN/Inf in H|psi> or psi)");
    }

    // cal_elem (:431-574): hcc(:nbase+nc, nbase:nbase+nc) = B^H H B_new, scc likewise, rows completed
    int cal_elem(int nbase, int nc) {
        gemm(CUBLAS_OP_C, nbase + nc, nc, dim_, 1.0, psi_iter_.ptr, dim_, hphi_.ptr + size_t(nbase) * dim_, dim_, 0.0,
             hcc_.ptr + size_t(nbase) * nx_, nx_);
        gemm(CUBLAS_OP_C, nbase + nc, nc, dim_, 1.0, psi_iter_.ptr, dim_, psi_iter_.ptr + size_t(nbase) * dim_, dim_, 0.0,
             scc_.ptr + size_t(nbase) * nx_, nx_);
        k_ds_herm_fill<<<grid_of(long(nc) * (nbase + nc)), kT, 0, s_>>>(nbase, nbase + nc, nx_, hcc_.ptr, scc_.ptr);
        check_launch();
        return nbase + nc;
    }

    // diag_zhegvx (:577-706): the lowest nband pairs of (hcc, scc) on copies of their leading nbase block
    void eigensolve(int nbase, bool init) {
        auto* A = reinterpret_cast<cuDoubleComplex*>(a_.ptr);
        auto* B = reinterpret_cast<cuDoubleComplex*>(b_.ptr);
        B200_CUDA(cudaMemsetAsync(info_.ptr, 0, sizeof(int), s_));
        if (init && subspace_) {
            k_ds_diag_as_eig<<<grid_of(nb_), kT, 0, s_>>>(nb_, nx_, hcc_.ptr, w_.ptr, vcc_.ptr);
            check_launch();
            fetch_eigenvalues("subspace diagonal");
            return;
        }
        const size_t pitch = size_t(nx_) * sizeof(double2);
        B200_CUDA(cudaMemcpy2DAsync(a_.ptr, pitch, hcc_.ptr, pitch, size_t(nbase) * sizeof(double2), nbase,
                                    cudaMemcpyDeviceToDevice, s_));
        if (init) {
            // standard problem of the nband input vectors (dnevx, :646-655); nbase == nband here
            B200_CUSOLVER(cusolverDnZheevd(cs_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nbase, A, nx_,
                                              w_.ptr, reinterpret_cast<cuDoubleComplex*>(work_.ptr), lwork_, info_.ptr));
        } else {
            B200_CUDA(cudaMemcpy2DAsync(b_.ptr, pitch, scc_.ptr, pitch, size_t(nbase) * sizeof(double2), nbase,
                                        cudaMemcpyDeviceToDevice, s_));
            int meig = 0;
            B200_CUSOLVER(cusolverDnZhegvdx(cs_, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I,
                                               CUBLAS_FILL_MODE_UPPER, nbase, A, nx_, B, nx_, 0.0, 0.0, 1, nb_, &meig,
                                               w_.ptr, reinterpret_cast<cuDoubleComplex*>(work_.ptr), lwork_,
                                               info_.ptr));
        }
        B200_CUDA(cudaMemcpy2DAsync(vcc_.ptr, pitch, a_.ptr, pitch, size_t(nbase) * sizeof(double2), nb_,
                                    cudaMemcpyDeviceToDevice, s_));
        fetch_eigenvalues(init ? "Zheevd" : "Zhegvdx");
    }

    // cal_grad (:294-428): preconditioned, normalised residuals of the nc unconverged bands as basis
    // columns nbase..nbase+nc-1, and their H|psi>
    void cal_grad(const HPsiDevice& f, int nbase, int nc) {
        B200_CUDA(cudaMemcpyAsync(unconv_d_.ptr, unconv_.data(), size_t(nc) * sizeof(int), cudaMemcpyHostToDevice, s_));
        k_ds_gather<<<grid_of(long(nbase) * nc), kT, 0, s_>>>(nbase, nx_, nc, unconv_d_.ptr, vcc_.ptr, w_.ptr, vc_.ptr,
                                                              vcl_.ptr, lam_.ptr);
        check_launch();
        double2* X = psi_iter_.ptr + size_t(nbase) * dim_;
        gemm(CUBLAS_OP_N, dim_, nc, nbase, 1.0, psi_iter_.ptr, dim_, vcl_.ptr, nx_, 0.0, X, dim_);
        gemm(CUBLAS_OP_N, dim_, nc, nbase, 1.0, hphi_.ptr, dim_, vc_.ptr, nx_, 1.0, X, dim_);
        k_ds_precond_normalise<<<nc, kDsNormThreads, 0, s_>>>(dim_, X, pc_.ptr, lam_.ptr);
        check_launch();
        apply_h(f, psi_iter_.ptr, hphi_.ptr + size_t(nbase) * dim_, nbase, nbase + nc - 1);
    }

    // refresh (:709-801): hphi(:, :nband) rotated to the Ritz vectors (through the scratch columns
    // nband..2 nband-1 of psi_iter, as the reference), the leading blocks reset
    void refresh(int nbase) {
        gemm(CUBLAS_OP_N, dim_, nb_, nbase, 1.0, hphi_.ptr, dim_, vcc_.ptr, nx_, 0.0, psi_iter_.ptr + size_t(nb_) * dim_,
             dim_);
        B200_CUDA(cudaMemcpyAsync(hphi_.ptr, psi_iter_.ptr + size_t(nb_) * dim_, size_t(nb_) * dim_ * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, s_));
        const size_t pitch = size_t(nx_) * sizeof(double2), width = size_t(nb_) * sizeof(double2);
        B200_CUDA(cudaMemset2DAsync(hcc_.ptr, pitch, 0, width, nb_, s_));
        B200_CUDA(cudaMemset2DAsync(scc_.ptr, pitch, 0, width, nb_, s_));
        B200_CUDA(cudaMemset2DAsync(vcc_.ptr, pitch, 0, width, nb_, s_));
        // the eigenvalues of the exit step are w[:nband] (eigenvalue_in_hsolver there)
        k_ds_refresh_diag<<<grid_of(nb_), kT, 0, s_>>>(nb_, nx_, w_.ptr, hcc_.ptr, scc_.ptr, vcc_.ptr);
        check_launch();
    }

    int diag_once(const HPsiDevice& f, double2* psi, int ldpsi, double* eig) {
        const size_t row = size_t(dim_) * sizeof(double2);
        B200_CUDA(cudaMemcpy2DAsync(psi_iter_.ptr, row, psi, size_t(ldpsi) * sizeof(double2), row, nb_,
                                    cudaMemcpyDeviceToDevice, s_));
        apply_h(f, psi_iter_.ptr, hphi_.ptr, 0, nb_ - 1);
        int nbase = cal_elem(0, nb_);
        eigensolve(nbase, true);
        for (int m = 0; m < nb_; ++m) eig[m] = e_iter_[m];
        notconv_ = nb_;
        for (int m = 0; m < nb_; ++m) unconv_[m] = m;
        const double empty_thr = std::max(thr_ * 5.0, 1e-5);
        int iter = 0;
        while (true) {
            ++iter;
            cal_grad(f, nbase, notconv_);
            nbase = cal_elem(nbase, notconv_);
            eigensolve(nbase, false);
            notconv_ = 0;
            double dmax = 0.0;
            for (int m = 0; m < nb_; ++m) {
                const double de = std::fabs(e_iter_[m] - eig[m]);
                dmax = std::max(dmax, de);
                if (!(de < (occ_[m] ? thr_ : empty_thr))) unconv_[notconv_++] = m;
                eig[m] = e_iter_[m];
            }
            if (verbosity_ > 0)
                std::fprintf(stderr, "[dav_subspace] iter %3d nbase %4d notconv %4d max|dE| %.3e\n", iter, nbase,
                             notconv_, dmax);
            if (notconv_ == 0 || nbase + notconv_ + 1 > nx_ || iter == maxiter_) {
                B200_CUDA(cudaMemsetAsync(psi, 0, size_t(nb_) * ldpsi * sizeof(double2), s_));
                gemm(CUBLAS_OP_N, dim_, nb_, nbase, 1.0, psi_iter_.ptr, dim_, vcc_.ptr, nx_, 0.0, psi, ldpsi);
                B200_CUDA(cudaMemcpy2DAsync(psi_iter_.ptr, row, psi, size_t(ldpsi) * sizeof(double2), row, nb_,
                                            cudaMemcpyDeviceToDevice, s_));
                refresh(nbase);
                nbase = nb_;
                if (notconv_ == 0 || iter == maxiter_) break;
            }
        }
        return iter;
    }

    // diagH_subspace (:860-957): Rayleigh-Ritz of psi with the generalised problem of its nband vectors,
    // all pairs; psi <- psi V, eig <- the Ritz values.  psi is staged in psi_iter (stride dim) for H.
    void diagh_subspace(const HPsiDevice& f, double2* psi, int ldpsi, double* eig) {
        const size_t row = size_t(dim_) * sizeof(double2);
        B200_CUDA(cudaMemcpy2DAsync(psi_iter_.ptr, row, psi, size_t(ldpsi) * sizeof(double2), row, nb_,
                                    cudaMemcpyDeviceToDevice, s_));
        apply_h(f, psi_iter_.ptr, hphi_.ptr, 0, nb_ - 1);
        gemm(CUBLAS_OP_C, nb_, nb_, dim_, 1.0, psi_iter_.ptr, dim_, hphi_.ptr, dim_, 0.0, a_.ptr, nb_);
        gemm(CUBLAS_OP_C, nb_, nb_, dim_, 1.0, psi_iter_.ptr, dim_, psi_iter_.ptr, dim_, 0.0, b_.ptr, nb_);
        B200_CUDA(cudaMemsetAsync(info_.ptr, 0, sizeof(int), s_));
        B200_CUSOLVER(cusolverDnZhegvd(cs_, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb_,
                                          reinterpret_cast<cuDoubleComplex*>(a_.ptr), nb_,
                                          reinterpret_cast<cuDoubleComplex*>(b_.ptr), nb_, w_.ptr,
                                          reinterpret_cast<cuDoubleComplex*>(work_.ptr), lwork_, info_.ptr));
        gemm(CUBLAS_OP_N, dim_, nb_, nb_, 1.0, psi_iter_.ptr, dim_, a_.ptr, nb_, 0.0, psi, ldpsi);
        fetch_eigenvalues("Zhegvd (subspace rotation)");
        for (int m = 0; m < nb_; ++m) eig[m] = e_iter_[m];
    }
};

}  // namespace

std::unique_ptr<DavSubspaceBase> make_dav_subspace(int nband, int dim, int david_ndim, double diag_thr, int diag_nmax,
                                                   bool need_subspace, const double* precond_d) {
    B200_CHECK(precond_d != nullptr, kInvalidArgument, "NULL precondition");
    return std::make_unique<DavSubspace>(nband, dim, david_ndim, diag_thr, diag_nmax, need_subspace, precond_d);
}

}  // namespace b200
