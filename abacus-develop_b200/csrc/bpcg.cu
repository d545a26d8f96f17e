// Band-parallel preconditioned conjugate gradient on the device, restating hsolver::DiagoBPCG
// (module_hsolver/diago_bpcg.cpp:18-306) with its kernels line_minimize_with_block and calc_grad_with_block
// (module_hsolver/kernels/math_kernel_op.cpp:10-100, kernels/cuda/math_kernel_op.cu:75-300), FP64.
//
// One diag call:
//  * the Rayleigh-Ritz of psi (calc_hsub_with_block :215-233): H psi, hsub = psi^H H psi, all pairs
//    (Zheevd), psi and H psi rotated to the Ritz vectors;
//  * grad_old = 0, beta = +inf; up to 4 iterations (24 on the first SCF step), each: per band psi and
//    H psi normalised, eps = <psi|H psi>, r = H psi - eps psi, err = |r|, beta = sum |r|^2 / prec,
//    grad = -r / prec + beta / beta_old grad_old (k_bp_grad); grad projected off span(psi) (two GEMMs);
//    grad_old = grad; H grad; per band grad and H grad normalised and psi <- cos(theta) psi + sin(theta) grad
//    with theta = |atan(2 e1 / (e0 - e2))| / 2 (k_bp_line_min); psi and H psi made orthonormal through the
//    inverse of the upper Cholesky factor of psi^H psi, as the reference does (trtri, then a GEMM; here the
//    inverse comes from a triangular solve against I); on the first SCF step a Rayleigh-Ritz every 4 iterations;
//    stop once no band's err exceeds 1e-5;
//  * the exit Rayleigh-Ritz (:235-250) on the loop's H psi, psi rotated, its Ritz values returned.
// Per-band reductions run one CTA per band in a fixed order (deterministic); one host read of the nband
// residual norms per iteration drives the stop test, as the reference's test_error does.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <utility>
#include <vector>

#include "bpcg.h"
#include "common.h"
#include "linalg_status.h"

namespace b200 {

namespace {

constexpr int kBpThreads = 1024;

// sum over the CTA of K values per thread (fixed order); every thread gets the sums
template <int K> __device__ void bp_block_sum(double (&v)[K]) {
    __shared__ double part[K][kBpThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        if (lane == 0) part[k][warp] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int w = 0; w < kBpThreads / 32; ++w) s += part[k][w];
        v[k] = s;
    }
    __syncthreads();
}

// calc_grad_with_block_op for band blockIdx.x
__global__ void __launch_bounds__(kBpThreads) k_bp_grad(long n, const double* __restrict__ prec,
                                                        double2* __restrict__ psi, double2* __restrict__ hpsi,
                                                        double2* __restrict__ grad, const double2* __restrict__ grad_old,
                                                        double* __restrict__ beta, double* __restrict__ err) {
    const long off = long(blockIdx.x) * n;
    // the previous beta, read before any barrier: thread 0 overwrites it at the end, possibly before a slow
    // warp would otherwise have read it
    const double beta_old = beta[blockIdx.x];
    double2* p = psi + off;
    double2* hp = hpsi + off;
    double s[1] = {0.0};
#pragma unroll 4
    for (long i = threadIdx.x; i < n; i += kBpThreads) s[0] += p[i].x * p[i].x + p[i].y * p[i].y;
    bp_block_sum<1>(s);
    const double nrm = 1.0 / sqrt(s[0]);
    double e[1] = {0.0};
#pragma unroll 4
    for (long i = threadIdx.x; i < n; i += kBpThreads) {
        const double2 a = make_double2(p[i].x * nrm, p[i].y * nrm), b = make_double2(hp[i].x * nrm, hp[i].y * nrm);
        p[i] = a;
        hp[i] = b;
        e[0] += b.x * a.x + b.y * a.y;  // Re(hpsi * conj(psi))
    }
    bp_block_sum<1>(e);
    const double eps = e[0];
    double rb[2] = {0.0, 0.0};  // sum |r|^2, sum |r|^2 / prec
#pragma unroll 4
    for (long i = threadIdx.x; i < n; i += kBpThreads) {
        const double rx = hp[i].x - eps * p[i].x, ry = hp[i].y - eps * p[i].y;
        const double r2 = rx * rx + ry * ry;
        rb[0] += r2;
        rb[1] += r2 / prec[i];
    }
    bp_block_sum<2>(rb);
    const double ratio = rb[1] / beta_old;
    double2* g = grad + off;
    const double2* go = grad_old + off;
#pragma unroll 4
    for (long i = threadIdx.x; i < n; i += kBpThreads) {
        const double rx = hp[i].x - eps * p[i].x, ry = hp[i].y - eps * p[i].y;
        const double q = prec[i];
        g[i] = make_double2(-rx / q + ratio * go[i].x, -ry / q + ratio * go[i].y);
    }
    if (threadIdx.x == 0) {
        beta[blockIdx.x] = rb[1];
        err[blockIdx.x] = sqrt(rb[0]);
    }
}

// line_minimize_with_block_op for band blockIdx.x
__global__ void __launch_bounds__(kBpThreads) k_bp_line_min(long n, double2* __restrict__ grad,
                                                            double2* __restrict__ hgrad, double2* __restrict__ psi,
                                                            double2* __restrict__ hpsi) {
    const long off = long(blockIdx.x) * n;
    double2* g = grad + off;
    double2* hg = hgrad + off;
    double2* p = psi + off;
    double2* hp = hpsi + off;
    double s[1] = {0.0};
#pragma unroll 4
    for (long i = threadIdx.x; i < n; i += kBpThreads) s[0] += g[i].x * g[i].x + g[i].y * g[i].y;
    bp_block_sum<1>(s);
    const double nrm = 1.0 / sqrt(s[0]);
    double e[3] = {0.0, 0.0, 0.0};
#pragma unroll 4
    for (long i = threadIdx.x; i < n; i += kBpThreads) {
        const double2 a = make_double2(g[i].x * nrm, g[i].y * nrm), b = make_double2(hg[i].x * nrm, hg[i].y * nrm);
        g[i] = a;
        hg[i] = b;
        const double2 pp = p[i], hh = hp[i];
        e[0] += hh.x * pp.x + hh.y * pp.y;  // Re(hpsi conj(psi))
        e[1] += a.x * hh.x + a.y * hh.y;    // Re(grad conj(hpsi))
        e[2] += a.x * b.x + a.y * b.y;      // Re(grad conj(hgrad))
    }
    bp_block_sum<3>(e);
    const double theta = 0.5 * fabs(atan(2.0 * e[1] / (e[0] - e[2])));
    const double c = cos(theta), sn = sin(theta);
#pragma unroll 4
    for (long i = threadIdx.x; i < n; i += kBpThreads) {
        p[i] = make_double2(p[i].x * c + g[i].x * sn, p[i].y * c + g[i].y * sn);
        hp[i] = make_double2(hp[i].x * c + hg[i].x * sn, hp[i].y * c + hg[i].y * sn);
    }
}

__global__ void k_bp_fill(long n, double v, double* __restrict__ x) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) x[i] = v;
}

__global__ void k_bp_identity(int n, double2* __restrict__ a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x)
        a[i] = make_double2(i % n == i / n ? 1.0 : 0.0, 0.0);
}

class Bpcg : public BpcgBase {
  public:
    Bpcg(int nband, int nbasis, const double* precond_d) : nb_(nband), n_(nbasis) {
        B200_CHECK(nband > 0 && nbasis >= nband, kInvalidArgument, "need 0 < nband <= nbasis");
        B200_CUBLAS(cublasCreate(&cb_));
        B200_CUSOLVER(cusolverDnCreate(&cs_));
        set_handles_stream();
        const size_t blk = size_t(nb_) * n_;
        hpsi_.resize(blk);
        grad_.resize(blk);
        hgrad_.resize(blk);
        grad_old_.resize(blk);
        work_.resize(blk);
        hsub_.resize(size_t(nb_) * nb_);
        uinv_.resize(size_t(nb_) * nb_);
        prec_.resize(n_);
        eig_d_.resize(nb_);
        beta_.resize(nb_);
        err_.resize(nb_);
        info_.resize(1);
        B200_CUDA(cudaMemcpyAsync(prec_.ptr, precond_d, size_t(n_) * sizeof(double), cudaMemcpyDeviceToDevice, s_));
        int l1 = 0, l2 = 0;
        auto* H = reinterpret_cast<cuDoubleComplex*>(hsub_.ptr);
        B200_CUSOLVER(cusolverDnZheevd_bufferSize(cs_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb_, H, nb_,
                                                     eig_d_.ptr, &l1));
        B200_CUSOLVER(cusolverDnZpotrf_bufferSize(cs_, CUBLAS_FILL_MODE_UPPER, nb_, H, nb_, &l2));
        lwork_ = std::max(1, std::max(l1, l2));
        lw_.resize(size_t(lwork_));
        err_h_.assign(nb_, 0.0);
        B200_CUDA(cudaStreamSynchronize(s_));
    }
    ~Bpcg() override {
        if (cb_) cublasDestroy(cb_);
        if (cs_) cusolverDnDestroy(cs_);
    }

    int diag(const HPsiDevice& f, void* psi_v, double* eig, int scf_iter) override {
        auto* psi = static_cast<double2*>(psi_v);
        hpsi_bands_ = 0;
        rayleigh_ritz(f, psi, true, true);
        B200_CUDA(cudaMemsetAsync(grad_old_.ptr, 0, grad_old_.n * sizeof(double2), s_));
        k_bp_fill<<<1, 256, 0, s_>>>(nb_, std::numeric_limits<double>::infinity(), beta_.ptr);
        check_launch();
        const int max_iter = scf_iter > 1 ? kNline : kNline * 6;
        int ntry = 0;
        while (true) {
            ++ntry;
            k_bp_grad<<<nb_, kBpThreads, 0, s_>>>(n_, prec_.ptr, psi, hpsi_.ptr, grad_.ptr, grad_old_.ptr, beta_.ptr,
                                                  err_.ptr);
            check_launch();
            // orth_projection (:139-156): grad_i -= sum_k <psi_k|grad_i> psi_k
            gemm(CUBLAS_OP_C, nb_, nb_, n_, 1.0, psi, n_, grad_.ptr, n_, 0.0, hsub_.ptr, nb_);
            gemm(CUBLAS_OP_N, n_, nb_, nb_, -1.0, psi, n_, hsub_.ptr, nb_, 1.0, grad_.ptr, n_);
            B200_CUDA(cudaMemcpyAsync(grad_old_.ptr, grad_.ptr, grad_.n * sizeof(double2), cudaMemcpyDeviceToDevice, s_));
            apply_h(f, grad_.ptr, hgrad_.ptr);
            k_bp_line_min<<<nb_, kBpThreads, 0, s_>>>(n_, grad_.ptr, hgrad_.ptr, psi, hpsi_.ptr);
            check_launch();
            orth_cholesky(psi);
            if (scf_iter == 1 && ntry % kNline == 0) {
                check_info("Zpotrf (BPCG orthonormalisation)");
                rayleigh_ritz(f, psi, true, true);
            }
            int info = 0;
            B200_CUDA(cudaMemcpyAsync(err_h_.data(), err_.ptr, size_t(nb_) * sizeof(double), cudaMemcpyDeviceToHost, s_));
            B200_CUDA(cudaMemcpyAsync(&info, info_.ptr, sizeof(int), cudaMemcpyDeviceToHost, s_));
            B200_CUDA(cudaStreamSynchronize(s_));
            B200_CHECK(info == 0, kNumericalError,
                       "Zpotrf (BPCG orthonormalisation) failed, info " + std::to_string(info));
            bool above = false;
            for (int m = 0; m < nb_; ++m) {
                B200_CHECK(std::isfinite(err_h_[m]), kNumericalError, "non-finite residual (NaN/Inf in H|psi> or psi)");
                above = above || err_h_[m] > kThr;
            }
            if (!(ntry < max_iter && above)) break;
        }
        rayleigh_ritz(f, psi, false, false);
        B200_CUDA(cudaMemcpyAsync(eig, eig_d_.ptr, size_t(nb_) * sizeof(double), cudaMemcpyDeviceToHost, s_));
        B200_CUDA(cudaStreamSynchronize(s_));
        return ntry;
    }
    void set_stream(cudaStream_t s) override {
        B200_CUDA(cudaStreamSynchronize(s_));
        s_ = s;
        set_handles_stream();
    }
    double max_err() const override { return err_h_.empty() ? 0.0 : *std::max_element(err_h_.begin(), err_h_.end()); }
    int hpsi_bands() const override { return hpsi_bands_; }
    size_t device_bytes() const override {
        return (hpsi_.n + grad_.n + hgrad_.n + grad_old_.n + work_.n + hsub_.n + uinv_.n + lw_.n) * sizeof(double2) +
               (prec_.n + eig_d_.n + beta_.n + err_.n) * sizeof(double);
    }

  private:
    static constexpr int kNline = 4;       // nline (diago_bpcg.h)
    static constexpr double kThr = 1e-5;   // all_band_cg_thr (diago_bpcg.h)
    int nb_, n_;
    int hpsi_bands_ = 0;
    cudaStream_t s_ = 0;
    cublasHandle_t cb_ = nullptr;
    cusolverDnHandle_t cs_ = nullptr;
    DeviceArray<double2> hpsi_, grad_, hgrad_, grad_old_, work_, hsub_, uinv_, lw_;
    DeviceArray<double> prec_, eig_d_, beta_, err_;
    DeviceArray<int> info_;
    int lwork_ = 0;
    std::vector<double> err_h_;

    void set_handles_stream() {
        B200_CUBLAS(cublasSetStream(cb_, s_));
        B200_CUSOLVER(cusolverDnSetStream(cs_, s_));
    }
    void check_launch() {
        note_launch();
        B200_CUDA(cudaGetLastError());
    }
    void gemm(cublasOperation_t a, int m, int n, int k, double al_re, const double2* A, int lda, const double2* B,
              int ldb, double be_re, double2* C, int ldc) {
        const cuDoubleComplex al = make_cuDoubleComplex(al_re, 0.0), be = make_cuDoubleComplex(be_re, 0.0);
        B200_CUBLAS(cublasZgemm3m(cb_, a, CUBLAS_OP_N, m, n, k, &al, reinterpret_cast<const cuDoubleComplex*>(A), lda,
                                     reinterpret_cast<const cuDoubleComplex*>(B), ldb, &be,
                                     reinterpret_cast<cuDoubleComplex*>(C), ldc));
    }
    void apply_h(const HPsiDevice& f, const double2* x, double2* hx) {
        f(x, hx, nb_, n_, 0, nb_ - 1, s_);
        hpsi_bands_ += nb_;
    }
    void check_info(const char* what) {
        int info = 0;
        B200_CUDA(cudaMemcpyAsync(&info, info_.ptr, sizeof(int), cudaMemcpyDeviceToHost, s_));
        B200_CUDA(cudaStreamSynchronize(s_));
        B200_CHECK(info == 0, kNumericalError, std::string(what) + " failed, info " + std::to_string(info));
    }

    // calc_hsub_with_block (:215-233) when apply is set (H psi recomputed), calc_hsub_with_block_exit
    // (:235-250) otherwise; H psi is rotated with psi when rotate_h is set
    void rayleigh_ritz(const HPsiDevice& f, double2* psi, bool apply, bool rotate_h) {
        if (apply) apply_h(f, psi, hpsi_.ptr);
        gemm(CUBLAS_OP_C, nb_, nb_, n_, 1.0, psi, n_, hpsi_.ptr, n_, 0.0, hsub_.ptr, nb_);
        B200_CUDA(cudaMemsetAsync(info_.ptr, 0, sizeof(int), s_));
        B200_CUSOLVER(cusolverDnZheevd(cs_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb_,
                                          reinterpret_cast<cuDoubleComplex*>(hsub_.ptr), nb_, eig_d_.ptr,
                                          reinterpret_cast<cuDoubleComplex*>(lw_.ptr), lwork_, info_.ptr));
        gemm(CUBLAS_OP_N, n_, nb_, nb_, 1.0, psi, n_, hsub_.ptr, nb_, 0.0, work_.ptr, n_);
        B200_CUDA(cudaMemcpyAsync(psi, work_.ptr, work_.n * sizeof(double2), cudaMemcpyDeviceToDevice, s_));
        if (rotate_h) {
            gemm(CUBLAS_OP_N, n_, nb_, nb_, 1.0, hpsi_.ptr, n_, hsub_.ptr, nb_, 0.0, work_.ptr, n_);
            std::swap(hpsi_, work_);
        }
        check_info("Zheevd (BPCG subspace)");
    }

    // orth_cholesky (:86-106): psi^H psi = U^H U; psi <- psi U^-1, H psi <- H psi U^-1
    void orth_cholesky(double2* psi) {
        auto* S = reinterpret_cast<cuDoubleComplex*>(hsub_.ptr);
        // S = psi^H psi as a full GEMM (Zgemm3m runs faster than Zherk on these tall shapes; potrf reads the
        // upper triangle only)
        gemm(CUBLAS_OP_C, nb_, nb_, n_, 1.0, psi, n_, psi, n_, 0.0, hsub_.ptr, nb_);
        B200_CUDA(cudaMemsetAsync(info_.ptr, 0, sizeof(int), s_));
        B200_CUSOLVER(cusolverDnZpotrf(cs_, CUBLAS_FILL_MODE_UPPER, nb_, S, nb_,
                                          reinterpret_cast<cuDoubleComplex*>(lw_.ptr), lwork_, info_.ptr));
        // U^-1 (upper, exact zeros below) by a triangular solve against I, then two GEMMs: the tall
        // triangular solves psi U^-1, H psi U^-1 themselves run well below GEMM speed
        const cuDoubleComplex c1 = make_cuDoubleComplex(1.0, 0.0);
        k_bp_identity<<<ceil_div(long(nb_) * nb_, 256), 256, 0, s_>>>(nb_, uinv_.ptr);
        check_launch();
        B200_CUBLAS(cublasZtrsm(cb_, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, nb_,
                                   nb_, &c1, S, nb_, reinterpret_cast<cuDoubleComplex*>(uinv_.ptr), nb_));
        gemm(CUBLAS_OP_N, n_, nb_, nb_, 1.0, psi, n_, uinv_.ptr, nb_, 0.0, work_.ptr, n_);
        B200_CUDA(cudaMemcpyAsync(psi, work_.ptr, work_.n * sizeof(double2), cudaMemcpyDeviceToDevice, s_));
        gemm(CUBLAS_OP_N, n_, nb_, nb_, 1.0, hpsi_.ptr, n_, uinv_.ptr, nb_, 0.0, work_.ptr, n_);
        std::swap(hpsi_, work_);
        // info_ is read with the residual norms at the end of the iteration
    }
};

}  // namespace

std::unique_ptr<BpcgBase> make_bpcg(int nband, int nbasis, const double* precond_d) {
    B200_CHECK(precond_d != nullptr, kInvalidArgument, "NULL precondition");
    return std::make_unique<Bpcg>(nband, nbasis, precond_d);
}

}  // namespace b200
