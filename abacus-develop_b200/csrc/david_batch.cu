// Davidson of all k-points of a pool in lock-step: the k loop of HSolverPW::solve (hsolver_pw.cpp:240-270)
// with every k-point's DiagoDavid iteration (diago_david.cpp:151-341) advanced together, so that each phase of
// an iteration is one launch (or one batched library call) for all k instead of one per k-point:
//   * H|psi> of the new vectors of every k-point: Hamilt::hpsi_kbatch (the local pass in one launch per FFT
//     pass for all k);
//   * the residuals, projections, Gram matrices and subspace rows: strided-batched ZGEMMs over k;
//   * Cholesky-QR of the new blocks: batched ZPOTRF + ZTRSM;
//   * the subspace eigensolves: one batched Hermitian eigensolver call (cusolverDnXsyevBatched);
//   * the convergence test |d lambda| < thr per band: on the device, one small read per iteration.
// The k-points differ in their numbers of unconverged bands; every k-point adds the same number nc (the
// largest) of new columns, the surplus ones "dummy": zero vectors, which the Gram matrix sees as unit
// columns and the subspace matrix as an isolated eigenvalue far above the band energies (kDummyDiag), so they
// never enter the lowest nband Ritz pairs.  Vectors are padded with zeros to the largest npw of the batch.
// FP64 throughout; differences from one DiagoDavid per k-point (same mathematics): a block Gram-Schmidt +
// Cholesky-QR orthogonalisation (twice) instead of the per-vector SchmidtOrth, S = I, and a common restart
// (refresh) of all k-points whenever the common basis would overflow david_ndim * nband.
#include <algorithm>
#include <vector>

#include "capi_guard.h"
#include "../../include/abacus_b200.h"
#include "capi_handles.h"
#include "linalg_status.h"

namespace b200 {
namespace {

constexpr int kBT = 256;
constexpr double kDummyDiag = 1.0e3;  // Ry: far above any band energy, so dummy columns stay out of the lowest pairs

inline int blocks_of(long n) {
    long b = (n + kBT - 1) / kBT;
    if (b > 148L * 16) b = 148L * 16;
    return int(b < 1 ? 1 : b);
}

// basis_k[:, m] = psi_k[:, m] for g < dim_k, 0 beyond (psi_k = psi[k], pitch ldpsi)
__global__ void k_load_start(int nk, int nband, int ld, long sb, const int* __restrict__ dims,
                             const double2* const* __restrict__ psi, int ldpsi, double2* __restrict__ basis) {
    const long total = long(nk) * nband * ld;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int g = int(i % ld);
        const int m = int((i / ld) % nband);
        const int k = int(i / (long(ld) * nband));
        basis[k * sb + long(m) * ld + g] = g < dims[k] ? psi[k][long(m) * ldpsi + g] : make_double2(0.0, 0.0);
    }
}

// residual coefficients of the new block: vc(:, m) = vcc(:nbase, unconv[m]), vcl = -lambda vc for the
// unconverged bands m < notconv_k, zero for the dummy columns notconv_k <= m < nc; marks the new columns
// of the basis (real or dummy)
__global__ void k_gather_batch(int nk, int nbase, int nbase_x, int nband, int nc, const int* __restrict__ notconv,
                               const int* __restrict__ unconv, const double2* __restrict__ vcc,
                               const double* __restrict__ w, double2* __restrict__ vc, double2* __restrict__ vcl,
                               unsigned char* __restrict__ colmask) {
    const long total = long(nk) * nc * nbase;
    const long sh = long(nbase_x) * nbase_x, sv = long(nbase_x) * nband;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int r = int(i % nbase);
        const int m = int((i / nbase) % nc);
        const int k = int(i / (long(nbase) * nc));
        double2 v = make_double2(0.0, 0.0), vl = v;
        if (m < notconv[k]) {
            const int col = unconv[k * nband + m];
            v = vcc[k * sh + long(col) * nbase_x + r];
            const double lam = w[long(k) * nbase_x + col];
            vl = make_double2(-lam * v.x, -lam * v.y);
        }
        vc[k * sv + long(m) * nbase_x + r] = v;
        vcl[k * sv + long(m) * nbase_x + r] = vl;
        if (r == 0) colmask[long(k) * nbase_x + nbase + m] = m < notconv[k] ? 1 : 0;
    }
}

// X_k(:, m) /= precondition_k (the reference's vector_div_vector_op), zero in the padding rows
__global__ void k_precond_batch(int nk, int nc, int ld, long sb, long off, const int* __restrict__ dims,
                                const double* __restrict__ pc, double2* __restrict__ basis) {
    const long total = long(nk) * nc * ld;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int g = int(i % ld);
        const int m = int((i / ld) % nc);
        const int k = int(i / (long(ld) * nc));
        double2* x = basis + k * sb + off + long(m) * ld + g;
        if (g < dims[k]) {
            const double p = pc[long(k) * ld + g];
            *x = make_double2(x->x / p, x->y / p);
        } else {
            *x = make_double2(0.0, 0.0);
        }
    }
}

// Gram matrices of the new blocks: the dummy columns (m >= notconv_k) become unit columns, so the Cholesky
// factor keeps them apart and they stay zero through X U^-1
__global__ void k_fix_gram(int nk, int nc, int ldg, const int* __restrict__ notconv, double2* __restrict__ gram) {
    const long total = long(nk) * nc * nc;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int i = int(t % nc);
        const int j = int((t / nc) % nc);
        const int k = int(t / (long(nc) * nc));
        if (i >= notconv[k] || j >= notconv[k])
            gram[long(k) * ldg * ldg + long(j) * ldg + i] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    }
}

__global__ void k_fill_ptrs(int nk, double2* base, long stride, long off, double2** out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nk) out[k] = base + k * stride + off;
}

// eigensolver input: the leading n x n block of each hcc (lower triangle), compact with lda = n; rows and
// columns of dummy basis vectors become kDummyDiag on the diagonal and 0 elsewhere; a non-finite entry of the
// lower triangle sets bad[k] (that matrix is then replaced by I, so the eigensolver never sees NaN)
__global__ void k_eig_in(int nk, int n, int nbase_x, const unsigned char* __restrict__ colmask,
                         const double2* __restrict__ hcc, double2* __restrict__ a, int* __restrict__ bad) {
    const long total = long(nk) * n * n;
    const long sh = long(nbase_x) * nbase_x;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int i = int(t % n);
        const int j = int((t / n) % n);
        const int k = int(t / (long(n) * n));
        double2 v = make_double2(0.0, 0.0);
        if (i >= j) {
            const bool real = colmask[long(k) * nbase_x + i] && colmask[long(k) * nbase_x + j];
            if (real) {
                v = hcc[k * sh + long(j) * nbase_x + i];
                if (!(isfinite(v.x) && isfinite(v.y))) atomicOr(bad + k, 1);
            } else if (i == j) {
                v = make_double2(kDummyDiag, 0.0);
            }
        }
        a[t] = v;
    }
}
__global__ void k_eig_guard(int nk, int n, const int* __restrict__ bad, double2* __restrict__ a) {
    const long total = long(nk) * n * n;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int k = int(t / (long(n) * n));
        if (bad[k]) {
            const int i = int(t % n), j = int((t / n) % n);
            a[t] = make_double2(i == j ? 1.0 : 0.0, 0.0);
        }
    }
}

// lowest nband eigenpairs of each matrix -> vcc(:, :nband) (rows >= n zeroed) and w(:nband)
__global__ void k_eig_out(int nk, int n, int nbase_x, int nband, const double2* __restrict__ a,
                          const double* __restrict__ wa, double2* __restrict__ vcc, double* __restrict__ w) {
    const long total = long(nk) * nband * nbase_x;
    const long sh = long(nbase_x) * nbase_x;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int r = int(t % nbase_x);
        const int m = int((t / nbase_x) % nband);
        const int k = int(t / (long(nbase_x) * nband));
        vcc[k * sh + long(m) * nbase_x + r] = r < n ? a[long(k) * n * n + long(m) * n + r] : make_double2(0.0, 0.0);
        if (r == 0) w[long(k) * nbase_x + m] = wa[long(k) * n + m];
    }
}

// the convergence test of every k-point (diago_david.cpp:273): band m is unconverged while |w - w_old| >= thr;
// one warp per k-point compacts its unconverged bands; status[0] = largest notconv, status[1] = k-points with
// unconverged bands, status[2] = any non-finite eigenvalue
__global__ void k_converge(int nk, int nband, int nbase_x, double thr, int iter, const double* __restrict__ w,
                           double* __restrict__ e_old, int* __restrict__ notconv, int* __restrict__ unconv,
                           int* __restrict__ iters, int* __restrict__ status) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= nk) return;
    const int k = warp;
    int count = 0;
    for (int m0 = 0; m0 < nband; m0 += 32) {
        const int m = m0 + lane;
        bool un = false;
        if (m < nband) {
            const double e = w[long(k) * nbase_x + m];
            const double de = fabs(e - e_old[long(k) * nband + m]);
            un = !(de < thr);
            if (!isfinite(e)) atomicOr(status + 2, 1);
            e_old[long(k) * nband + m] = e;
        }
        const unsigned b = __ballot_sync(0xffffffffu, un);
        if (un) unconv[k * nband + count + __popc(b & ((1u << lane) - 1u))] = m;
        count += __popc(b);
    }
    if (lane == 0) {
        notconv[k] = count;
        if (count > 0) {
            atomicMax(status + 0, count);
            atomicAdd(status + 1, 1);
            iters[k] = iter;
        }
    }
}

// restart: basis(:, :nband) <- newv, hp(:, :nband) <- newh; hcc = diag(e), vcc = I (first nband), masks reset
__global__ void k_restart(int nk, int nband, int ld, int nbase_x, long sb, const double2* __restrict__ newv,
                          const double2* __restrict__ newh, double2* __restrict__ basis, double2* __restrict__ hp) {
    const long total = long(nk) * nband * ld;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int g = int(i % ld);
        const int m = int((i / ld) % nband);
        const int k = int(i / (long(ld) * nband));
        basis[k * sb + long(m) * ld + g] = newv[i];
        hp[k * sb + long(m) * ld + g] = newh[i];
    }
}
__global__ void k_restart_small(int nk, int nband, int nbase_x, const double* __restrict__ e_old, double2* __restrict__ hcc,
                                double2* __restrict__ vcc, unsigned char* __restrict__ colmask) {
    const long sh = long(nbase_x) * nbase_x;
    const long total = long(nk) * nbase_x;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int i = int(t % nbase_x);
        const int k = int(t / nbase_x);
        colmask[t] = i < nband ? 1 : 0;
        if (i < nband) {
            hcc[k * sh + long(i) * nbase_x + i] = make_double2(e_old[long(k) * nband + i], 0.0);
            vcc[k * sh + long(i) * nbase_x + i] = make_double2(1.0, 0.0);
        }
    }
}

__global__ void k_info_max(int nk, const int* __restrict__ info, int* __restrict__ out) {
    for (int k = threadIdx.x; k < nk; k += blockDim.x)
        if (info[k] != 0) atomicOr(out, 1);
}

__global__ void k_mask_start(int nk, int nband, int nbase_x, unsigned char* __restrict__ colmask) {
    const long total = long(nk) * nbase_x;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x)
        colmask[t] = int(t % nbase_x) < nband ? 1 : 0;
}

// psi_k(:, m) <- v_k(:, m) (pitch ld) for g < ld, 0 for ld <= g < ldpsi
__global__ void k_store_psi(int nk, int nband, int ld, int ldpsi, const double2* __restrict__ v,
                            double2* const* __restrict__ psi) {
    const long total = long(nk) * nband * ldpsi;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int g = int(i % ldpsi);
        const int m = int((i / ldpsi) % nband);
        const int k = int(i / (long(ldpsi) * nband));
        psi[k][long(m) * ldpsi + g] = g < ld ? v[(long(k) * nband + m) * ld + g] : make_double2(0.0, 0.0);
    }
}

class DavidBatch {
  public:
    DavidBatch(Hamilt* H, int nk, const int* iks, int spin, int nband, int ndim, const double* const* precond_d,
               cudaStream_t s)
        : H_(H), nk_(nk), iks_(iks, iks + nk), spin_(spin), nband_(nband), nbase_x_(ndim * nband), s_(s) {
        B200_CHECK(nk >= 1 && nk <= kMaxKBatch, kInvalidArgument, "1..128 k-points per batch");
        B200_CHECK(ndim >= 2 && nband >= 1, kInvalidArgument, "need david_ndim >= 2 and nband >= 1");
        std::vector<int> dims(nk);
        ld_ = 0;
        for (int q = 0; q < nk; ++q) {
            B200_CHECK(iks[q] >= 0 && iks[q] < int(H->grid->kmaps.size()), kInvalidArgument, "k-point index out of range");
            dims[q] = H->grid->kmaps[iks[q]].npw;
            B200_CHECK(nbase_x_ < dims[q], kInvalidArgument, "need david_ndim*nband < npw of every k-point");
            ld_ = std::max(ld_, dims[q]);
        }
        sb_ = long(nbase_x_) * ld_;
        const long sh = long(nbase_x_) * nbase_x_;
        basis_.resize(size_t(nk) * sb_);
        hp_.resize(size_t(nk) * sb_);
        hcc_.resize(size_t(nk) * sh);
        vcc_.resize(size_t(nk) * sh);
        a64_.resize(size_t(nk) * sh);
        w_.resize(size_t(nk) * nbase_x_);
        wa_.resize(size_t(nk) * nbase_x_);
        eold_.resize(size_t(nk) * nband);
        vc_.resize(size_t(nk) * nbase_x_ * nband);
        vcl_.resize(size_t(nk) * nbase_x_ * nband);
        lag_.resize(size_t(nk) * nbase_x_ * nband);
        gram_.resize(size_t(nk) * nband * nband);
        newv_.resize(size_t(nk) * nband * ld_);
        newh_.resize(size_t(nk) * nband * ld_);
        pc_.resize(size_t(nk) * ld_);
        dims_.resize(nk);
        notconv_.resize(nk);
        unconv_.resize(size_t(nk) * nband);
        iters_.resize(nk);
        status_.resize(4);
        bad_.resize(nk);
        pinfo_.resize(nk);
        colmask_.resize(size_t(nk) * nbase_x_);
        xptr_.resize(nk);
        gptr_.resize(nk);
        psiptr_.resize(nk);
        B200_CUDA(cudaMemcpyAsync(dims_.ptr, dims.data(), nk * sizeof(int), cudaMemcpyHostToDevice, s_));
        B200_CUDA(cudaMemsetAsync(pc_.ptr, 0, pc_.n * sizeof(double), s_));
        for (int q = 0; q < nk; ++q)
            B200_CUDA(cudaMemcpyAsync(pc_.ptr + size_t(q) * ld_, precond_d[q], dims[q] * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s_));
        B200_CUBLAS(cublasCreate(&cb_));
        B200_CUBLAS(cublasSetStream(cb_, s_));
        B200_CUSOLVER(cusolverDnCreate(&cs_));
        B200_CUSOLVER(cusolverDnSetStream(cs_, s_));
        B200_CUSOLVER(cusolverDnCreateParams(&prm_));
        // batched eigensolver workspace: the largest over the subspace sizes a solve can reach
        size_t dws = 0, hws = 0;
        for (int n = nband; n <= nbase_x_; ++n) {
            size_t d = 0, hh = 0;
            B200_CUSOLVER(cusolverDnXsyevBatched_bufferSize(cs_, prm_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n,
                                                            CUDA_C_64F, a64_.ptr, n, CUDA_R_64F, wa_.ptr, CUDA_C_64F, &d,
                                                            &hh, nk));
            dws = std::max(dws, d);
            hws = std::max(hws, hh);
        }
        eig_work_.resize(dws / sizeof(double2) + 1);
        eig_hwork_.assign(hws + 1, 0);
        einfo_.resize(nk);
        B200_CUDA(cudaStreamSynchronize(s_));
    }
    ~DavidBatch() {
        if (prm_) cusolverDnDestroyParams(prm_);
        if (cs_) cusolverDnDestroy(cs_);
        if (cb_) cublasDestroy(cb_);
    }

    // psi_d[q]: nband start vectors of k-point iks[q] at psi_d[q] + m*ldpsi, overwritten with the eigenvectors;
    // eig (host, nk x nband); iters (host, nk): the iteration after which each k-point had converged
    void solve(double2* const* psi_d, int ldpsi, double* eig, double thr, int maxiter, int* iters_out) {
        B200_CHECK(ldpsi >= ld_, kInvalidArgument, "ldpsi smaller than the largest npw of the batch");
        const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
        const long sh = long(nbase_x_) * nbase_x_;
        B200_CUDA(cudaMemcpyAsync(psiptr_.ptr, psi_d, nk_ * sizeof(double2*), cudaMemcpyHostToDevice, s_));
        for (auto* a : {&hcc_, &vcc_})
            B200_CUDA(cudaMemsetAsync(a->ptr, 0, a->n * sizeof(double2), s_));
        B200_CUDA(cudaMemsetAsync(hp_.ptr, 0, hp_.n * sizeof(double2), s_));
        B200_CUDA(cudaMemsetAsync(iters_.ptr, 0, nk_ * sizeof(int), s_));
        B200_CUDA(cudaMemsetAsync(status_.ptr, 0, status_.n * sizeof(int), s_));
        k_load_start<<<blocks_of(long(nk_) * nband_ * ld_), kBT, 0, s_>>>(nk_, nband_, ld_, sb_, dims_.ptr,
                                                                        psiptr_.ptr, ldpsi, basis_.ptr);
        // the start block: every band of every k-point is real
        k_mask_start<<<blocks_of(long(nk_) * nbase_x_), kBT, 0, s_>>>(nk_, nband_, nbase_x_, colmask_.ptr);
        note_launch(2);
        B200_CUDA(cudaGetLastError());
        std::vector<int> notconv_h(nk_, nband_);
        B200_CUDA(cudaMemcpyAsync(notconv_.ptr, notconv_h.data(), nk_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        orth(0, nband_);
        apply_h(0, nband_, notconv_h);
        elem(0, nband_);
        int nbase = nband_;
        eigsolve(nbase);
        fill_eold_inf();  // every band starts unconverged
        int status[4];
        converge(thr, 0, status, notconv_h);
        int iter = 0;
        while (true) {
            ++iter;
            const int nc = status[0];
            // new block: residuals of the unconverged bands, preconditioned, orthogonalised, H applied
            k_gather_batch<<<blocks_of(long(nk_) * nc * nbase), kBT, 0, s_>>>(nk_, nbase, nbase_x_, nband_, nc,
                                                                            notconv_.ptr, unconv_.ptr, vcc_.ptr,
                                                                            w_.ptr, vc_.ptr, vcl_.ptr, colmask_.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
            double2* X = basis_.ptr + long(nbase) * ld_;
            const long sv = long(nbase_x_) * nband_;
            gemm_b(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nc, nbase, one, hp_.ptr, ld_, sb_, vc_.ptr, nbase_x_, sv, zero, X, ld_, sb_);
            gemm_b(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nc, nbase, one, basis_.ptr, ld_, sb_, vcl_.ptr, nbase_x_, sv, one, X, ld_,
                   sb_);
            k_precond_batch<<<blocks_of(long(nk_) * nc * ld_), kBT, 0, s_>>>(nk_, nc, ld_, sb_, long(nbase) * ld_,
                                                                            dims_.ptr, pc_.ptr, basis_.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
            orth(nbase, nc);
            apply_h(nbase, nc, notconv_h);
            elem(nbase, nc);
            nbase += nc;
            eigsolve(nbase);
            converge(thr, iter, status, notconv_h);
            const bool done = status[1] == 0 || iter == maxiter;
            if (done || nbase + status[0] > nbase_x_) {
                // psi = basis vcc(:, :nband) for every k-point (the refresh's first step, and the result)
                gemm_b(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nband_, nbase, one, basis_.ptr, ld_, sb_, vcc_.ptr, nbase_x_, sh,
                       zero, newv_.ptr, ld_, long(nband_) * ld_);
                if (done) break;
                gemm_b(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nband_, nbase, one, hp_.ptr, ld_, sb_, vcc_.ptr, nbase_x_, sh, zero,
                       newh_.ptr, ld_, long(nband_) * ld_);
                k_restart<<<blocks_of(long(nk_) * nband_ * ld_), kBT, 0, s_>>>(nk_, nband_, ld_, nbase_x_, sb_,
                                                                              newv_.ptr, newh_.ptr, basis_.ptr, hp_.ptr);
                B200_CUDA(cudaMemsetAsync(hcc_.ptr, 0, hcc_.n * sizeof(double2), s_));
                B200_CUDA(cudaMemsetAsync(vcc_.ptr, 0, vcc_.n * sizeof(double2), s_));
                k_restart_small<<<blocks_of(long(nk_) * nbase_x_), kBT, 0, s_>>>(nk_, nband_, nbase_x_, eold_.ptr,
                                                                                hcc_.ptr, vcc_.ptr, colmask_.ptr);
                note_launch(2);
                B200_CUDA(cudaGetLastError());
                nbase = nband_;
            }
        }
        // results: eigenvectors into psi, eigenvalues and iteration counts to the host
        k_store_psi<<<blocks_of(long(nk_) * nband_ * ldpsi), kBT, 0, s_>>>(nk_, nband_, ld_, ldpsi, newv_.ptr, psiptr_.ptr);
        note_launch();
        B200_CUDA(cudaGetLastError());
        std::vector<double> wh(size_t(nk_) * nbase_x_);
        B200_CUDA(cudaMemcpyAsync(wh.data(), w_.ptr, wh.size() * sizeof(double), cudaMemcpyDeviceToHost, s_));
        if (iters_out) B200_CUDA(cudaMemcpyAsync(iters_out, iters_.ptr, nk_ * sizeof(int), cudaMemcpyDeviceToHost, s_));
        B200_CUDA(cudaStreamSynchronize(s_));
        for (int q = 0; q < nk_; ++q)
            for (int m = 0; m < nband_; ++m) eig[size_t(q) * nband_ + m] = wh[size_t(q) * nbase_x_ + m];
        if (iters_out)
            for (int q = 0; q < nk_; ++q) iters_out[q] = std::min(iters_out[q] + 1, iter);
    }

  private:
    // C_k = al op(A_k) op(B_k) + be C_k for every k-point (strides between k-points)
    void gemm_b(cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, double2 al, const double2* A, int lda,
                long sa, const double2* B, int ldb, long sbb, double2 be, double2* C, int ldc, long sc) {
        if (m <= 0 || n <= 0) return;
        B200_CUBLAS(cublasZgemmStridedBatched(cb_, ta, tb, m, n, k, (const cuDoubleComplex*)&al,
                                              (const cuDoubleComplex*)A, lda, sa, (const cuDoubleComplex*)B, ldb, sbb,
                                              (const cuDoubleComplex*)&be, (cuDoubleComplex*)C, ldc, sc, nk_));
    }

    // block Gram-Schmidt against the first nbase columns and Cholesky-QR of the nc new ones, twice
    void orth(int nbase, int nc) {
        const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0), mone = make_double2(-1.0, 0.0);
        double2* X = basis_.ptr + long(nbase) * ld_;
        const long sv = long(nbase_x_) * nband_, sg = long(nband_) * nband_;
        k_fill_ptrs<<<(nk_ + 127) / 128, 128, 0, s_>>>(nk_, basis_.ptr, sb_, long(nbase) * ld_, xptr_.ptr);
        k_fill_ptrs<<<(nk_ + 127) / 128, 128, 0, s_>>>(nk_, gram_.ptr, sg, 0, gptr_.ptr);
        note_launch(2);
        for (int pass = 0; pass < 2; ++pass) {
            if (nbase > 0) {
                gemm_b(CUBLAS_OP_C, CUBLAS_OP_N, nbase, nc, ld_, one, basis_.ptr, ld_, sb_, X, ld_, sb_, zero, lag_.ptr,
                       nbase_x_, sv);
                gemm_b(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nc, nbase, mone, basis_.ptr, ld_, sb_, lag_.ptr, nbase_x_, sv, one,
                       X, ld_, sb_);
            }
            gemm_b(CUBLAS_OP_C, CUBLAS_OP_N, nc, nc, ld_, one, X, ld_, sb_, X, ld_, sb_, zero, gram_.ptr, nband_, sg);
            k_fix_gram<<<blocks_of(long(nk_) * nc * nc), kBT, 0, s_>>>(nk_, nc, nband_, notconv_.ptr, gram_.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
            B200_CUSOLVER(cusolverDnZpotrfBatched(cs_, CUBLAS_FILL_MODE_UPPER, nc, (cuDoubleComplex**)gptr_.ptr, nband_,
                                                  pinfo_.ptr, nk_));
            B200_CUBLAS(cublasZtrsmBatched(cb_, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                                           CUBLAS_DIAG_NON_UNIT, ld_, nc, (const cuDoubleComplex*)&one,
                                           (const cuDoubleComplex* const*)gptr_.ptr, nband_,
                                           (cuDoubleComplex* const*)xptr_.ptr, ld_, nk_));
            // a failed factorisation (linearly dependent directions) is reported with the iteration's status
            k_info_max<<<1, 32, 0, s_>>>(nk_, pinfo_.ptr, status_.ptr + 3);
            note_launch();
        }
    }

    // H applied to the nc new columns of every k-point that still has unconverged bands
    void apply_h(int nbase, int nc, const std::vector<int>& notconv_h) {
        std::vector<int> iks;
        std::vector<const double2*> xs;
        std::vector<double2*> hs;
        for (int q = 0; q < nk_; ++q) {
            if (notconv_h[q] == 0) continue;  // all of its new columns are dummy (zero), and so is their H image
            iks.push_back(iks_[q]);
            xs.push_back(basis_.ptr + q * sb_ + long(nbase) * ld_);
            hs.push_back(hp_.ptr + q * sb_ + long(nbase) * ld_);
        }
        // the H images of skipped k-points' dummy columns are zero: hp was cleared at the start and on
        // restarts only the first nband columns are rewritten
        B200_CUDA(cudaMemset2DAsync(hp_.ptr + long(nbase) * ld_, sb_ * sizeof(double2), 0,
                                    size_t(nc) * ld_ * sizeof(double2), nk_, s_));
        if (!iks.empty()) H_->hpsi_kbatch<double2>(int(iks.size()), iks.data(), spin_, nc, ld_, xs.data(), hs.data(), s_, &W_);
    }

    // new rows of every subspace matrix: hcc(nbase:nbase+nc, :nbase+nc) = X^H [hp(:, :nbase+nc)]
    void elem(int nbase, int nc) {
        const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
        gemm_b(CUBLAS_OP_C, CUBLAS_OP_N, nc, nbase + nc, ld_, one, basis_.ptr + long(nbase) * ld_, ld_, sb_, hp_.ptr, ld_,
               sb_, zero, hcc_.ptr + nbase, nbase_x_, long(nbase_x_) * nbase_x_);
    }

    // lowest nband eigenpairs of every subspace matrix (one batched eigensolver call)
    void eigsolve(int n) {
        B200_CUDA(cudaMemsetAsync(bad_.ptr, 0, nk_ * sizeof(int), s_));
        k_eig_in<<<blocks_of(long(nk_) * n * n), kBT, 0, s_>>>(nk_, n, nbase_x_, colmask_.ptr, hcc_.ptr, a64_.ptr,
                                                               bad_.ptr);
        k_eig_guard<<<blocks_of(long(nk_) * n * n), kBT, 0, s_>>>(nk_, n, bad_.ptr, a64_.ptr);
        note_launch(2);
        B200_CUDA(cudaGetLastError());
        B200_CUSOLVER(cusolverDnXsyevBatched(cs_, prm_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_C_64F,
                                             a64_.ptr, n, CUDA_R_64F, wa_.ptr, CUDA_C_64F, eig_work_.ptr,
                                             eig_work_.n * sizeof(double2), eig_hwork_.data(), eig_hwork_.size(),
                                             einfo_.ptr, nk_));
        k_eig_out<<<blocks_of(long(nk_) * nband_ * nbase_x_), kBT, 0, s_>>>(nk_, n, nbase_x_, nband_, a64_.ptr, wa_.ptr,
                                                                            vcc_.ptr, w_.ptr);
        k_info_max<<<1, 32, 0, s_>>>(nk_, bad_.ptr, status_.ptr + 2);
        k_info_max<<<1, 32, 0, s_>>>(nk_, einfo_.ptr, status_.ptr + 2);
        note_launch(3);
        B200_CUDA(cudaGetLastError());
    }

    void fill_eold_inf() {  // +big: the first test counts every band as changed
        std::vector<double> inf(size_t(nk_) * nband_, 1e300);
        B200_CUDA(cudaMemcpyAsync(eold_.ptr, inf.data(), inf.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
        B200_CUDA(cudaStreamSynchronize(s_));
    }

    // the convergence test of the iteration, and its status and per-k counts of unconverged bands to the host
    // (the one synchronisation per iteration)
    void converge(double thr, int iter, int* status, std::vector<int>& notconv_h) {
        B200_CUDA(cudaMemsetAsync(status_.ptr, 0, 2 * sizeof(int), s_));
        k_converge<<<(nk_ * 32 + 255) / 256, 256, 0, s_>>>(nk_, nband_, nbase_x_, thr, iter, w_.ptr, eold_.ptr,
                                                          notconv_.ptr, unconv_.ptr, iters_.ptr, status_.ptr);
        note_launch();
        B200_CUDA(cudaGetLastError());
        B200_CUDA(cudaMemcpyAsync(status, status_.ptr, 4 * sizeof(int), cudaMemcpyDeviceToHost, s_));
        B200_CUDA(cudaMemcpyAsync(notconv_h.data(), notconv_.ptr, nk_ * sizeof(int), cudaMemcpyDeviceToHost, s_));
        B200_CUDA(cudaStreamSynchronize(s_));
        B200_CHECK(status[2] == 0, kNumericalError,
                   "subspace eigensolver failed or non-finite entries (NaN/Inf in psi, V_eff, D or H|psi>)");
        B200_CHECK(status[3] == 0, kNumericalError, "Cholesky of a new block failed (linearly dependent directions)");
    }

    Hamilt* H_;
    int nk_;
    std::vector<int> iks_;
    int spin_, nband_, nbase_x_, ld_ = 0;
    long sb_ = 0;
    cudaStream_t s_;
    cublasHandle_t cb_ = nullptr;
    cusolverDnHandle_t cs_ = nullptr;
    cusolverDnParams_t prm_ = nullptr;
    HpsiWork W_;
    DeviceArray<double2> basis_, hp_, hcc_, vcc_, a64_, vc_, vcl_, lag_, gram_, newv_, newh_, eig_work_;
    DeviceArray<double> w_, wa_, eold_, pc_;
    DeviceArray<int> dims_, notconv_, unconv_, iters_, status_, bad_, pinfo_, einfo_;
    DeviceArray<unsigned char> colmask_;
    DeviceArray<double2*> xptr_, gptr_;
    DeviceArray<double2*> psiptr_;
    std::vector<char> eig_hwork_;
};

}  // namespace
}  // namespace b200

extern "C" int b200_solve_kpoints_batched(b200_hamilt* h, int nk, const int* iks, int spin, int nband, int david_ndim,
                                          const double* const* precond_d, void* const* psi_d, int ldpsi,
                                          double* eigenvalues, double thr, int maxiter, int* iters, void* stream) {
    return b200::guarded([&] {
        B200_CHECK(h && iks && precond_d && psi_d && eigenvalues, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(maxiter >= 1, b200::kInvalidArgument, "maxiter must be positive");
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        b200::DavidBatch d(h->h.get(), nk, iks, spin, nband, david_ndim, precond_d, s);
        d.solve(reinterpret_cast<double2* const*>(psi_d), ldpsi, eigenvalues, thr, maxiter, iters);
    });
}
