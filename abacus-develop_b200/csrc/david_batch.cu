// Davidson of many k-points in lock-step: the k loop of HSolverPW::solve (hsolver_pw.cpp:240-270) with every
// k-point's DiagoDavid iteration (diago_david.cpp:151-341) advanced together, so that each phase of an
// iteration is one launch (or one batched library call) for all k instead of one per k-point:
//   * H|psi> of the new vectors of every k-point: Hamilt::hpsi_kbatch (the local pass in one launch per FFT
//     pass for all k);
//   * the residuals, projections, Gram matrices and subspace rows: strided-batched GEMMs over k;
//   * Cholesky-QR of the new blocks: batched FP64 ZPOTRF + triangular solves;
//   * the subspace eigensolves: one batched FP64 Hermitian eigensolver call (cusolverDnXsyevBatched);
//   * the convergence test |d lambda| < thr per band: on the device, one small read per iteration.
// The k-points differ in their numbers of unconverged bands; every k-point adds the same number nc (the
// largest) of new columns, the surplus ones "dummy": zero vectors, which the Gram matrix sees as unit
// columns and the subspace matrix as an isolated eigenvalue far above the band energies (kDummyDiag), so they
// never enter the lowest nband Ritz pairs.  Vectors are padded with zeros to the largest npw of the batch.
// Differences from one DiagoDavid per k-point (same mathematics): a block Gram-Schmidt + Cholesky-QR
// orthogonalisation (twice) instead of the per-vector SchmidtOrth, S = I, and a common restart (refresh) of
// all k-points whenever the common basis would overflow david_ndim * nband.
// Mixed precision: an FP32 stage (FP32 H|psi>, FP32 vectors and subspace products, FP64 Cholesky and
// eigensolves, FP64 convergence test) to 1e-7, then the FP64 iteration from its vectors to the requested
// threshold, as the single-k-point mixed solve does.
#include <algorithm>
#include <memory>
#include <type_traits>
#include <vector>

#include "capi_guard.h"
#include "../../include/abacus_b200.h"
#include "capi_handles.h"
#include "david_batch.h"
#include "linalg_status.h"

namespace b200 {
namespace {

constexpr int kBT = 256;
constexpr double kDummyDiag = 1.0e3;  // Ry: far above any band energy, so dummy columns stay out of the lowest pairs
constexpr double kMixedThr = 1e-7;    // hand-over threshold of the FP32 stage

inline int blocks_of(long n) {
    long b = (n + kBT - 1) / kBT;
    if (b > 148L * 16) b = 148L * 16;
    return int(b < 1 ? 1 : b);
}
inline int even(int n) { return n + (n & 1); }

template <typename T> __device__ __forceinline__ T tz() { return cmake<T>(0, 0); }
template <typename T, typename S> __device__ __forceinline__ T cvt(S v) { return cmake<T>(v.x, v.y); }

// batched linear algebra of one precision
template <typename T> struct BLin;
template <> struct BLin<double2> {
    static void gemm(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, double2 al,
                     const double2* A, int lda, long sa, const double2* B, int ldb, long sb, double2 be, double2* C,
                     int ldc, long sc, int batch) {
        B200_CUBLAS(cublasZgemmStridedBatched(h, ta, tb, m, n, k, (const cuDoubleComplex*)&al, (const cuDoubleComplex*)A,
                                              lda, sa, (const cuDoubleComplex*)B, ldb, sb, (const cuDoubleComplex*)&be,
                                              (cuDoubleComplex*)C, ldc, sc, batch));
    }
    static void trsm(cublasHandle_t h, int m, int n, const double2* const* U, int ldu, double2* const* X, int ldx,
                     int batch) {
        const double2 one = make_double2(1.0, 0.0);
        B200_CUBLAS(cublasZtrsmBatched(h, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, m,
                                       n, (const cuDoubleComplex*)&one, (const cuDoubleComplex* const*)U, ldu,
                                       (cuDoubleComplex* const*)X, ldx, batch));
    }
};
template <> struct BLin<float2> {
    static void gemm(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, float2 al,
                     const float2* A, int lda, long sa, const float2* B, int ldb, long sb, float2 be, float2* C, int ldc,
                     long sc, int batch) {
        B200_CUBLAS(cublasCgemmStridedBatched(h, ta, tb, m, n, k, (const cuComplex*)&al, (const cuComplex*)A, lda, sa,
                                              (const cuComplex*)B, ldb, sb, (const cuComplex*)&be, (cuComplex*)C, ldc, sc,
                                              batch));
    }
    static void trsm(cublasHandle_t h, int m, int n, const float2* const* U, int ldu, float2* const* X, int ldx,
                     int batch) {
        const float2 one = make_float2(1.f, 0.f);
        B200_CUBLAS(cublasCtrsmBatched(h, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, m,
                                       n, (const cuComplex*)&one, (const cuComplex* const*)U, ldu,
                                       (cuComplex* const*)X, ldx, batch));
    }
};

// basis_k[:, m] = psi_k[:, m] for g < dim_k, 0 beyond (psi_k = psi[k], FP64, pitch ldpsi)
template <typename T>
__global__ void k_load_start(int nk, int nband, int ld, long sb, const int* __restrict__ dims,
                             const double2* const* __restrict__ psi, int ldpsi, T* __restrict__ basis) {
    const long total = long(nk) * nband * ld;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int g = int(i % ld);
        const int m = int((i / ld) % nband);
        const int k = int(i / (long(ld) * nband));
        basis[k * sb + long(m) * ld + g] = g < dims[k] ? cvt<T>(psi[k][long(m) * ldpsi + g]) : tz<T>();
    }
}

// residual coefficients of the new block: vc(:, m) = vcc(:nbase, unconv[m]), vcl = -lambda vc for the
// unconverged bands m < notconv_k, zero for the dummy columns notconv_k <= m < nc; marks the new columns
// of the basis (real or dummy)
template <typename T>
__global__ void k_gather_batch(int nk, int nbase, int nbase_x, int nband, int nc, const int* __restrict__ notconv,
                               const int* __restrict__ unconv, const T* __restrict__ vcc, const double* __restrict__ w,
                               T* __restrict__ vc, T* __restrict__ vcl, unsigned char* __restrict__ colmask) {
    const long total = long(nk) * nc * nbase;
    const long sh = long(nbase_x) * nbase_x, sv = long(nbase_x) * nband;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int r = int(i % nbase);
        const int m = int((i / nbase) % nc);
        const int k = int(i / (long(nbase) * nc));
        T v = tz<T>(), vl = tz<T>();
        if (m < notconv[k]) {
            const int col = unconv[k * nband + m];
            v = vcc[k * sh + long(col) * nbase_x + r];
            const double lam = w[long(k) * nbase_x + col];
            vl = cmake<T>(-lam * v.x, -lam * v.y);
        }
        vc[k * sv + long(m) * nbase_x + r] = v;
        vcl[k * sv + long(m) * nbase_x + r] = vl;
        if (r == 0) colmask[long(k) * nbase_x + nbase + m] = m < notconv[k] ? 1 : 0;
    }
}

// X_k(:, m) /= precondition_k (the reference's vector_div_vector_op), zero in the padding rows
template <typename T>
__global__ void k_precond_batch(int nk, int nc, int ld, long sb, long off, const int* __restrict__ dims,
                                const double* __restrict__ pc, T* __restrict__ basis) {
    const long total = long(nk) * nc * ld;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int g = int(i % ld);
        const int m = int((i / ld) % nc);
        const int k = int(i / (long(ld) * nc));
        T* x = basis + k * sb + off + long(m) * ld + g;
        if (g < dims[k]) {
            const double p = pc[long(k) * ld + g];
            *x = cmake<T>(double(x->x) / p, double(x->y) / p);
        } else {
            *x = tz<T>();
        }
    }
}

// Gram matrices of the new blocks (FP64 copies): the dummy columns (m >= notconv_k) become unit columns, so
// the Cholesky factor keeps them apart and they stay zero through X U^-1
template <typename T>
__global__ void k_gram64(int nk, int nc, int ldg, const int* __restrict__ notconv, const T* __restrict__ g,
                         double2* __restrict__ g64) {
    const long total = long(nk) * nc * nc;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int i = int(t % nc);
        const int j = int((t / nc) % nc);
        const int k = int(t / (long(nc) * nc));
        const long o = long(k) * ldg * ldg + long(j) * ldg + i;
        g64[o] = (i >= notconv[k] || j >= notconv[k]) ? make_double2(i == j ? 1.0 : 0.0, 0.0) : cvt<double2>(g[o]);
    }
}
// the FP64 Cholesky factors back in the vectors' precision
template <typename T>
__global__ void k_gram_back(int nk, int nc, int ldg, const double2* __restrict__ g64, T* __restrict__ g) {
    const long total = long(nk) * nc * nc;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int i = int(t % nc);
        const int j = int((t / nc) % nc);
        const int k = int(t / (long(nc) * nc));
        const long o = long(k) * ldg * ldg + long(j) * ldg + i;
        g[o] = cvt<T>(g64[o]);
    }
}

template <typename P> __global__ void k_fill_ptrs(int nk, P* base, long stride, long off, P** out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nk) out[k] = base + k * stride + off;
}

// eigensolver input: the leading n x n block of each hcc (lower triangle) in FP64, compact with lda = n; rows
// and columns of dummy basis vectors become kDummyDiag on the diagonal and 0 elsewhere; a non-finite entry of
// the lower triangle sets bad[k] (that matrix is then replaced by I, so the eigensolver never sees NaN)
template <typename T>
__global__ void k_eig_in(int nk, int n, int nbase_x, const unsigned char* __restrict__ colmask, const T* __restrict__ hcc,
                         double2* __restrict__ a, int* __restrict__ bad) {
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
                v = cvt<double2>(hcc[k * sh + long(j) * nbase_x + i]);
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
template <typename T>
__global__ void k_eig_out(int nk, int n, int nbase_x, int nband, const double2* __restrict__ a,
                          const double* __restrict__ wa, T* __restrict__ vcc, double* __restrict__ w) {
    const long total = long(nk) * nband * nbase_x;
    const long sh = long(nbase_x) * nbase_x;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int r = int(t % nbase_x);
        const int m = int((t / nbase_x) % nband);
        const int k = int(t / (long(nbase_x) * nband));
        vcc[k * sh + long(m) * nbase_x + r] = r < n ? cvt<T>(a[long(k) * n * n + long(m) * n + r]) : tz<T>();
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

// restart: basis(:, :nband) <- newv, hp(:, :nband) <- newh
template <typename T>
__global__ void k_restart(int nk, int nband, int ld, long sb, const T* __restrict__ newv, const T* __restrict__ newh,
                          T* __restrict__ basis, T* __restrict__ hp) {
    const long total = long(nk) * nband * ld;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int g = int(i % ld);
        const int m = int((i / ld) % nband);
        const int k = int(i / (long(ld) * nband));
        basis[k * sb + long(m) * ld + g] = newv[i];
        hp[k * sb + long(m) * ld + g] = newh[i];
    }
}
// restart of the small matrices: hcc = diag(e), vcc = I (first nband), masks of the first nband columns
template <typename T>
__global__ void k_restart_small(int nk, int nband, int nbase_x, const double* __restrict__ e_old, T* __restrict__ hcc,
                                T* __restrict__ vcc, unsigned char* __restrict__ colmask) {
    const long sh = long(nbase_x) * nbase_x;
    const long total = long(nk) * nbase_x;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int i = int(t % nbase_x);
        const int k = int(t / nbase_x);
        colmask[t] = i < nband ? 1 : 0;
        if (i < nband) {
            hcc[k * sh + long(i) * nbase_x + i] = cmake<T>(e_old[long(k) * nband + i], 0.0);
            vcc[k * sh + long(i) * nbase_x + i] = cmake<T>(1.0, 0.0);
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

// psi_k(:, m) <- v_k(:, m) (pitch ld) for g < ld, 0 for ld <= g < ldpsi (FP64 psi)
template <typename T>
__global__ void k_store_psi(int nk, int nband, int ld, int ldpsi, const T* __restrict__ v,
                            double2* const* __restrict__ psi) {
    const long total = long(nk) * nband * ldpsi;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int g = int(i % ldpsi);
        const int m = int((i / ldpsi) % nband);
        const int k = int(i / (long(ldpsi) * nband));
        psi[k][long(m) * ldpsi + g] = g < ld ? cvt<double2>(v[(long(k) * nband + m) * ld + g]) : make_double2(0.0, 0.0);
    }
}

// One precision's lock-step Davidson for up to `cap` k-points with at most `dim_cap` plane waves each.  Every
// buffer is made at construction; setup() points the engine at a batch of k-points, solve() runs it.
template <typename T> class BatchEngine {
    static constexpr bool kF32 = std::is_same<T, float2>::value;

  public:
    BatchEngine(Hamilt* H, int cap, int nband, int ndim, int dim_cap, cudaStream_t s)
        : H_(H), cap_(cap), nband_(nband), nbase_x_(ndim * nband), s_(s) {
        B200_CHECK(cap >= 1 && cap <= kMaxKBatch, kInvalidArgument, "1..128 k-points per batch");
        B200_CHECK(ndim >= 2 && nband >= 1, kInvalidArgument, "need david_ndim >= 2 and nband >= 1");
        B200_CHECK(nbase_x_ < dim_cap, kInvalidArgument, "need david_ndim*nband < npw");
        ld_ = kF32 ? even(dim_cap) : dim_cap;  // FP32: an even pitch, valid for the tensor-core products of H|psi>
        sb_ = long(nbase_x_) * ld_;
        const long sh = long(nbase_x_) * nbase_x_;
        basis_.resize(size_t(cap) * sb_);
        hp_.resize(size_t(cap) * sb_);
        hcc_.resize(size_t(cap) * sh);
        vcc_.resize(size_t(cap) * sh);
        a64_.resize(size_t(cap) * sh);
        w_.resize(size_t(cap) * nbase_x_);
        wa_.resize(size_t(cap) * nbase_x_);
        eold_.resize(size_t(cap) * nband);
        vc_.resize(size_t(cap) * nbase_x_ * nband);
        vcl_.resize(size_t(cap) * nbase_x_ * nband);
        lag_.resize(size_t(cap) * nbase_x_ * nband);
        gram_.resize(size_t(cap) * nband * nband);
        gram64_.resize(size_t(cap) * nband * nband);
        newv_.resize(size_t(cap) * nband * ld_);
        newh_.resize(size_t(cap) * nband * ld_);
        pc_.resize(size_t(cap) * ld_);
        dims_.resize(cap);
        notconv_.resize(cap);
        unconv_.resize(size_t(cap) * nband);
        iters_.resize(cap);
        status_.resize(4);
        bad_.resize(cap);
        pinfo_.resize(cap);
        einfo_.resize(cap);
        colmask_.resize(size_t(cap) * nbase_x_);
        xptr_.resize(cap);
        gptr_.resize(cap);
        g64ptr_.resize(cap);
        psiptr_.resize(cap);
        B200_CUBLAS(cublasCreate(&cb_));
        B200_CUBLAS(cublasSetStream(cb_, s_));
        B200_CUSOLVER(cusolverDnCreate(&cs_));
        B200_CUSOLVER(cusolverDnSetStream(cs_, s_));
        B200_CUSOLVER(cusolverDnCreateParams(&prm_));
        // batched eigensolver workspace: the largest over the subspace sizes and batch sizes a solve can reach
        size_t dws = 0, hws = 0;
        for (int n = nband; n <= nbase_x_; ++n)
            for (int b : {1, cap}) {
                size_t d = 0, hh = 0;
                B200_CUSOLVER(cusolverDnXsyevBatched_bufferSize(cs_, prm_, CUSOLVER_EIG_MODE_VECTOR,
                                                                CUBLAS_FILL_MODE_LOWER, n, CUDA_C_64F, a64_.ptr, n,
                                                                CUDA_R_64F, wa_.ptr, CUDA_C_64F, &d, &hh, b));
                dws = std::max(dws, d);
                hws = std::max(hws, hh);
            }
        eig_work_.resize(dws / sizeof(double2) + 1);
        eig_hwork_.assign(hws + 1, 0);
        B200_CUDA(cudaStreamSynchronize(s_));
    }
    ~BatchEngine() {
        if (prm_) cusolverDnDestroyParams(prm_);
        if (cs_) cusolverDnDestroy(cs_);
        if (cb_) cublasDestroy(cb_);
    }
    BatchEngine(const BatchEngine&) = delete;
    BatchEngine& operator=(const BatchEngine&) = delete;

    int cap() const { return cap_; }
    int dim_cap() const { return ld_; }

    // the batch: k-points iks (their npw <= the capacity) with their FP64 preconditioners
    void setup(int nk, const int* iks, int spin, const double* const* precond_d) {
        B200_CHECK(nk >= 1 && nk <= cap_, kInvalidArgument, "more k-points than the batch capacity");
        nk_ = nk;
        spin_ = spin;
        iks_.assign(iks, iks + nk);
        std::vector<int> dims(nk);
        for (int q = 0; q < nk; ++q) {
            B200_CHECK(iks[q] >= 0 && iks[q] < int(H_->grid->kmaps.size()), kInvalidArgument, "k-point index out of range");
            dims[q] = H_->grid->kmaps[iks[q]].npw;
            B200_CHECK(dims[q] <= ld_ && nbase_x_ < dims[q], kInvalidArgument,
                       "need david_ndim*nband < npw <= the batch's plane-wave capacity");
        }
        B200_CUDA(cudaMemcpyAsync(dims_.ptr, dims.data(), nk * sizeof(int), cudaMemcpyHostToDevice, s_));
        B200_CUDA(cudaMemsetAsync(pc_.ptr, 0, pc_.n * sizeof(double), s_));
        for (int q = 0; q < nk; ++q)
            B200_CUDA(cudaMemcpyAsync(pc_.ptr + size_t(q) * ld_, precond_d[q], dims[q] * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s_));
        B200_CUDA(cudaStreamSynchronize(s_));  // dims (host vector) and the preconditioner copies complete
    }

    // psi_d (device array of nk FP64 pointers): nband start vectors of each k-point at m*ldpsi, overwritten
    // with the eigenvectors; eig (host, nk x nband); iters (host, nk): the iteration after which each
    // k-point had converged.  Returns the iterations run.
    int solve(double2* const* psi_d, int ldpsi, double* eig, double thr, int maxiter, int* iters_out) {
        B200_CHECK(ldpsi >= ld_ || (kF32 && ldpsi >= ld_ - 1), kInvalidArgument,
                   "ldpsi smaller than the largest npw of the batch");
        const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
        const long sh = long(nbase_x_) * nbase_x_;
        B200_CUDA(cudaMemcpyAsync(psiptr_.ptr, psi_d, nk_ * sizeof(double2*), cudaMemcpyDeviceToDevice, s_));
        B200_CUDA(cudaMemsetAsync(hcc_.ptr, 0, hcc_.n * sizeof(T), s_));
        B200_CUDA(cudaMemsetAsync(vcc_.ptr, 0, vcc_.n * sizeof(T), s_));
        B200_CUDA(cudaMemsetAsync(hp_.ptr, 0, hp_.n * sizeof(T), s_));
        B200_CUDA(cudaMemsetAsync(iters_.ptr, 0, iters_.n * sizeof(int), s_));
        B200_CUDA(cudaMemsetAsync(status_.ptr, 0, status_.n * sizeof(int), s_));
        k_load_start<T><<<blocks_of(long(nk_) * nband_ * ld_), kBT, 0, s_>>>(nk_, nband_, ld_, sb_, dims_.ptr,
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
            k_gather_batch<T><<<blocks_of(long(nk_) * nc * nbase), kBT, 0, s_>>>(nk_, nbase, nbase_x_, nband_, nc,
                                                                               notconv_.ptr, unconv_.ptr, vcc_.ptr,
                                                                               w_.ptr, vc_.ptr, vcl_.ptr, colmask_.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
            T* X = basis_.ptr + long(nbase) * ld_;
            const long sv = long(nbase_x_) * nband_;
            gemm(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nc, nbase, one, hp_.ptr, ld_, sb_, vc_.ptr, nbase_x_, sv, zero, X, ld_, sb_);
            gemm(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nc, nbase, one, basis_.ptr, ld_, sb_, vcl_.ptr, nbase_x_, sv, one, X, ld_,
                 sb_);
            k_precond_batch<T><<<blocks_of(long(nk_) * nc * ld_), kBT, 0, s_>>>(nk_, nc, ld_, sb_, long(nbase) * ld_,
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
                gemm(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nband_, nbase, one, basis_.ptr, ld_, sb_, vcc_.ptr, nbase_x_, sh,
                     zero, newv_.ptr, ld_, long(nband_) * ld_);
                if (done) break;
                gemm(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nband_, nbase, one, hp_.ptr, ld_, sb_, vcc_.ptr, nbase_x_, sh, zero,
                     newh_.ptr, ld_, long(nband_) * ld_);
                k_restart<T><<<blocks_of(long(nk_) * nband_ * ld_), kBT, 0, s_>>>(nk_, nband_, ld_, sb_, newv_.ptr,
                                                                                 newh_.ptr, basis_.ptr, hp_.ptr);
                B200_CUDA(cudaMemsetAsync(hcc_.ptr, 0, hcc_.n * sizeof(T), s_));
                B200_CUDA(cudaMemsetAsync(vcc_.ptr, 0, vcc_.n * sizeof(T), s_));
                k_restart_small<T><<<blocks_of(long(nk_) * nbase_x_), kBT, 0, s_>>>(nk_, nband_, nbase_x_, eold_.ptr,
                                                                                   hcc_.ptr, vcc_.ptr, colmask_.ptr);
                note_launch(2);
                B200_CUDA(cudaGetLastError());
                nbase = nband_;
            }
        }
        // results: eigenvectors into psi, eigenvalues and iteration counts to the host
        k_store_psi<T><<<blocks_of(long(nk_) * nband_ * ldpsi), kBT, 0, s_>>>(nk_, nband_, ld_, ldpsi, newv_.ptr,
                                                                             psiptr_.ptr);
        note_launch();
        B200_CUDA(cudaGetLastError());
        std::vector<double> wh(size_t(nk_) * nbase_x_);
        B200_CUDA(cudaMemcpyAsync(wh.data(), w_.ptr, wh.size() * sizeof(double), cudaMemcpyDeviceToHost, s_));
        std::vector<int> ith(nk_);
        B200_CUDA(cudaMemcpyAsync(ith.data(), iters_.ptr, nk_ * sizeof(int), cudaMemcpyDeviceToHost, s_));
        B200_CUDA(cudaStreamSynchronize(s_));
        for (int q = 0; q < nk_; ++q)
            for (int m = 0; m < nband_; ++m) eig[size_t(q) * nband_ + m] = wh[size_t(q) * nbase_x_ + m];
        if (iters_out)
            for (int q = 0; q < nk_; ++q) iters_out[q] = std::min(ith[q] + 1, iter);
        return iter;
    }

  private:
    void gemm(cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, T al, const T* A, int lda, long sa,
              const T* B, int ldb, long sbb, T be, T* C, int ldc, long sc) {
        if (m <= 0 || n <= 0) return;
        BLin<T>::gemm(cb_, ta, tb, m, n, k, al, A, lda, sa, B, ldb, sbb, be, C, ldc, sc, nk_);
    }

    // block Gram-Schmidt against the first nbase columns and Cholesky-QR (FP64 Cholesky) of the nc new ones,
    // twice
    void orth(int nbase, int nc) {
        const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0), mone = cmake<T>(-1, 0);
        T* X = basis_.ptr + long(nbase) * ld_;
        const long sv = long(nbase_x_) * nband_, sg = long(nband_) * nband_;
        k_fill_ptrs<T><<<(nk_ + 127) / 128, 128, 0, s_>>>(nk_, basis_.ptr, sb_, long(nbase) * ld_, xptr_.ptr);
        k_fill_ptrs<T><<<(nk_ + 127) / 128, 128, 0, s_>>>(nk_, gram_.ptr, sg, 0, gptr_.ptr);
        k_fill_ptrs<double2><<<(nk_ + 127) / 128, 128, 0, s_>>>(nk_, gram64_.ptr, sg, 0, g64ptr_.ptr);
        note_launch(3);
        for (int pass = 0; pass < 2; ++pass) {
            if (nbase > 0) {
                gemm(CUBLAS_OP_C, CUBLAS_OP_N, nbase, nc, ld_, one, basis_.ptr, ld_, sb_, X, ld_, sb_, zero, lag_.ptr,
                     nbase_x_, sv);
                gemm(CUBLAS_OP_N, CUBLAS_OP_N, ld_, nc, nbase, mone, basis_.ptr, ld_, sb_, lag_.ptr, nbase_x_, sv, one, X,
                     ld_, sb_);
            }
            gemm(CUBLAS_OP_C, CUBLAS_OP_N, nc, nc, ld_, one, X, ld_, sb_, X, ld_, sb_, zero, gram_.ptr, nband_, sg);
            k_gram64<T><<<blocks_of(long(nk_) * nc * nc), kBT, 0, s_>>>(nk_, nc, nband_, notconv_.ptr, gram_.ptr,
                                                                       gram64_.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
            B200_CUSOLVER(cusolverDnZpotrfBatched(cs_, CUBLAS_FILL_MODE_UPPER, nc, (cuDoubleComplex**)g64ptr_.ptr, nband_,
                                                  pinfo_.ptr, nk_));
            if constexpr (kF32) {
                k_gram_back<T><<<blocks_of(long(nk_) * nc * nc), kBT, 0, s_>>>(nk_, nc, nband_, gram64_.ptr, gram_.ptr);
                note_launch();
                BLin<T>::trsm(cb_, ld_, nc, gptr_.ptr, nband_, xptr_.ptr, ld_, nk_);
            } else {
                BLin<T>::trsm(cb_, ld_, nc, g64ptr_.ptr, nband_, xptr_.ptr, ld_, nk_);
            }
            // a failed factorisation (linearly dependent directions) is reported with the iteration's status
            k_info_max<<<1, 32, 0, s_>>>(nk_, pinfo_.ptr, status_.ptr + 3);
            note_launch();
            B200_CUDA(cudaGetLastError());
        }
    }

    // H applied to the nc new columns of every k-point that still has unconverged bands
    void apply_h(int nbase, int nc, const std::vector<int>& notconv_h) {
        std::vector<int> iks;
        std::vector<const T*> xs;
        std::vector<T*> hs;
        for (int q = 0; q < nk_; ++q) {
            if (notconv_h[q] == 0) continue;  // all of its new columns are dummy (zero), and so is their H image
            iks.push_back(iks_[q]);
            xs.push_back(basis_.ptr + q * sb_ + long(nbase) * ld_);
            hs.push_back(hp_.ptr + q * sb_ + long(nbase) * ld_);
        }
        B200_CUDA(cudaMemset2DAsync(hp_.ptr + long(nbase) * ld_, sb_ * sizeof(T), 0, size_t(nc) * ld_ * sizeof(T), nk_,
                                    s_));
        if (!iks.empty()) H_->hpsi_kbatch<T>(int(iks.size()), iks.data(), spin_, nc, ld_, xs.data(), hs.data(), s_, &W_);
    }

    // new rows of every subspace matrix: hcc(nbase:nbase+nc, :nbase+nc) = X^H hp(:, :nbase+nc)
    void elem(int nbase, int nc) {
        const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
        gemm(CUBLAS_OP_C, CUBLAS_OP_N, nc, nbase + nc, ld_, one, basis_.ptr + long(nbase) * ld_, ld_, sb_, hp_.ptr, ld_,
             sb_, zero, hcc_.ptr + nbase, nbase_x_, long(nbase_x_) * nbase_x_);
    }

    // lowest nband eigenpairs of every subspace matrix, in FP64 (one batched eigensolver call)
    void eigsolve(int n) {
        B200_CUDA(cudaMemsetAsync(bad_.ptr, 0, nk_ * sizeof(int), s_));
        k_eig_in<T><<<blocks_of(long(nk_) * n * n), kBT, 0, s_>>>(nk_, n, nbase_x_, colmask_.ptr, hcc_.ptr, a64_.ptr,
                                                                  bad_.ptr);
        k_eig_guard<<<blocks_of(long(nk_) * n * n), kBT, 0, s_>>>(nk_, n, bad_.ptr, a64_.ptr);
        note_launch(2);
        B200_CUDA(cudaGetLastError());
        B200_CUSOLVER(cusolverDnXsyevBatched(cs_, prm_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_C_64F,
                                             a64_.ptr, n, CUDA_R_64F, wa_.ptr, CUDA_C_64F, eig_work_.ptr,
                                             eig_work_.n * sizeof(double2), eig_hwork_.data(), eig_hwork_.size(),
                                             einfo_.ptr, nk_));
        k_eig_out<T><<<blocks_of(long(nk_) * nband_ * nbase_x_), kBT, 0, s_>>>(nk_, n, nbase_x_, nband_, a64_.ptr,
                                                                               wa_.ptr, vcc_.ptr, w_.ptr);
        k_info_max<<<1, 32, 0, s_>>>(nk_, bad_.ptr, status_.ptr + 2);
        k_info_max<<<1, 32, 0, s_>>>(nk_, einfo_.ptr, status_.ptr + 2);
        note_launch(3);
        B200_CUDA(cudaGetLastError());
    }

    void fill_eold_inf() {  // a huge previous eigenvalue: the first test counts every band as changed
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
        if constexpr (kF32) {
            const int e = W_.tcw.err.ptr ? W_.tcw.read_error(s_) : 0;
            B200_CHECK(e == 0, kCudaError, "tensor-core GEMM wait ran out in H|psi> (error word " + std::to_string(e) + ")");
        }
    }

    Hamilt* H_;
    int cap_, nband_, nbase_x_, ld_ = 0, nk_ = 0, spin_ = 0;
    std::vector<int> iks_;
    long sb_ = 0;
    cudaStream_t s_;
    cublasHandle_t cb_ = nullptr;
    cusolverDnHandle_t cs_ = nullptr;
    cusolverDnParams_t prm_ = nullptr;
    HpsiWork W_;
    DeviceArray<T> basis_, hp_, hcc_, vcc_, vc_, vcl_, lag_, gram_, newv_, newh_;
    DeviceArray<double2> a64_, gram64_, eig_work_;
    DeviceArray<double> w_, wa_, eold_, pc_;
    DeviceArray<int> dims_, notconv_, unconv_, iters_, status_, bad_, pinfo_, einfo_;
    DeviceArray<unsigned char> colmask_;
    DeviceArray<T*> xptr_, gptr_;
    DeviceArray<double2*> g64ptr_, psiptr_;
    std::vector<char> eig_hwork_;
};

}  // namespace

// The batched solver of a Hamiltonian: an FP64 engine, and for mixed precision an FP32 engine whose result
// the FP64 engine refines.  Reusable: every buffer is made at construction (capacity in k-points and plane
// waves), so repeated solves allocate nothing.
class DavidBatchSolver {
  public:
    DavidBatchSolver(Hamilt* H, int cap, int nband, int ndim, int dim_cap, int precision, cudaStream_t s)
        : precision_(precision), nband_(nband), s_(s) {
        B200_CHECK(precision == B200_PREC_FP64 || precision == B200_PREC_MIXED, kInvalidArgument, "bad precision");
        e64_ = std::make_unique<BatchEngine<double2>>(H, cap, nband, ndim, dim_cap, s);
        if (precision == B200_PREC_MIXED) e32_ = std::make_unique<BatchEngine<float2>>(H, cap, nband, ndim, dim_cap, s);
        psiptr_.resize(cap);
    }
    int cap() const { return e64_->cap(); }
    int dim_cap() const { return e64_->dim_cap(); }
    // psi_h: host array of nk device pointers (FP64); returns the iterations of both stages
    int solve(int nk, const int* iks, int spin, const double* const* precond_d, void* const* psi_h, int ldpsi,
              double* eig, double thr, int maxiter, int* iters) {
        B200_CUDA(cudaMemcpyAsync(psiptr_.ptr, psi_h, nk * sizeof(double2*), cudaMemcpyHostToDevice, s_));
        int total = 0;
        std::vector<int> it32(nk, 0);
        if (e32_) {
            e32_->setup(nk, iks, spin, precond_d);
            total += e32_->solve(psiptr_.ptr, ldpsi, eig, thr > kMixedThr ? thr : kMixedThr, maxiter, it32.data());
        }
        e64_->setup(nk, iks, spin, precond_d);
        total += e64_->solve(psiptr_.ptr, ldpsi, eig, thr, maxiter, iters);
        if (iters)
            for (int q = 0; q < nk; ++q) iters[q] += it32[q];
        return total;
    }

  private:
    int precision_, nband_;
    cudaStream_t s_;
    std::unique_ptr<BatchEngine<double2>> e64_;
    std::unique_ptr<BatchEngine<float2>> e32_;
    DeviceArray<double2*> psiptr_;
};

void david_batch_destroy(DavidBatchSolver* d) { delete d; }
std::unique_ptr<DavidBatchSolver, void (*)(DavidBatchSolver*)> make_david_batch(Hamilt* H, int cap, int nband, int ndim,
                                                                                int dim_cap, int precision,
                                                                                cudaStream_t s) {
    return {new DavidBatchSolver(H, cap, nband, ndim, dim_cap, precision, s), &david_batch_destroy};
}
int david_batch_solve(DavidBatchSolver& d, int nk, const int* iks, int spin, const double* const* precond_d,
                      void* const* psi_h, int ldpsi, double* eig, double thr, int maxiter, int* iters) {
    return d.solve(nk, iks, spin, precond_d, psi_h, ldpsi, eig, thr, maxiter, iters);
}

}  // namespace b200

extern "C" int b200_solve_kpoints_batched(b200_hamilt* h, int nk, const int* iks, int spin, int nband, int david_ndim,
                                          int precision, const double* const* precond_d, void* const* psi_d, int ldpsi,
                                          double* eigenvalues, double thr, int maxiter, int* iters, void* stream) {
    return b200::guarded([&] {
        B200_CHECK(h && iks && precond_d && psi_d && eigenvalues, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(maxiter >= 1, b200::kInvalidArgument, "maxiter must be positive");
        B200_CHECK(nk >= 1 && nk <= b200::kMaxKBatch, b200::kInvalidArgument, "1..128 k-points per batch");
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        int dim_cap = 0;
        for (int q = 0; q < nk; ++q) {
            B200_CHECK(iks[q] >= 0 && iks[q] < int(h->h->grid->kmaps.size()), b200::kInvalidArgument,
                       "k-point index out of range");
            dim_cap = std::max(dim_cap, h->h->grid->kmaps[iks[q]].npw);
        }
        KBatchSolverCache& c = h->kbatch;
        if (!c.solver || c.cap < nk || c.nband != nband || c.ndim != david_ndim || c.dim_cap < dim_cap ||
            c.precision != precision || c.stream != s) {
            c.solver.reset();  // the old solver's buffers go before the new ones are made
            c.solver = b200::make_david_batch(h->h.get(), nk, nband, david_ndim, dim_cap, precision, s);
            c.cap = nk;
            c.nband = nband;
            c.ndim = david_ndim;
            c.dim_cap = dim_cap;
            c.precision = precision;
            c.stream = s;
        }
        b200::david_batch_solve(*c.solver, nk, iks, spin, precond_d, psi_d, ldpsi, eigenvalues, thr, maxiter, iters);
    });
}
