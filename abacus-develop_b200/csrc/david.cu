// Block Davidson on the device, restating hsolver::DiagoDavid (diago_david.cpp:151-1240).
//
// Same iteration as the reference: Rayleigh-Ritz on the basis, residuals
// r_m = H x_m - lambda_m x_m of the unconverged bands (cal_grad :359-611),
// preconditioned by h_diag, orthogonalised and appended; the projected rows of
// hcc = basis^H H basis (cal_elem :626-717); the lowest nband eigenpairs of its
// lower triangle (diag_zhegvx :731-777); convergence |lambda_new - lambda_old|
// < thr per band (:270-280); restart through refresh (:797-934) when the basis
// would overflow nbase_x = david_ndim * nband; diag() retries (:1173-1240).
//
// B200 differences (same mathematics):
//  * the per-vector Gram-Schmidt (SchmidtOrth, :950-1075) becomes a block
//    classical Gram-Schmidt against the basis (two GEMMs) followed by
//    Cholesky-QR (twice) of the new block, with the Cholesky in FP64;
//  * S = I for norm-conserving pseudopotentials, so spsi aliases the basis and
//    scc (never read by the eigensolver) is not formed;
//  * no per-band cudaMalloc / host round trip; one small device-to-host copy of
//    the eigenvalues per iteration drives the host-side convergence test.
//  * mixed precision: the same iteration with FP32 vectors and FP32 GEMMs
//    (FP64 Cholesky and FP64 subspace eigensolve), then an FP64 Davidson from
//    the FP32 eigenvectors to the requested threshold.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.h"
#include "linalg_status.h"
#include "david.h"
#include "fft_core.cuh"
#include "gemm_oz.h"
#include "gemm_tc.h"

namespace b200 {

namespace {

constexpr int kT = 256;
inline int grid_of(long n) {
    long b = (n + kT - 1) / kT;
    if (b > 148L * 8) b = 148L * 8;
    return int(b < 1 ? 1 : b);
}

template <typename T, typename R>
__global__ void k_precond(long dim, long ld, int nc, T* __restrict__ v, const R* __restrict__ pc) {
    const long n = dim * nc;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const long m = i / dim;
        const long g = i - m * dim;
        const R p = pc[g];
        T* x = v + m * ld + g;
        *x = cmake<T>(x->x / p, x->y / p);
    }
}

// vc(:, m) = vcc(:nbase, unconv[m]); vcl(:, m) = -lambda_{unconv[m]} vc(:, m)
template <typename T>
__global__ void k_gather_cols(int nbase, int nbase_x, int nc, int ldv, const int* __restrict__ unconv,
                              const T* __restrict__ vcc, const double* __restrict__ w, T* __restrict__ vc,
                              T* __restrict__ vcl) {
    using R = typename RealOf<T>::type;
    const long n = long(nbase) * nc;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int m = int(i / nbase);
        const int r = int(i - long(m) * nbase);
        const int col = unconv[m];
        const T v = vcc[long(col) * nbase_x + r];
        vc[long(m) * ldv + r] = v;
        vcl[long(m) * ldv + r] = cscale(v, R(-w[col]));
    }
}

// squared norm of each of the nc columns of X (dim rows, stride ld), in FP64; one block per column
template <typename T>
__global__ void k_colnorm2(long dim, long ld, const T* __restrict__ X, double* __restrict__ out) {
    __shared__ double part[32];
    const T* x = X + long(blockIdx.x) * ld;
    double acc = 0.0;
    for (long g = threadIdx.x; g < dim; g += blockDim.x) acc += double(x[g].x) * x[g].x + double(x[g].y) * x[g].y;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) out[blockIdx.x] = acc;
    }
}

// flag = 1 if a column kept less than a quarter of its squared norm through the projection (G(j, j) is its
// squared norm after it, n2 before it): the projection cancelled most of the column, so what is left is
// dominated by rounding and needs a second pass ("twice is enough")
__global__ void k_reorth_flag(int nc, int ldg, const double2* __restrict__ G, const double* __restrict__ n2,
                              int* __restrict__ flag) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nc; j += gridDim.x * blockDim.x)
        if (G[long(j) * ldg + j].x < 0.25 * n2[j]) atomicOr(flag, 1);
}

template <typename T>
__global__ void k_refresh_diag(int nband, int nbase_x, const double* __restrict__ e, T* __restrict__ hcc,
                               T* __restrict__ vcc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nband; i += gridDim.x * blockDim.x) {
        hcc[long(i) * nbase_x + i] = cmake<T>(e[i], 0);
        vcc[long(i) * nbase_x + i] = cmake<T>(1, 0);
    }
}

template <typename A, typename B> __global__ void k_convert(long n, const A* __restrict__ a, B* __restrict__ b) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        b[i] = cmake<B>(a[i].x, a[i].y);
}

// subspace matrix -> FP64 eigensolver input (columns of ld, the leading nbase rows used); a non-finite entry
// there sets *flag
template <typename A>
__global__ void k_to_eig_input(int nbase, int ld, const A* __restrict__ a, double2* __restrict__ b, int* flag) {
    const long n = long(ld) * nbase;
    int bad = 0;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const double re = double(a[i].x), im = double(a[i].y);
        b[i] = make_double2(re, im);
        if (int(i % ld) < nbase && !(isfinite(re) && isfinite(im))) bad = 1;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}
// after k_to_eig_input flagged a non-finite entry: the eigensolver gets I instead (the solve is reported as a
// numerical error afterwards; the eigensolver never iterates on NaN/Inf)
__global__ void k_eig_input_guard(int nbase, int ld, const int* __restrict__ flag, double2* __restrict__ b) {
    if (*flag == 0) return;
    const long n = long(ld) * nbase;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        b[i] = make_double2(long(i % ld) == i / ld ? 1.0 : 0.0, 0.0);
}

template <typename R> __global__ void k_convert_real(long n, const double* __restrict__ a, R* __restrict__ b) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) b[i] = R(a[i]);
}

template <typename T> struct Lin;
template <> struct Lin<double2> {
    // cublasZgemm3m: the same bits as cublasZgemm on these shapes with B200's cuBLAS 12.9, 18-20 % faster
    static void gemm(cublasHandle_t h, cublasOperation_t a, cublasOperation_t b, int m, int n, int k, double2 al,
                     const double2* A, int lda, const double2* B, int ldb, double2 be, double2* C, int ldc) {
        B200_CUBLAS(cublasZgemm3m(h, a, b, m, n, k, (const cuDoubleComplex*)&al, (const cuDoubleComplex*)A, lda,
                                  (const cuDoubleComplex*)B, ldb, (const cuDoubleComplex*)&be, (cuDoubleComplex*)C, ldc));
    }
    static void herk(cublasHandle_t h, int n, int k, const double2* A, int lda, double2* C, int ldc) {
        const double one = 1.0, zero = 0.0;
        B200_CUBLAS(cublasZherk(h, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, n, k, &one, (const cuDoubleComplex*)A, lda, &zero,
                                  (cuDoubleComplex*)C, ldc));
    }
    static void trsm(cublasHandle_t h, int m, int n, const double2* U, int ldu, double2* X, int ldx) {
        const double2 one = make_double2(1.0, 0.0);
        B200_CUBLAS(cublasZtrsm(h, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, m, n,
                                  (const cuDoubleComplex*)&one, (const cuDoubleComplex*)U, ldu, (cuDoubleComplex*)X, ldx));
    }
};
template <> struct Lin<float2> {
    static void gemm(cublasHandle_t h, cublasOperation_t a, cublasOperation_t b, int m, int n, int k, float2 al,
                     const float2* A, int lda, const float2* B, int ldb, float2 be, float2* C, int ldc) {
        B200_CUBLAS(cublasCgemm(h, a, b, m, n, k, (const cuComplex*)&al, (const cuComplex*)A, lda, (const cuComplex*)B,
                                  ldb, (const cuComplex*)&be, (cuComplex*)C, ldc));
    }
    static void herk(cublasHandle_t h, int n, int k, const float2* A, int lda, float2* C, int ldc) {
        const float one = 1.f, zero = 0.f;
        B200_CUBLAS(cublasCherk(h, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, n, k, &one, (const cuComplex*)A, lda, &zero,
                                  (cuComplex*)C, ldc));
    }
    static void trsm(cublasHandle_t h, int m, int n, const float2* U, int ldu, float2* X, int ldx) {
        const float2 one = make_float2(1.f, 0.f);
        B200_CUBLAS(cublasCtrsm(h, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, m, n,
                                  (const cuComplex*)&one, (const cuComplex*)U, ldu, (cuComplex*)X, ldx));
    }
};

__global__ void k_identity(int n, int ld, double2* __restrict__ w) {
    const long total = long(n) * ld;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i / ld), r = int(i - long(c) * ld);
        w[i] = make_double2(r == c ? 1.0 : 0.0, 0.0);
    }
}

inline int even(int n) { return n + (n & 1); }

// Vectors of length dim are stored with stride ld (dim for FP64; dim rounded up to even for FP32 so
// that every block is a valid TMA operand of the tensor-core GEMM).
template <typename T> struct Engine {
    using R = typename RealOf<T>::type;
    static constexpr bool kF32 = std::is_same<T, float2>::value;
    int nband, dim, nbase_x, ld, L, ncp;
    int dim_cap;  // capacity: every buffer holds vectors of up to dim_cap entries
    cudaStream_t s = 0;
    cublasHandle_t cb = nullptr;
    cusolverDnHandle_t cs = nullptr;
    DeviceArray<T> basis, hp, newv, hcc, vcc, vc, vcl, lag, gram;
    DeviceArray<double2> A64, gram64, winv, work;
    DeviceArray<double> w, ein;
    DeviceArray<R> pc;
    DeviceArray<int> unconv_d, info;
    DeviceArray<double> cn2;  // FP32 engine: squared column norms before the projection
    int reorth = 0;           // FP32 engine: second projection passes taken (counted per solve)
    TcGemmWorkspace tcw;
    // FP64 engine: the subspace products on the int8 tensor cores (exact modular emulation of the FP64
    // products, gemm_oz.h) instead of cuBLAS ZGEMM; op(A) residues and products are workspaces grown at
    // first use.  0: cuBLAS; 1: the emulation for the products it is faster on; 2: for every product
    int oz = 0;
    // FP64 engine of a mixed solve: the start vectors are the FP32 stage's Ritz vectors (first try only)
    bool handover = false;
    int ntry_ = 0;
    OzOperand ozA;
    OzWorkspace ozw;
    int lwork = 0;
    std::vector<double> eig_h;
    std::vector<int> unconv_h;
    // page-locked copy of the unconverged-band list: its upload is an asynchronous copy (from pageable
    // memory the copy would wait for the stream first, one more host round trip per iteration)
    int* unconv_pin = nullptr;
    bool ref_refresh = true;
    int hpsi_bands = 0;
    int verbosity = 0;
    DavidTrace* trace = nullptr;
    void record() {
        if (trace) trace->record(kF32 ? 1 : 0, eig_h.data(), nband);
    }
    // verbosity >= 2: synchronising phase timers (seconds) for H|psi>, subspace GEMMs / orthogonalisation, eigensolve
    double t_hpsi = 0, t_lin = 0, t_eig = 0;
    std::chrono::steady_clock::time_point tmark;
    void tick() {
        if (verbosity >= 2) {
            B200_CUDA(cudaStreamSynchronize(s));
            tmark = std::chrono::steady_clock::now();
        }
    }
    void tock(double& acc) {
        if (verbosity >= 2) {
            B200_CUDA(cudaStreamSynchronize(s));
            acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - tmark).count();
            tmark = std::chrono::steady_clock::now();
        }
    }

    Engine(int nb, int d, int ndim, const double* precond_d)
        : nband(nb), dim(d), nbase_x(ndim * nb), ld(kF32 ? even(d) : d), L(even(ndim * nb)), ncp(even(nb)), dim_cap(d) {
        B200_CHECK(ndim > 1 && nb > 0 && ndim * nb < d, kInvalidArgument, "need david_ndim > 1 and david_ndim*nband < dim");
        B200_CUBLAS(cublasCreate(&cb));
        B200_CUSOLVER(cusolverDnCreate(&cs));
        B200_CUBLAS(cublasSetStream(cb, s));
        B200_CUSOLVER(cusolverDnSetStream(cs, s));
        basis.resize(size_t(nbase_x) * ld);
        hp.resize(size_t(nbase_x) * ld);
        newv.resize(size_t(nband) * ld);
        hcc.resize(size_t(nbase_x) * nbase_x);
        vcc.resize(size_t(nbase_x) * nbase_x);
        vc.resize(size_t(L) * nband);
        vcl.resize(size_t(L) * nband);
        lag.resize(size_t(L) * nband);
        gram.resize(size_t(ncp) * ncp);
        A64.resize(size_t(nbase_x) * nbase_x);
        gram64.resize(size_t(ncp) * ncp);
        winv.resize(size_t(ncp) * ncp);
        w.resize(nbase_x);
        ein.resize(nband);
        pc.resize(dim);
        unconv_d.resize(nband);
        info.resize(5);  // eigensolver, Cholesky, cancellation, non-finite flags; the GEMMs' wait error word
        if constexpr (kF32) cn2.resize(nband);
        B200_CUDA(cudaMemsetAsync(hcc.ptr, 0, hcc.n * sizeof(T), s));
        B200_CUDA(cudaMemsetAsync(vcc.ptr, 0, vcc.n * sizeof(T), s));
        B200_CUDA(cudaMemsetAsync(basis.ptr, 0, basis.n * sizeof(T), s));
        B200_CUDA(cudaMemsetAsync(hp.ptr, 0, hp.n * sizeof(T), s));
        B200_CUDA(cudaMemsetAsync(newv.ptr, 0, newv.n * sizeof(T), s));
        B200_CUDA(cudaMemsetAsync(info.ptr, 0, 5 * sizeof(int), s));
        if constexpr (std::is_same<R, double>::value) {
            B200_CUDA(cudaMemcpyAsync(pc.ptr, precond_d, dim * sizeof(double), cudaMemcpyDeviceToDevice, s));
        } else {
            k_convert_real<R><<<grid_of(dim), kT, 0, s>>>(dim, precond_d, pc.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
        }
        int l1 = 0, l2 = 0, l3 = 0, meig = 0;
        B200_CUSOLVER(cusolverDnZheevd_bufferSize(cs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nbase_x,
                                                  (cuDoubleComplex*)A64.ptr, nbase_x, w.ptr, &l1));
        B200_CUSOLVER(cusolverDnZheevdx_bufferSize(cs, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I,
                                                   CUBLAS_FILL_MODE_LOWER, nbase_x, (cuDoubleComplex*)A64.ptr, nbase_x,
                                                   0.0, 0.0, 1, nband, &meig, w.ptr, &l3));
        l1 = l1 > l3 ? l1 : l3;
        B200_CUSOLVER(cusolverDnZpotrf_bufferSize(cs, CUBLAS_FILL_MODE_UPPER, nband, (cuDoubleComplex*)gram64.ptr, ncp, &l2));
        lwork = l1 > l2 ? l1 : l2;
        work.resize(size_t(lwork > 0 ? lwork : 1));
        eig_h.assign(nbase_x, 0.0);
        unconv_h.assign(nband, 0);
        B200_CUDA(cudaHostAlloc(&unconv_pin, size_t(nband) * sizeof(int), cudaHostAllocDefault));
        if constexpr (kF32) {
            // tensor-core GEMM workspaces for every subspace product of this engine, so that a solve allocates
            // nothing: split-K partial tiles of up to 16 splits of the largest C (nband x nbase_x), and B split
            // once per call for the tall products (K <= nbase_x, N <= nband)
            tcw.reserve(size_t(16) * 2 * size_t(nband) * nbase_x, size_t(2) * size_t(nbase_x + 1) * nband);
        }
        B200_CUDA(cudaStreamSynchronize(s));
    }
    // Re-use the buffers for vectors of length d <= dim_cap (another k-point of the same cell) with its
    // preconditioner; nothing is allocated.
    void retarget(int d, const double* precond_d) {
        B200_CHECK(d <= dim_cap && nbase_x < d, kInvalidArgument, "retarget: need david_ndim*nband < dim <= capacity");
        dim = d;
        ld = kF32 ? even(d) : d;
        if constexpr (std::is_same<R, double>::value) {
            B200_CUDA(cudaMemcpyAsync(pc.ptr, precond_d, dim * sizeof(double), cudaMemcpyDeviceToDevice, s));
        } else {
            k_convert_real<R><<<grid_of(dim), kT, 0, s>>>(dim, precond_d, pc.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
        }
    }
    size_t device_bytes() const {
        return (basis.n + hp.n + newv.n + hcc.n + vcc.n + vc.n + vcl.n + lag.n + gram.n) * sizeof(T) +
               (A64.n + gram64.n + winv.n + work.n) * sizeof(double2) + (w.n + ein.n) * sizeof(double) +
               pc.n * sizeof(R) + tcw.device_bytes() + ozA.device_bytes() + ozw.device_bytes();
    }
    ~Engine() {
        if (unconv_pin) cudaFreeHost(unconv_pin);
        if (cb) cublasDestroy(cb);
        if (cs) cusolverDnDestroy(cs);
    }
    void set_stream(cudaStream_t st) {
        B200_CUDA(cudaStreamSynchronize(s));
        s = st;
        B200_CUBLAS(cublasSetStream(cb, s));
        B200_CUSOLVER(cusolverDnSetStream(cs, s));
    }

    // C = al op(A) B + be C; FP32 operands go to the tensor cores (3xTF32) whenever they are valid TMA operands
    // verbosity >= 3: every GEMM and H|psi> call timed on its own (synchronising); calls over 20 ms reported
    struct SlowCall {
        Engine* e;
        const char* what;
        int m, n, k;
        std::chrono::steady_clock::time_point t0;
        SlowCall(Engine* en, const char* w, int m_, int n_, int k_) : e(en), what(w), m(m_), n(n_), k(k_) {
            if (e->verbosity >= 3) {
                cudaStreamSynchronize(e->s);
                t0 = std::chrono::steady_clock::now();
            }
        }
        ~SlowCall() {
            if (e->verbosity >= 3) {
                cudaStreamSynchronize(e->s);
                const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                if (dt > 0.02)
                    std::fprintf(stderr, "[david %s] slow %s m %d n %d k %d: %.3f s\n", kF32 ? "fp32" : "fp64", what, m, n,
                                 k, dt);
            }
        }
    };

    void gemm(cublasOperation_t a, cublasOperation_t b, int m, int n, int k, T al, const T* A, int lda, const T* B,
              int ldb, T be, T* C, int ldc) {
        if (m <= 0 || n <= 0) return;
        SlowCall sc(this, a == CUBLAS_OP_N ? "gemm N" : "gemm C", m, n, k);
        if constexpr (kF32) {
            const bool aligned = ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) == 0;
            if (k > 0 && b == CUBLAS_OP_N && (a == CUBLAS_OP_N || a == CUBLAS_OP_C) && lda % 2 == 0 && ldb % 2 == 0 &&
                aligned) {
                tc_cgemm(a == CUBLAS_OP_N ? 'N' : 'C', m, n, k, al, A, lda, B, ldb, be, C, ldc, tcw, s);
                return;
            }
        } else {
            // the emulation reduces both operands to residues in every call (work ~ (m + n) k) against m n k
            // products: it pays from m n / (m + n) of about 256 on (B200: a 51 627 x 160 x 512 product is
            // slower than cuBLAS, 124 289 x 480 x 480 1.4x and 480 x 1920 x 124 289 2x faster)
            if (oz && k > 0 && b == CUBLAS_OP_N && (a == CUBLAS_OP_N || a == CUBLAS_OP_C) &&
                (oz == 2 || (k >= 128 && double(m) * n / (double(m) + n) >= 256.0))) {
                const char opa = a == CUBLAS_OP_N ? 'N' : 'C';
                oz_prepare_a(opa, m, k, A, lda, kOzMaxMods, ozA, ozw, s);
                oz_zgemm(opa, m, n, k, al, ozA, B, ldb, be, C, ldc, ozw, nullptr, s);
                return;
            }
        }
        Lin<T>::gemm(cb, a, b, m, n, k, al, A, lda, B, ldb, be, C, ldc);
    }

    // X (dim x nc, stride ld) <- X U^-1 with X^H X = U^H U, U from an FP64 Cholesky; with check, info[2] is
    // set when a column's squared norm fell below a quarter of cn2 (its value before a projection)
    void cholqr(T* X, int nc, bool check = false) {
        const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
        const long n2 = long(ncp) * nc;
        double2* G = gram64.ptr;
        if constexpr (!kF32) {
            Lin<T>::herk(cb, nc, dim, X, ld, gram.ptr, ncp);
            B200_CUDA(cudaMemcpyAsync(G, gram.ptr, n2 * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        } else {
            gemm(CUBLAS_OP_C, CUBLAS_OP_N, nc, nc, dim, one, X, ld, X, ld, zero, gram.ptr, ncp);
            k_convert<T, double2><<<grid_of(n2), kT, 0, s>>>(n2, gram.ptr, G);
            note_launch();
            B200_CUDA(cudaGetLastError());
        }
        if (check) {
            k_reorth_flag<<<grid_of(nc), kT, 0, s>>>(nc, ncp, G, cn2.ptr, info.ptr + 2);
            note_launch();
            B200_CUDA(cudaGetLastError());
        }
        B200_CUSOLVER(cusolverDnZpotrf(cs, CUBLAS_FILL_MODE_UPPER, nc, (cuDoubleComplex*)G, ncp, (cuDoubleComplex*)work.ptr,
                                       lwork, info.ptr + 1));
        if constexpr (!kF32) {
            Lin<T>::trsm(cb, dim, nc, G, ncp, X, ld);
        } else {
            // U^-1 in FP64 (triangular solve against I), then X U^-1 as one tensor-core GEMM
            k_identity<<<grid_of(n2), kT, 0, s>>>(nc, ncp, winv.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
            const double2 done = make_double2(1.0, 0.0);
            B200_CUBLAS(cublasZtrsm(cb, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, nc, nc,
                                      (const cuDoubleComplex*)&done, (const cuDoubleComplex*)G, ncp,
                                      (cuDoubleComplex*)winv.ptr, ncp));
            k_convert<double2, T><<<grid_of(n2), kT, 0, s>>>(n2, winv.ptr, gram.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
            gemm(CUBLAS_OP_N, CUBLAS_OP_N, dim, nc, nc, one, X, ld, gram.ptr, ncp, zero, newv.ptr, ld);
            B200_CUDA(cudaMemcpyAsync(X, newv.ptr, size_t(nc) * ld * sizeof(T), cudaMemcpyDeviceToDevice, s));
        }
    }

    // orthonormalise X (dim x nc) against basis[:, :nprev] and within itself: block classical Gram-Schmidt
    // and Cholesky-QR, twice in the FP64 engine; the FP32 engine (whose result is refined in FP64) takes the
    // second pass on blocks of 128 bands or more only when the first projection cancelled most of some
    // column or its Cholesky failed.  The reference orthogonalises each new vector once
    // (diago_david.cpp, SchmidtOrth); the 216-atom FP32 stage runs the same iterations with one pass as with
    // two and 10 % faster.
    // one_pass: X is orthonormal to a few ulps of the lower precision already (the Ritz vectors the FP32 stage
    // of a mixed solve hands over): one Cholesky-QR pass brings it to FP64 orthonormality
    void orth_block(T* X, int nc, int nprev, bool one_pass = false) {
        const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0), mone = cmake<T>(-1, 0);
        // small blocks always take both passes: their products are latency-bound, the second pass costs
        // little, and k-point solves of 32 bands took 15 % more iterations with one
        const bool adaptive = kF32 && nprev > 0 && nband >= 128;
        if (adaptive) {
            k_colnorm2<T><<<nc, 256, 0, s>>>(dim, ld, X, cn2.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
            B200_CUDA(cudaMemsetAsync(info.ptr + 2, 0, sizeof(int), s));
        }
        for (int pass = 0; pass < 2; ++pass) {
            if (nprev > 0) {
                gemm(CUBLAS_OP_C, CUBLAS_OP_N, nprev, nc, dim, one, basis.ptr, ld, X, ld, zero, lag.ptr, L);
                gemm(CUBLAS_OP_N, CUBLAS_OP_N, dim, nc, nprev, mone, basis.ptr, ld, lag.ptr, L, one, X, ld);
            }
            cholqr(X, nc, adaptive && pass == 0);
            if (one_pass) break;
            if (adaptive && pass == 0) {
                int fl[2] = {0, 0};  // Cholesky info, cancellation flag: either asks for the second pass
                B200_CUDA(cudaMemcpyAsync(fl, info.ptr + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
                B200_CUDA(cudaStreamSynchronize(s));
                if (!fl[0] && !fl[1]) break;
                ++reorth;
            }
        }
    }

    void cal_elem(int nbase, int nc) {
        const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
        gemm(CUBLAS_OP_C, CUBLAS_OP_N, nc, nbase + nc, dim, one, basis.ptr + size_t(nbase) * ld, ld, hp.ptr, ld, zero,
             hcc.ptr + nbase, nbase_x);
    }

    void eigsolve(int nbase) {
        tick();
        const long n = long(nbase_x) * nbase;
        k_to_eig_input<T><<<grid_of(n), kT, 0, s>>>(nbase, nbase_x, hcc.ptr, A64.ptr, info.ptr + 3);
        k_eig_input_guard<<<grid_of(n), kT, 0, s>>>(nbase, nbase_x, info.ptr + 3, A64.ptr);
        note_launch(2);
        B200_CUDA(cudaGetLastError());
        // lowest nband eigenpairs only (the reference's zheevx range 'I', dngvd_op.cpp:142-235): divide and
        // conquer on the tridiagonal form, back-transforming nband vectors instead of nbase
        if (nbase > nband) {
            int meig = 0;
            B200_CUSOLVER(cusolverDnZheevdx(cs, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_LOWER,
                                            nbase, (cuDoubleComplex*)A64.ptr, nbase_x, 0.0, 0.0, 1, nband, &meig, w.ptr,
                                            (cuDoubleComplex*)work.ptr, lwork, info.ptr));
        } else {
            B200_CUSOLVER(cusolverDnZheevd(cs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nbase,
                                           (cuDoubleComplex*)A64.ptr, nbase_x, w.ptr, (cuDoubleComplex*)work.ptr, lwork,
                                           info.ptr));
        }
        const long nv = long(nbase_x) * nband;
        if constexpr (std::is_same<T, double2>::value) {
            B200_CUDA(cudaMemcpyAsync(vcc.ptr, A64.ptr, nv * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        } else {
            k_convert<double2, T><<<grid_of(nv), kT, 0, s>>>(nv, A64.ptr, vcc.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
        }
        // the tensor-core GEMMs' error word travels with the flags: one host round trip for all of them
        int* gemm_err = nullptr;
        if constexpr (kF32) gemm_err = tcw.err.ptr;
        else if (oz) gemm_err = ozw.err.ptr;
        if (gemm_err)
            B200_CUDA(cudaMemcpyAsync(info.ptr + 4, gemm_err, sizeof(int), cudaMemcpyDeviceToDevice, s));
        else
            B200_CUDA(cudaMemsetAsync(info.ptr + 4, 0, sizeof(int), s));
        int hinfo[5];
        B200_CUDA(cudaMemcpyAsync(eig_h.data(), w.ptr, nband * sizeof(double), cudaMemcpyDeviceToHost, s));
        B200_CUDA(cudaMemcpyAsync(hinfo, info.ptr, 5 * sizeof(int), cudaMemcpyDeviceToHost, s));
        B200_CUDA(cudaStreamSynchronize(s));
        if (hinfo[4] != 0) {
            B200_CUDA(cudaMemsetAsync(gemm_err, 0, sizeof(int), s));  // read once, then cleared
            B200_CUDA(cudaStreamSynchronize(s));
            throw Error(kCudaError, std::string(kF32 ? "tensor-core" : "int8 tensor-core") +
                                        " GEMM wait ran out (error word " + std::to_string(hinfo[4]) + ")");
        }
        B200_CHECK(hinfo[3] == 0, kNumericalError,
                   "non-finite entries in the subspace matrix (NaN/Inf in psi, V_eff, D or H|psi>)");
        B200_CHECK(hinfo[1] == 0, kNumericalError,
                   "Cholesky of the new block failed (linearly dependent search directions), info " + std::to_string(hinfo[1]));
        B200_CHECK(hinfo[0] == 0, kNumericalError, "subspace eigensolver failed, info " + std::to_string(hinfo[0]));
        for (int m = 0; m < nband; ++m)
            B200_CHECK(std::isfinite(eig_h[m]), kNumericalError, "non-finite eigenvalue (NaN/Inf in H|psi> or psi)");
        tock(t_eig);
    }

    void cal_grad(const HPsiDevice& f, int nbase, int nc) {
        const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
        tick();
        // the previous upload from unconv_pin completed before the last eigensolve's results were read
        std::memcpy(unconv_pin, unconv_h.data(), size_t(nc) * sizeof(int));
        B200_CUDA(cudaMemcpyAsync(unconv_d.ptr, unconv_pin, nc * sizeof(int), cudaMemcpyHostToDevice, s));
        k_gather_cols<T><<<grid_of(long(nbase) * nc), kT, 0, s>>>(nbase, nbase_x, nc, L, unconv_d.ptr, vcc.ptr, w.ptr,
                                                                  vc.ptr, vcl.ptr);
        note_launch();
        B200_CUDA(cudaGetLastError());
        T* X = basis.ptr + size_t(nbase) * ld;
        gemm(CUBLAS_OP_N, CUBLAS_OP_N, dim, nc, nbase, one, hp.ptr, ld, vc.ptr, L, zero, X, ld);
        gemm(CUBLAS_OP_N, CUBLAS_OP_N, dim, nc, nbase, one, basis.ptr, ld, vcl.ptr, L, one, X, ld);
        k_precond<T, R><<<grid_of(long(dim) * nc), kT, 0, s>>>(dim, ld, nc, X, pc.ptr);
        note_launch();
        B200_CUDA(cudaGetLastError());
        orth_block(X, nc, nbase);
        tock(t_lin);
        {
            SlowCall sc(this, "hpsi", dim, nc, 0);
            f(basis.ptr, hp.ptr + size_t(nbase) * ld, nbase_x, ld, nbase, nbase + nc - 1, s);
        }
        hpsi_bands += nc;
        tock(t_hpsi);
    }

    void refresh(int nbase, const double* eig_in, T* psi, int ldpsi) {
        const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
        gemm(CUBLAS_OP_N, CUBLAS_OP_N, dim, nband, nbase, one, hp.ptr, ld, vcc.ptr, nbase_x, zero, newv.ptr, ld);
        B200_CUDA(cudaMemcpyAsync(hp.ptr, newv.ptr, size_t(nband) * ld * sizeof(T), cudaMemcpyDeviceToDevice, s));
        B200_CUDA(cudaMemcpy2DAsync(basis.ptr, ld * sizeof(T), psi, size_t(ldpsi) * sizeof(T), dim * sizeof(T), nband,
                                    cudaMemcpyDeviceToDevice, s));
        B200_CUDA(cudaMemsetAsync(hcc.ptr, 0, hcc.n * sizeof(T), s));
        if (!ref_refresh) B200_CUDA(cudaMemsetAsync(vcc.ptr, 0, vcc.n * sizeof(T), s));
        B200_CUDA(cudaMemcpyAsync(ein.ptr, eig_in, nband * sizeof(double), cudaMemcpyHostToDevice, s));
        k_refresh_diag<T><<<grid_of(nband), kT, 0, s>>>(nband, nbase_x, ein.ptr, hcc.ptr, vcc.ptr);
        note_launch();
        B200_CUDA(cudaGetLastError());
    }

    int diag_once(const HPsiDevice& f, int ldpsi, T* psi, double* eig_in, double thr, int maxiter, int& notconv) {
        const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
        B200_CUDA(cudaMemsetAsync(info.ptr, 0, 5 * sizeof(int), s));
        B200_CUDA(cudaMemcpy2DAsync(basis.ptr, ld * sizeof(T), psi, size_t(ldpsi) * sizeof(T), dim * sizeof(T), nband,
                                    cudaMemcpyDeviceToDevice, s));
        orth_block(basis.ptr, nband, 0, handover && ntry_ == 0);
        f(basis.ptr, hp.ptr, nbase_x, ld, 0, nband - 1, s);
        hpsi_bands += nband;
        cal_elem(0, nband);
        int nbase = nband;
        eigsolve(nbase);
        record();
        for (int m = 0; m < nband; ++m) eig_in[m] = eig_h[m];
        notconv = nband;
        for (int m = 0; m < nband; ++m) unconv_h[m] = m;
        int iter = 0;
        while (true) {
            ++iter;
            cal_grad(f, nbase, notconv);
            tick();
            cal_elem(nbase, notconv);
            tock(t_lin);
            nbase += notconv;
            eigsolve(nbase);
            record();
            notconv = 0;
            double dmax = 0.0;
            for (int m = 0; m < nband; ++m) {
                const double de = std::fabs(eig_h[m] - eig_in[m]);
                dmax = de > dmax ? de : dmax;
                if (!(de < thr)) unconv_h[notconv++] = m;
                eig_in[m] = eig_h[m];
            }
            if (verbosity > 0)
                std::fprintf(stderr,
                             "[david %s] iter %3d nbase %4d notconv %4d max|dE| %.3e  t(hpsi/lin/eig) %.3f %.3f %.3f  "
                             "second passes %d\n",
                             kF32 ? "fp32" : "fp64", iter, nbase, notconv, dmax, t_hpsi, t_lin, t_eig, reorth);
            if (notconv == 0 || nbase + notconv > nbase_x || iter == maxiter) {
                B200_CUDA(cudaMemsetAsync(psi, 0, size_t(nband) * ldpsi * sizeof(T), s));
                gemm(CUBLAS_OP_N, CUBLAS_OP_N, dim, nband, nbase, one, basis.ptr, ld, vcc.ptr, nbase_x, zero, psi, ldpsi);
                if (notconv == 0 || iter == maxiter) break;
                refresh(nbase, eig_in, psi, ldpsi);
                nbase = nband;
            }
        }
        B200_CUDA(cudaStreamSynchronize(s));
        return iter;
    }

    int diag(const HPsiDevice& f, int ldpsi, T* psi, double* eig, double thr, int maxiter, int ntry_max, int notconv_max,
             int& notconv) {
        int ntry = 0, total = 0;
        notconv = 0;
        ntry_ = 0;
        reorth = 0;
        // a fresh subspace, as a newly constructed DiagoDavid has (diago_david.cpp:34-148): the refresh reads
        // columns of vcc that this solve may not have written, so a reused solver must start from zeros
        B200_CUDA(cudaMemsetAsync(hcc.ptr, 0, hcc.n * sizeof(T), s));
        B200_CUDA(cudaMemsetAsync(vcc.ptr, 0, vcc.n * sizeof(T), s));
        do {
            total += diag_once(f, ldpsi, psi, eig, thr, maxiter, notconv);
            ++ntry;
            ntry_ = ntry;
        } while (!(ntry > ntry_max || notconv <= notconv_max));
        return total;
    }
};

class David : public DavidBase {
  public:
    David(int nband, int dim, int ndim, int precision, const double* precond_d)
        : nband_(nband), dim_(dim), cap_(dim), ndim_(ndim), precision_(precision) {
        B200_CHECK(precision == 0 || precision == 1, kInvalidArgument, "bad precision");
        pc_.resize(dim);
        B200_CUDA(cudaMemcpy(pc_.ptr, precond_d, dim * sizeof(double), cudaMemcpyDeviceToDevice));
        e64_ = std::make_unique<Engine<double2>>(nband, dim, ndim, pc_.ptr);
        // a mixed solver holds its FP32 engine from the start: every allocation happens here, as the
        // reference's constructor does (diago_david.cpp:34-148), not inside a solve
        if (precision == 1) {
            e32_ = std::make_unique<Engine<float2>>(nband, dim, ndim, pc_.ptr);
            psi32_.resize(size_t(nband) * dim);  // FP32 copy of psi for ldpsi == dim (grown only for a wider ldpsi)
        }
    }
    int diag(const HPsiDevice& f64, int ldpsi, void* psi, double* eig, double thr, int maxiter, int ntry_max,
             int notconv_max) override {
        B200_CHECK(precision_ == 0, kInvalidArgument, "a mixed-precision solve needs a Hamiltonian handle");
        stats_ = DavidStats{};
        trace_.reset();
        e64_->trace = &trace_;
        e64_->hpsi_bands = 0;
        e64_->oz = fp64_gemm_ == 3 ? 2 : fp64_gemm_ == 2 ? 1 : 0;
        e64_->handover = false;
        int nc = 0;
        const int it = e64_->diag(f64, ldpsi, (double2*)psi, eig, thr, maxiter, ntry_max, notconv_max, nc);
        stats_.iters_fp64 = it;
        stats_.hpsi_bands = e64_->hpsi_bands;
        notconv_ = nc;
        return it;
    }
    int diag_hamilt(const HPsiDevice& f64, const HPsiDevice& f32, int precision, int ldpsi, void* psi, double* eig,
                    double thr, int maxiter, int ntry_max, int notconv_max) override {
        stats_ = DavidStats{};
        trace_.reset();
        e64_->trace = &trace_;
        int total = 0, nc = 0;
        if (precision == 1) {
            if (!e32_) {
                // the engine's constructor works on the legacy stream: let the writes of pc_ queued on the
                // solver's stream finish first, then re-target on that stream (the current k-point's
                // preconditioner, in stream order)
                B200_CUDA(cudaStreamSynchronize(stream_));
                e32_ = std::make_unique<Engine<float2>>(nband_, cap_, low_ndim_ > 0 ? low_ndim_ : ndim_, pc_.ptr);
                e32_->set_stream(stream_);
                e32_->retarget(dim_, pc_.ptr);
            }
            // the FP32 stage of a block of 128 bands or more restarts from the exact Ritz basis (vcc = I): with
            // the reference's stale off-diagonal vcc entries the first residuals after each restart are those of
            // mixed vectors (the 216-atom stage ran 20 % longer); smaller blocks keep the reference's refresh,
            // with which 32-band k-point solves took 25 iterations instead of 29
            e32_->ref_refresh = e64_->ref_refresh && nband_ < 128;
            e32_->trace = &trace_;
            e32_->verbosity = verbosity_;
            e32_->hpsi_bands = 0;
            psi32_.resize(size_t(nband_) * ldpsi);
            const long n = long(nband_) * ldpsi;
            k_convert<double2, float2><<<grid_of(n), kT, 0, stream_>>>(n, (const double2*)psi, psi32_.ptr);
            note_launch();
            B200_CUDA(cudaGetLastError());
            const double t32 = thr > mixed_thr_ ? thr : mixed_thr_;
            const int it32 = e32_->diag(f32, ldpsi, psi32_.ptr, eig, t32, maxiter, 0, nband_, nc);
            k_convert<float2, double2><<<grid_of(n), kT, 0, stream_>>>(n, psi32_.ptr, (double2*)psi);
            note_launch();
            B200_CUDA(cudaGetLastError());
            stats_.iters_low = it32;
            stats_.hpsi_bands += e32_->hpsi_bands;
            total += it32;
        }
        e64_->hpsi_bands = 0;
        e64_->oz = fp64_gemm_ == 3 ? 2 : (fp64_gemm_ == 2 || (fp64_gemm_ == 1 && precision == 1)) ? 1 : 0;
        e64_->handover = precision == 1;
        const int it64 = e64_->diag(f64, ldpsi, (double2*)psi, eig, thr, maxiter, ntry_max, notconv_max, nc);
        stats_.iters_fp64 = it64;
        stats_.hpsi_bands += e64_->hpsi_bands;
        notconv_ = nc;
        return total + it64;
    }
    const DavidStats& stats() const override { return stats_; }
    DavidTrace& trace() override { return trace_; }
    void set_mixed_thr(double thr) override { mixed_thr_ = thr; }
    void set_low_ndim(int ndim) override {
        B200_CHECK(ndim >= 2, kInvalidArgument, "david_ndim of the FP32 stage must be at least 2");
        if (ndim != (low_ndim_ > 0 ? low_ndim_ : ndim_)) e32_.reset();  // rebuilt at the next mixed solve
        low_ndim_ = ndim;
    }
    int precision() const override { return precision_; }
    void set_stream(cudaStream_t st) override {
        stream_ = st;
        e64_->set_stream(st);
        if (e32_) e32_->set_stream(st);
    }
    void set_verbosity(int level) override {
        verbosity_ = level;
        e64_->verbosity = level;
        if (e32_) e32_->verbosity = level;
    }
    void retarget(int dim, const double* precond_d) override {
        B200_CHECK(dim <= cap_, kInvalidArgument, "retarget beyond the solver's capacity");
        B200_CUDA(cudaMemcpyAsync(pc_.ptr, precond_d, dim * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        dim_ = dim;
        e64_->retarget(dim, pc_.ptr);
        if (e32_) e32_->retarget(dim, pc_.ptr);
    }
    size_t device_bytes() const override {
        size_t b = pc_.n * sizeof(double) + psi32_.n * sizeof(float2) + e64_->device_bytes();
        if (e32_) b += e32_->device_bytes();
        return b;
    }
    // the reference's refresh (stale off-diagonal vcc entries) for the FP64 iteration; the FP32 stage of a
    // mixed solve always restarts cleanly
    void set_reference_refresh(bool on) override { e64_->ref_refresh = on; }
    void set_fp64_gemm(int mode) override {
        B200_CHECK(mode >= 0 && mode <= 3, kInvalidArgument, "FP64 GEMM mode must be 0, 1, 2 or 3");
        fp64_gemm_ = mode;
    }

  private:
    int nband_, dim_, cap_, ndim_, precision_;
    int notconv_ = 0;
    int verbosity_ = 0;
    cudaStream_t stream_ = 0;
    double mixed_thr_ = 1e-7;
    int low_ndim_ = 0;
    int fp64_gemm_ = 0;
    DeviceArray<double> pc_;
    DeviceArray<float2> psi32_;
    std::unique_ptr<Engine<double2>> e64_;
    std::unique_ptr<Engine<float2>> e32_;
    DavidStats stats_;
    DavidTrace trace_;
};

}  // namespace

std::unique_ptr<DavidBase> make_david(int nband, int dim, int david_ndim, int precision, const double* precond_d) {
    return std::make_unique<David>(nband, dim, david_ndim, precision, precond_d);
}

}  // namespace b200
