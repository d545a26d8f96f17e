// The FP64 BLAS functors of the Davidson / nonlocal path as C-ABI drop-ins: gemm_op and gemv_op
// <std::complex<double>, DEVICE_GPU> (module_hsolver/kernels/cuda/math_kernel_op.cu:741-874) on cuBLAS, as
// the reference does, and dot_real_op<std::complex<T>, DEVICE_GPU> (:460-506), Re sum conj(L) R, as this
// library's own deterministic two-pass reduction (the reference calls cublas?dot on the 2*dim reals).
#include <cublas_v2.h>

#include "capi_guard.h"
#include "common.h"
#include "linalg_status.h"

namespace {

using b200::guarded;

// one cuBLAS handle per host thread and device, made at first use on that device (the reference keeps one
// static handle on its one device); a thread that moves between devices gets the current device's handle
struct ThreadBlas {
    static constexpr int kMaxDev = 64;
    cublasHandle_t h[kMaxDev] = {};
    ~ThreadBlas() {
        for (int d = 0; d < kMaxDev; ++d)
            if (h[d]) cublasDestroy(h[d]);
    }
    cublasHandle_t get(cudaStream_t s) {
        int dev = 0;
        B200_CUDA(cudaGetDevice(&dev));
        B200_CHECK(dev >= 0 && dev < kMaxDev, b200::kInvalidArgument, "device ordinal out of range");
        if (!h[dev]) B200_CUBLAS(cublasCreate(&h[dev]));
        B200_CUBLAS(cublasSetStream(h[dev], s));
        return h[dev];
    }
};
thread_local ThreadBlas g_blas;

bool op_of(char t, cublasOperation_t* op) {
    switch (t) {
        case 'N': case 'n': *op = CUBLAS_OP_N; return true;
        case 'T': case 't': *op = CUBLAS_OP_T; return true;
        case 'C': case 'c': *op = CUBLAS_OP_C; return true;
        default: return false;
    }
}

constexpr int kDotThreads = 256;
constexpr int kDotBlocks = 148 * 4;

// partial sums of Re(conj(L) R) per block (fixed order), then one block adds the partials in order
template <typename T>
__global__ void __launch_bounds__(kDotThreads) k_dot_partial(long n, const T* __restrict__ L, const T* __restrict__ R,
                                                             double* __restrict__ part) {
    __shared__ double s[kDotThreads / 32];
    double acc = 0.0;
    for (long i = blockIdx.x * long(kDotThreads) + threadIdx.x; i < n; i += long(gridDim.x) * kDotThreads)
        acc += double(L[i].x) * double(R[i].x) + double(L[i].y) * double(R[i].y);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kDotThreads / 32; ++w) t += s[w];
        part[blockIdx.x] = t;
    }
}

__global__ void k_dot_final(int nparts, const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double s[kDotThreads / 32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < int(blockDim.x) / 32; ++w) t += s[w];
        *out = t;
    }
}

// kDotBlocks partial sums and the result, per host thread and device (as the cuBLAS handles)
struct DotScratch {
    b200::DeviceArray<double> part[ThreadBlas::kMaxDev];
    b200::DeviceArray<double>& on_current_device() {
        int dev = 0;
        B200_CUDA(cudaGetDevice(&dev));
        B200_CHECK(dev >= 0 && dev < ThreadBlas::kMaxDev, b200::kInvalidArgument, "device ordinal out of range");
        return part[dev];
    }
};
thread_local DotScratch g_dot_scratch;

template <typename T> double dot_real(int dim, const void* l, const void* r, cudaStream_t s) {
    b200::DeviceArray<double>& part = g_dot_scratch.on_current_device();
    part.resize(kDotBlocks + 1);
    const long n = dim;
    k_dot_partial<T><<<kDotBlocks, kDotThreads, 0, s>>>(n, static_cast<const T*>(l), static_cast<const T*>(r),
                                                        part.ptr);
    b200::note_launch();
    B200_CUDA(cudaGetLastError());
    k_dot_final<<<1, kDotThreads, 0, s>>>(kDotBlocks, part.ptr, part.ptr + kDotBlocks);
    b200::note_launch();
    B200_CUDA(cudaGetLastError());
    double out = 0.0;
    B200_CUDA(cudaMemcpyAsync(&out, part.ptr + kDotBlocks, sizeof(double), cudaMemcpyDeviceToHost, s));
    B200_CUDA(cudaStreamSynchronize(s));
    return out;
}

}  // namespace

extern "C" {

int b200_gemm_op_f64(char transa, char transb, int m, int n, int k, const double* alpha, const void* a, int lda,
                     const void* b, int ldb, const double* beta, void* c, int ldc, void* stream) {
    return guarded([&] {
        cublasOperation_t oa, ob;
        B200_CHECK(op_of(transa, &oa) && op_of(transb, &ob), b200::kInvalidArgument, "trans must be N, T or C");
        B200_CHECK(alpha && beta && (m == 0 || n == 0 || (a && b && c)), b200::kInvalidArgument, "NULL argument");
        B200_CHECK(m >= 0 && n >= 0 && k >= 0, b200::kInvalidArgument, "negative dimension");
        if (m == 0 || n == 0) return;
        cublasHandle_t h = g_blas.get(reinterpret_cast<cudaStream_t>(stream));
        B200_CUBLAS(cublasZgemm(h, oa, ob, m, n, k, reinterpret_cast<const cuDoubleComplex*>(alpha),
                                static_cast<const cuDoubleComplex*>(a), lda, static_cast<const cuDoubleComplex*>(b), ldb,
                                reinterpret_cast<const cuDoubleComplex*>(beta), static_cast<cuDoubleComplex*>(c), ldc));
    });
}

int b200_gemv_op_f64(char trans, int m, int n, const double* alpha, const void* a, int lda, const void* x, int incx,
                     const double* beta, void* y, int incy, void* stream) {
    return guarded([&] {
        cublasOperation_t op;
        B200_CHECK(op_of(trans, &op), b200::kInvalidArgument, "trans must be N, T or C");
        B200_CHECK(alpha && beta && a && x && y, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(m >= 0 && n >= 0 && incx != 0 && incy != 0, b200::kInvalidArgument, "bad dimension or increment");
        cublasHandle_t h = g_blas.get(reinterpret_cast<cudaStream_t>(stream));
        B200_CUBLAS(cublasZgemv(h, op, m, n, reinterpret_cast<const cuDoubleComplex*>(alpha),
                                static_cast<const cuDoubleComplex*>(a), lda, static_cast<const cuDoubleComplex*>(x), incx,
                                reinterpret_cast<const cuDoubleComplex*>(beta), static_cast<cuDoubleComplex*>(y), incy));
    });
}

int b200_dot_real_op_f64(int dim, const void* psi_l, const void* psi_r, int reduce, double* result, void* stream) {
    return guarded([&] {
        B200_CHECK(psi_l && psi_r && result && dim >= 0, b200::kInvalidArgument, "NULL argument or negative dim");
        (void)reduce;  // one process per pool: the pool reduction is the identity
        *result = dot_real<double2>(dim, psi_l, psi_r, reinterpret_cast<cudaStream_t>(stream));
    });
}

int b200_dot_real_op_f32(int dim, const void* psi_l, const void* psi_r, int reduce, float* result, void* stream) {
    return guarded([&] {
        B200_CHECK(psi_l && psi_r && result && dim >= 0, b200::kInvalidArgument, "NULL argument or negative dim");
        (void)reduce;
        *result = float(dot_real<float2>(dim, psi_l, psi_r, reinterpret_cast<cudaStream_t>(stream)));
    });
}

}  // extern "C"
