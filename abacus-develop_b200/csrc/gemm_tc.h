// Complex FP32 GEMM on tcgen05 tensor cores with 3xTF32 split precision (gemm_tc.cu).
#pragma once
#include <cuda_runtime.h>

#include "common.h"

namespace b200 {

struct TcGemmWorkspace {
    DeviceArray<float> ws;  // split-K partial tiles
    DeviceArray<int> err;   // nonzero after a bounded wait ran out inside the kernel
    void ensure();
    int read_error(cudaStream_t s = 0);  // read of the error word after the work queued on s
    size_t device_bytes() const { return ws.n * sizeof(float) + err.n * sizeof(int); }
};

// C (M x N) = alpha * op(A) * B + beta * C, complex64, column-major, op(A) in {'N', 'C'}.
// lda and ldb must be even and A, B 16-byte aligned (TMA row pitch).
void tc_cgemm(char opa, int M, int N, int K, float2 alpha, const float2* A, int lda, const float2* B, int ldb,
              float2 beta, float2* C, int ldc, TcGemmWorkspace& w, cudaStream_t s);

}  // namespace b200
