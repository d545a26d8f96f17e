// Complex FP32 GEMM on tcgen05 tensor cores with 3xTF32 split precision (gemm_tc.cu).
#pragma once
#include <cuda_runtime.h>

#include "common.h"

namespace b200 {

struct TcGemmWorkspace {
    DeviceArray<float> ws;  // split-K partial tiles
    DeviceArray<float2> bsplit;  // hi / lo halves of a B split once per call
    DeviceArray<int> err;   // nonzero after a bounded wait ran out inside the kernel
    size_t ws_cap = 0;      // floats; nonzero: split-K counts whose partial tiles exceed it are not used
    void ensure();
    // allocate up front (no allocation inside later calls whose workspace fits): split-K partial tiles of
    // at most ws_floats (also the cap), and a pre-split B of up to bsplit_elems complex values
    void reserve(size_t ws_floats, size_t bsplit_elems);
    int read_error(cudaStream_t s = 0);  // read (and clear) of the error word after the work queued on s
    size_t device_bytes() const { return ws.n * sizeof(float) + bsplit.n * sizeof(float2) + err.n * sizeof(int); }
};

// C (M x N) = alpha * op(A) * B + beta * C, complex64, column-major, op(A) in {'N', 'C'}.
// lda and ldb must be even and A, B 16-byte aligned (TMA row pitch).
void tc_cgemm(char opa, int M, int N, int K, float2 alpha, const float2* A, int lda, const float2* B, int ldb,
              float2 beta, float2* C, int ldc, TcGemmWorkspace& w, cudaStream_t s);

// Time limit of every pipeline wait inside the tensor-core GEMM kernels launched from now on, all threads
// (0 restores the default of 2 s).  A wait that runs out sets the workspace's error word.
void set_tc_wait_limit_ns(unsigned long long ns);
// the current limit (the tensor-core GEMMs of gemm_tc.cu and gemm_oz.cu both use it)
unsigned long long tc_wait_limit_ns();

}  // namespace b200
