// Arithmetic peaks of this GPU, measured: FP64 and FP32 fused multiply-add chains on the CUDA cores, and
// FP64 tensor-core MMAs (mma.sync m8n8k4 f64, the instruction the FP64 GEMMs of the plain path issue).
// They are the denominators of the compute side of the rooflines (the FFT passes run on the FP64 / FP32
// pipes; the FP64 projector and subspace products on the FP64 tensor pipe).  No counterpart in the
// reference.
#include "capi_guard.h"
#include "common.h"

namespace b200 {
namespace {

constexpr int kPeakThreads = 256;
constexpr int kChains = 8;  // independent accumulators per thread (hides the pipe latency)

// each thread: kChains independent chains of `iters` FMAs a = a * m + c
template <typename R>
__global__ void __launch_bounds__(kPeakThreads) k_fma_chain(int iters, R m, R c, R* __restrict__ sink) {
    R a[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) a[j] = R(threadIdx.x + j);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < kChains; ++j) a[j] = fma(a[j], m, c);
    }
    R s = 0;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += a[j];
    if (s == R(-12345.678)) sink[blockIdx.x * kPeakThreads + threadIdx.x] = s;  // keeps the chains alive
}

// each warp: 4 independent accumulator tiles of m8n8k4 f64 MMAs, `iters` rounds
__global__ void __launch_bounds__(kPeakThreads) k_dmma_chain(int iters, double* __restrict__ sink) {
    const int lane = threadIdx.x & 31;
    double a = 1.0 + 1e-3 * lane, b = 1.0 - 1e-3 * lane;
    double d[4][2];
#pragma unroll
    for (int j = 0; j < 4; ++j) d[j][0] = d[j][1] = 0.0;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                         : "+d"(d[j][0]), "+d"(d[j][1])
                         : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) s += d[j][0] + d[j][1];
    if (s == -12345.678) sink[blockIdx.x * kPeakThreads + threadIdx.x] = s;
}

template <typename K> float time_ms(K launch) {
    cudaEvent_t e0, e1;
    B200_CUDA(cudaEventCreate(&e0));
    B200_CUDA(cudaEventCreate(&e1));
    launch();  // warm-up
    B200_CUDA(cudaEventRecord(e0, 0));
    launch();
    B200_CUDA(cudaEventRecord(e1, 0));
    B200_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    B200_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    B200_CUDA(cudaGetLastError());
    return ms;
}

}  // namespace
}  // namespace b200

extern "C" int b200_measure_peaks(double* fp64_tflops, double* fp32_tflops, double* dmma_tflops) {
    using namespace b200;
    return guarded([&] {
        B200_CHECK(fp64_tflops && fp32_tflops && dmma_tflops, kInvalidArgument, "NULL argument");
        int dev = 0, sms = 0;
        B200_CUDA(cudaGetDevice(&dev));
        B200_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int blocks = sms * 8;
        DeviceArray<double> sink(size_t(blocks) * kPeakThreads);
        const int it64 = 4096, it32 = 8192, itm = 2048;
        const float ms64 = time_ms([&] {
            k_fma_chain<double><<<blocks, kPeakThreads>>>(it64, 0.999999, 1e-7, sink.ptr);
            note_launch();
        });
        const float ms32 = time_ms([&] {
            k_fma_chain<float><<<blocks, kPeakThreads>>>(it32, 0.999999f, 1e-7f, reinterpret_cast<float*>(sink.ptr));
            note_launch();
        });
        const float msm = time_ms([&] {
            k_dmma_chain<<<blocks, kPeakThreads>>>(itm, sink.ptr);
            note_launch();
        });
        const double thr = double(blocks) * kPeakThreads;
        *fp64_tflops = 2.0 * kChains * it64 * thr / (ms64 * 1e-3) / 1e12;
        *fp32_tflops = 2.0 * kChains * it32 * thr / (ms32 * 1e-3) / 1e12;
        const double warps = thr / 32.0;
        *dmma_tflops = 2.0 * 8 * 8 * 4 * 4.0 * itm * warps / (msm * 1e-3) / 1e12;
    });
}
