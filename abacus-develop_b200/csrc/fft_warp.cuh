// Warp-synchronous mixed-radix FFT of a compile-time length N held in shared memory.
//
// One warp transforms one length-N vector in place, with only __syncwarp between
// passes (no block barrier).  The passes are the self-sorting Stockham passes of
// fft_core.cuh (same radix order 4,2,3,5 and the same host-built twiddle table),
// but with N, the radices and the products p known at compile time: every index
// is a constant expression and the per-lane butterflies of a pass are unrolled.
// Within a pass every lane first reads all its inputs into registers, the warp
// synchronises, then every lane writes its outputs to the same buffer -- so no
// second (ping-pong) buffer is needed.
#pragma once
#include "fft_core.cuh"

namespace b200 {

constexpr int fw_count(int n, int f) {
    int c = 0;
    while (n % f == 0) {
        n /= f;
        ++c;
    }
    return c;
}
// number of passes with the host plan's radix order (4s, then a 2, then 3s, then 5s)
constexpr int fw_npass(int n) {
    const int c2 = fw_count(n, 2);
    return c2 / 2 + (c2 % 2) + fw_count(n, 3) + fw_count(n, 5);
}
constexpr int fw_radix(int n, int j) {
    const int c2 = fw_count(n, 2);
    const int n4 = c2 / 2, n2 = c2 % 2, n3 = fw_count(n, 3);
    if (j < n4) return 4;
    j -= n4;
    if (j < n2) return 2;
    j -= n2;
    if (j < n3) return 3;
    return 5;
}
constexpr int fw_p(int n, int j) {
    int p = 1;
    for (int i = 0; i < j; ++i) p *= fw_radix(n, i);
    return p;
}
constexpr int fw_twoff(int n, int j) {
    int o = 0;
    for (int i = 0; i < j; ++i) o += fw_p(n, i) * (fw_radix(n, i) - 1);
    return o;
}
constexpr bool fw_smooth(int n) {
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    while (n % 5 == 0) n /= 5;
    return n == 1;
}

template <typename T, int DIR, int N, int PASS>
__device__ __forceinline__ void fw_pass(T* buf, int lane, const T* __restrict__ tw) {
    constexpr int R = fw_radix(N, PASS);
    constexpr int P = fw_p(N, PASS);
    constexpr int M = N / R;
    constexpr int PER = (M + 31) / 32;
    const T* t = tw + fw_twoff(N, PASS);
    T u[PER][R];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int i = lane + 32 * q;
        if (M % 32 == 0 || i < M) {
#pragma unroll
            for (int r = 0; r < R; ++r) u[q][r] = buf[i + r * M];
        }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int i = lane + 32 * q;
        if (M % 32 == 0 || i < M) {
            const int k = i % P;
            if (P > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    const T w = __ldg(t + k * (R - 1) + r - 1);
                    u[q][r] = DIR < 0 ? cmul(u[q][r], w) : cmulc(u[q][r], w);
                }
            }
            dftR<T, DIR, R>(u[q]);
            const int j = (i - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[j + r * P] = u[q][r];
        }
    }
    __syncwarp();
}

template <typename T, int DIR, int N, int PASS = 0>
__device__ __forceinline__ void fft_warp(T* buf, int lane, const T* __restrict__ tw) {
    if constexpr (PASS < fw_npass(N)) {
        fw_pass<T, DIR, N, PASS>(buf, lane, tw);
        fft_warp<T, DIR, N, PASS + 1>(buf, lane, tw);
    }
}

}  // namespace b200
