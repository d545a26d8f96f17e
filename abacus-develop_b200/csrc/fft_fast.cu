// Warp-synchronous forms of the three fused local H|psi> passes for the grid sizes
// of the standard workloads (18, 36, 45, 90, 96, 125, 128 along z; square xy
// planes of 18, 36, 45, 96, 125, 128).  Same data layouts and results as the
// generic kernels in fft_kernels.cu; each 1-D transform is done by one warp with
// compile-time radices (fft_warp.cuh), so a CTA needs only a handful of block
// barriers.  Other sizes use the generic kernels.
#include "fft_warp.cuh"
#include "plane_t.cuh"
#include "pw_grid.h"

namespace b200 {

namespace {

template <typename T> __device__ __forceinline__ T zero_c() { return cmake<T>(0, 0); }

constexpr int kZWarps = 8;       // z passes: 8 warps, 16 sticks per CTA
constexpr int kPlaneWarps = 16;  // plane pass: 16 warps per (band, z)

template <typename T, int NZ>
__global__ void __launch_bounds__(kZWarps * 32) k_zinv_w(StickMapView sm, const T* __restrict__ twz,
                                                        const T* __restrict__ psi, int ld, T* __restrict__ sb) {
    constexpr int LDZ = NZ | 1;
    __shared__ T A[kStickTile * LDZ];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int s0 = blockIdx.x * kStickTile;
    const int ns = min(kStickTile, sm.nst - s0);
    const int band = blockIdx.y;
    for (int i = tid; i < kStickTile * LDZ; i += kZWarps * 32) A[i] = zero_c<T>();
    __syncthreads();
    const T* p = psi + size_t(band) * ld;
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    for (int j = j0 + tid; j < j1; j += kZWarps * 32) {
        const int pk = sm.gpk[j];
        A[((pk >> 10) - s0) * LDZ + (pk & 1023)] = p[sm.glist[j]];
    }
    __syncthreads();
    for (int sl = warp; sl < ns; sl += kZWarps) fft_warp<T, +1, NZ>(A + sl * LDZ, lane, twz);
    __syncthreads();
    T* out = sb + size_t(band) * NZ * sm.nst;
    for (int i = tid; i < ns * NZ; i += kZWarps * 32) {
        const int z = i / ns;
        const int sl = i - z * ns;
        out[size_t(z) * sm.nst + s0 + sl] = A[sl * LDZ + z];
    }
}

template <typename T, typename R, int NZ>
__global__ void __launch_bounds__(kZWarps * 32) k_zfwd_w(StickMapView sm, const T* __restrict__ twz,
                                                        const T* __restrict__ sb, const T* __restrict__ psi,
                                                        T* __restrict__ hpsi, int ld, int npw,
                                                        const R* __restrict__ gk2, R tpiba2, R invn, int accumulate) {
    constexpr int LDZ = NZ | 1;
    __shared__ T A[kStickTile * LDZ];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int s0 = blockIdx.x * kStickTile;
    const int ns = min(kStickTile, sm.nst - s0);
    const int band = blockIdx.y;
    const T* in = sb + size_t(band) * NZ * sm.nst;
    for (int i = tid; i < ns * NZ; i += kZWarps * 32) {
        const int z = i / ns;
        const int sl = i - z * ns;
        A[sl * LDZ + z] = in[size_t(z) * sm.nst + s0 + sl];
    }
    __syncthreads();
    for (int sl = warp; sl < ns; sl += kZWarps) fft_warp<T, -1, NZ>(A + sl * LDZ, lane, twz);
    __syncthreads();
    const T* p = psi + size_t(band) * ld;
    T* h = hpsi + size_t(band) * ld;
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    for (int j = j0 + tid; j < j1; j += kZWarps * 32) {
        const int pk = sm.gpk[j];
        const int g = sm.glist[j];
        T v = cscale(A[((pk >> 10) - s0) * LDZ + (pk & 1023)], invn);
        v = cadd(v, cscale(p[g], gk2[g] * tpiba2));
        if (accumulate) v = cadd(v, h[g]);
        h[g] = v;
    }
    if (!accumulate && blockIdx.x == 0)
        for (int g = npw + tid; g < ld; g += kZWarps * 32) h[g] = zero_c<T>();
}

template <typename T, typename R, int NX, int NY>
__global__ void __launch_bounds__(kPlaneWarps * 32) k_plane_w(PlaneMapView pm, int nz, const T* __restrict__ twx,
                                                             const T* __restrict__ twy, const R* __restrict__ veff_zyx,
                                                             T* __restrict__ sb) {
    constexpr int LDY = NY | 1;
    constexpr int NT = kPlaneWarps * 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* rows = reinterpret_cast<T*>(smem_raw);  // kPlaneWarps private rows of NX
    T* A = rows + kPlaneWarps * NX;            // nxc columns of LDY
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int band = blockIdx.x;
    const int z = blockIdx.y;
    const int nxc = pm.nxc;
    for (int i = tid; i < nxc * LDY; i += NT) A[i] = zero_c<T>();
    __syncthreads();
    T* plane = sb + (size_t(band) * nz + z) * pm.nst;
    for (int s = tid; s < pm.nst; s += NT) A[pm.xc[s] * LDY + pm.sy[s]] = plane[s];
    __syncthreads();
    for (int c = warp; c < nxc; c += kPlaneWarps) fft_warp<T, +1, NY>(A + c * LDY, lane, twy);
    __syncthreads();
    T* row = rows + warp * NX;
    const R* vz = veff_zyx + size_t(z) * NY * NX;
    for (int y = warp; y < NY; y += kPlaneWarps) {
        for (int x = lane; x < NX; x += 32) row[x] = zero_c<T>();
        __syncwarp();
        for (int c = lane; c < nxc; c += 32) row[pm.xpos[c]] = A[c * LDY + y];
        __syncwarp();
        fft_warp<T, +1, NX>(row, lane, twx);
        const R* vr = vz + y * NX;
        for (int x = lane; x < NX; x += 32) row[x] = cscale(row[x], vr[x]);
        __syncwarp();
        fft_warp<T, -1, NX>(row, lane, twx);
        for (int c = lane; c < nxc; c += 32) A[c * LDY + y] = row[pm.xpos[c]];
        __syncwarp();
    }
    __syncthreads();
    for (int c = warp; c < nxc; c += kPlaneWarps) fft_warp<T, -1, NY>(A + c * LDY, lane, twy);
    __syncthreads();
    for (int s = tid; s < pm.nst; s += NT) plane[s] = A[pm.xc[s] * LDY + pm.sy[s]];
}

// ---- register / shuffle transforms for square planes of N = 32*M (M = 2, 3, 4) ----
// One warp holds one length-N vector, M values per lane.  The inverse transform (exp(+i)) is decimation in
// frequency: x[32*n1 + lane] -> a radix-M DFT in registers, twiddles W_N^{-lane*k1}, then a 32-point
// transform across the lanes (five radix-2 stages, partner values by warp shuffles); lane L then holds
// the outputs k1 + M*bitrev5(L).  The forward transform (exp(-i)) is the transposed algorithm
// (decimation in time): it takes the values in that permuted order and returns x[32*n1 + lane] in natural
// order.  The r-space product with V_eff happens in between, on the permuted order, with V_eff stored
// permuted once (launch_permute_veff); no transform touches shared memory, which the plane pass then uses
// only to hold the plane and to move a row or column into registers.
template <typename T> __device__ __forceinline__ T shfl_x(T v, int m) {
    return cmake<T>(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// Per-lane twiddles.  lk[k1] = W_N^{lane*k1}.  For the five lane stages (h = 16 >> j) the butterflies are
// written without branches or selects, with this lane's role folded into its twiddles:
//   inverse (DIF):  u' = (p + sg*u) * wi[j]     p = partner's u; sg = -1 on the bottom lane of a pair, +1 on
//                                               the top; wi = conj(W_{2h}^{lane mod h}) on the bottom, 1 on the top;
//   forward (DIT):  s = wf[j] * u, u' = p + sg*s   p = partner's s; wf = W_{2h}^{lane mod h} on the bottom, 1
//                                               on the top (top: u + w u_bottom, bottom: u_top - w u).
template <typename T> struct LaneTw {
    using R = typename RealOf<T>::type;
    R sg[5];
    T wi[5], wf[5];
};

template <typename T, int N>
__device__ __forceinline__ void lane_twiddles(const T* __restrict__ roots, int lane, T* lk, LaneTw<T>& tw) {
    using R = typename RealOf<T>::type;
    constexpr int M = N / 32;
#pragma unroll
    for (int k1 = 0; k1 < M; ++k1) lk[k1] = roots[(lane * k1) % N];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        const int h = 16 >> j;
        const bool bottom = lane & h;
        const T w = roots[M * (lane % h) * (16 / h)];
        tw.sg[j] = bottom ? R(-1) : R(1);
        tw.wi[j] = bottom ? cmake<T>(w.x, -w.y) : cmake<T>(R(1), R(0));
        tw.wf[j] = bottom ? w : cmake<T>(R(1), R(0));
    }
}

template <typename T, int M>
__device__ __forceinline__ void regfft_inv_dif(T* u, const T* lk, const LaneTw<T>& tw, int lane) {
    dftR<T, +1, M>(u);
#pragma unroll
    for (int k1 = 1; k1 < M; ++k1) u[k1] = cmulc(u[k1], lk[k1]);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        const int h = 16 >> j;
#pragma unroll
        for (int k1 = 0; k1 < M; ++k1) {
            const T p = shfl_x(u[k1], h);
            const T t = cmake<T>(fma(tw.sg[j], u[k1].x, p.x), fma(tw.sg[j], u[k1].y, p.y));
            u[k1] = (j == 4) ? t : cmul(t, tw.wi[j]);  // the last stage's twiddle is 1
        }
    }
}

template <typename T, int M>
__device__ __forceinline__ void regfft_fwd_dit(T* u, const T* lk, const LaneTw<T>& tw, int lane) {
#pragma unroll
    for (int j = 4; j >= 0; --j) {
        const int h = 16 >> j;
#pragma unroll
        for (int k1 = 0; k1 < M; ++k1) {
            const T sv = (j == 4) ? u[k1] : cmul(u[k1], tw.wf[j]);  // the first stage's twiddle is 1
            const T p = shfl_x(sv, h);
            u[k1] = cmake<T>(fma(tw.sg[j], sv.x, p.x), fma(tw.sg[j], sv.y, p.y));
        }
    }
#pragma unroll
    for (int k1 = 1; k1 < M; ++k1) u[k1] = cmul(u[k1], lk[k1]);
    dftR<T, -1, M>(u);
}

// ---- register transforms with P lanes per line (N = P*Q; P = 8, 16 or 32) ----
// The generalisation of the above: lane L of a group of P lanes holds x[P*n1 + L] (n1 < Q); the inverse
// takes a Q-point DFT in registers, twiddles W_N^{-L*k1} and log2(P) radix-2 lane stages (xor h = P/2 .. 1,
// inside the group) and leaves lane L with the outputs k1 + Q*bitrev(L); the forward is the transposed
// algorithm.  Fewer lanes per line mean fewer lane stages: every lane stage moves each value through warp
// shuffles (two 32-bit shuffles per double), so P = 8 moves each value 3 times instead of 5, and a warp
// carries 32/P independent lines.  Lane twiddles come from the roots table (L1-resident) when used.

// Q-point DFT in registers, natural order in and out (DIR +1: exp(+i), -1: exp(-i)); Q = A*B with A, B in
// {2, 3, 4}: A-point DFTs of the stride-B subsets, twiddles W_Q^(n2 k1), B-point DFTs; roots[j] = W_N^j
template <typename T, int DIR, int Q>
__device__ __forceinline__ void dft_reg(T* u, const T* __restrict__ roots, int N) {
    if constexpr (Q <= 4) {
        dftR<T, DIR, Q>(u);
    } else {
        constexpr int A = (Q % 4 == 0) ? 4 : 3;
        constexpr int B = Q / A;
        static_assert(A * B == Q && B >= 2 && B <= 4, "Q = A*B with A, B in {2, 3, 4}");
        T y[B][A];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) {
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) y[n2][n1] = u[B * n1 + n2];
            dftR<T, DIR, A>(y[n2]);
#pragma unroll
            for (int k1 = 1; k1 < A; ++k1)
                if (n2 > 0) {
                    const T w = __ldg(roots + n2 * k1 * (N / Q));
                    y[n2][k1] = DIR < 0 ? cmul(y[n2][k1], w) : cmulc(y[n2][k1], w);
                }
        }
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            T z[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) z[n2] = y[n2][k1];
            dftR<T, DIR, B>(z);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) u[k1 + A * k2] = z[k2];
        }
    }
}

template <int P> constexpr int log2i() { return P == 8 ? 3 : P == 16 ? 4 : 5; }

// per-lane twiddle of each lane stage: w[j] = W_{2h}^{L mod h} (h = P >> (j + 1)); the butterflies derive
// their signs and the top lane's unit twiddle from L & h
template <typename T, int P> struct LaneTwP {
    T w[log2i<P>()];
};
template <typename T, int N, int P>
__device__ __forceinline__ void lane_twiddles_p(const T* __restrict__ roots, int L, LaneTwP<T, P>& tw) {
#pragma unroll
    for (int j = 0; j < log2i<P>(); ++j) {
        const int h = P >> (j + 1);
        tw.w[j] = roots[(N / (2 * h)) * (L % h)];
    }
}

template <typename T, int P, int Q>
__device__ __forceinline__ void regfftP_inv_dif(T* u, const T* __restrict__ roots, const LaneTwP<T, P>& tw, int L) {
    using R = typename RealOf<T>::type;
    constexpr int N = P * Q;
    dft_reg<T, +1, Q>(u, roots, N);
#pragma unroll
    for (int k1 = 1; k1 < Q; ++k1) u[k1] = cmulc(u[k1], __ldg(roots + (L * k1) % N));
#pragma unroll
    for (int j = 0; j < log2i<P>(); ++j) {
        const int h = P >> (j + 1);
        const bool bottom = L & h;
        const R sg = bottom ? R(-1) : R(1);
        const T wi = bottom ? cmake<T>(tw.w[j].x, -tw.w[j].y) : cmake<T>(R(1), R(0));
#pragma unroll
        for (int k1 = 0; k1 < Q; ++k1) {
            const T p = shfl_x(u[k1], h);
            const T t = cmake<T>(fma(sg, u[k1].x, p.x), fma(sg, u[k1].y, p.y));
            u[k1] = (j == log2i<P>() - 1) ? t : cmul(t, wi);  // the last stage's twiddle is 1
        }
    }
}

template <typename T, int P, int Q>
__device__ __forceinline__ void regfftP_fwd_dit(T* u, const T* __restrict__ roots, const LaneTwP<T, P>& tw, int L) {
    using R = typename RealOf<T>::type;
    constexpr int N = P * Q;
#pragma unroll
    for (int j = log2i<P>() - 1; j >= 0; --j) {
        const int h = P >> (j + 1);
        const bool bottom = L & h;
        const R sg = bottom ? R(-1) : R(1);
        const T wf = bottom ? tw.w[j] : cmake<T>(R(1), R(0));
#pragma unroll
        for (int k1 = 0; k1 < Q; ++k1) {
            const T sv = (j == log2i<P>() - 1) ? u[k1] : cmul(u[k1], wf);  // the first stage's twiddle is 1
            const T p = shfl_x(sv, h);
            u[k1] = cmake<T>(fma(sg, sv.x, p.x), fma(sg, sv.y, p.y));
        }
    }
#pragma unroll
    for (int k1 = 1; k1 < Q; ++k1) u[k1] = cmul(u[k1], __ldg(roots + (L * k1) % N));
    dft_reg<T, -1, Q>(u, roots, N);
}

// lanes per line of the plane pass: 32 (measured on the 96^3 plane pass of B200: P = 16 was 3 % / 5 %
// slower in FP64 / FP32 and P = 8 spills at two (FP64) or four (FP32) CTAs per SM; the values a lane holds
// and the larger in-register DFTs cost more than the lane stages they save)
template <typename T, int N> constexpr int plane_lanes() { return 32; }

// Plane pass on P-lane transforms; V_eff permuted along x and y by the P-lane slot map (launch_permute_veff).
// Shared memory: the plane (nxc occupied x-columns of N | 1) and the x -> column map.  W warps per CTA, at
// least MINB CTAs per SM; each warp transforms 32/P lines at a time.
template <typename T, typename R, int N, int P, int W, int MINB>
__global__ void __launch_bounds__(W * 32, MINB) k_plane_p(PlaneMapView pm, int nz, const T* __restrict__ roots,
                                                         const R* __restrict__ vperm, T* __restrict__ sb) {
    constexpr int Q = N / P;
    constexpr int G = 32 / P;
    constexpr int LD = N | 1;
    constexpr int NT = W * 32;
    static_assert(N % (W * G) == 0, "rows per round");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);
    const int nxc = pm.nxc;
    int* cmap = reinterpret_cast<int*>(A + nxc * LD);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int L = lane % P, grp = lane / P;
    const int band = blockIdx.x;
    const int z = blockIdx.y;
    for (int i = tid; i < nxc * LD; i += NT) A[i] = zero_c<T>();
    for (int i = tid; i < N; i += NT) cmap[i] = -1;
    __syncthreads();
    for (int c = tid; c < nxc; c += NT) cmap[pm.xpos[c]] = c;
    T* plane = sb + (size_t(band) * nz + z) * pm.nst;
    for (int s = tid; s < pm.nst; s += NT) A[pm.xc[s] * LD + pm.sy[s]] = plane[s];
    LaneTwP<T, P> tw;
    lane_twiddles_p<T, N, P>(roots, L, tw);
    __syncthreads();
    int cm[Q];
#pragma unroll
    for (int n1 = 0; n1 < Q; ++n1) cm[n1] = cmap[P * n1 + L];
    // inverse y transform of every occupied column (a group past the last column transforms a valid one
    // and stores nothing: the shuffles need the whole warp)
    for (int c0 = warp * G; c0 < nxc; c0 += W * G) {
        const int c = c0 + grp;
        const T* colr = A + (c < nxc ? c : c0) * LD;
        T u[Q];
#pragma unroll
        for (int n1 = 0; n1 < Q; ++n1) u[n1] = colr[P * n1 + L];
        regfftP_inv_dif<T, P, Q>(u, roots, tw, L);
        if (c < nxc) {
            T* col = A + c * LD;
#pragma unroll
            for (int k1 = 0; k1 < Q; ++k1) col[P * k1 + L] = u[k1];
        }
    }
    __syncthreads();
    // each row slot: inverse x transform, times V_eff(r), forward x transform
    const R* vz = vperm + size_t(z) * N * N;
    for (int sy0 = warp * G; sy0 < N; sy0 += W * G) {
        const int sy = sy0 + grp;
        T u[Q];
#pragma unroll
        for (int n1 = 0; n1 < Q; ++n1) u[n1] = cm[n1] >= 0 ? A[cm[n1] * LD + sy] : zero_c<T>();
        regfftP_inv_dif<T, P, Q>(u, roots, tw, L);
        const R* vr = vz + sy * N;
#pragma unroll
        for (int k1 = 0; k1 < Q; ++k1) u[k1] = cscale(u[k1], vr[P * k1 + L]);
        regfftP_fwd_dit<T, P, Q>(u, roots, tw, L);
#pragma unroll
        for (int n1 = 0; n1 < Q; ++n1)
            if (cm[n1] >= 0) A[cm[n1] * LD + sy] = u[n1];
    }
    __syncthreads();
    // forward y transform back to natural order
    for (int c0 = warp * G; c0 < nxc; c0 += W * G) {
        const int c = c0 + grp;
        const T* colr = A + (c < nxc ? c : c0) * LD;
        T u[Q];
#pragma unroll
        for (int k1 = 0; k1 < Q; ++k1) u[k1] = colr[P * k1 + L];
        regfftP_fwd_dit<T, P, Q>(u, roots, tw, L);
        if (c < nxc) {
            T* col = A + c * LD;
#pragma unroll
            for (int n1 = 0; n1 < Q; ++n1) col[P * n1 + L] = u[n1];
        }
    }
    __syncthreads();
    for (int s = tid; s < pm.nst; s += NT) plane[s] = A[pm.xc[s] * LD + pm.sy[s]];
}

// psi -> rho on the register transforms (elecstate_pw.cpp:160-216: rho(r) += w_b |psi_b(r)|^2 with the
// backward transform of each occupied band).  CTA (z slot, g): bands g, g + nsplit, ... of the chunk in the
// stick buffer; per band the plane's inverse y transform on the occupied columns and the inverse x
// transform of every row, and this warp's rows of w_b |psi|^2 summed in registers over the bands.  The
// partial plane (slot order) goes to ws[g], overwritten on the first chunk and added to afterwards: each
// (z slot, g) owns its plane, so the sums are deterministic.
template <typename T, typename R, int N>
__global__ void __launch_bounds__(kPlaneWarps * 32) k_rho_plane_r(PlaneMapView pm, int nz, const T* __restrict__ roots,
                                                                 const T* __restrict__ sb, int nbc,
                                                                 const double* __restrict__ w, int nsplit,
                                                                 R* __restrict__ ws, int first) {
    constexpr int M = N / 32;
    constexpr int LD = N | 1;
    constexpr int NT = kPlaneWarps * 32;
    constexpr int RW = N / kPlaneWarps;  // rows per warp
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);
    const int nxc = pm.nxc;
    int* cmap = reinterpret_cast<int*>(A + nxc * LD);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sz = blockIdx.x, g = blockIdx.y;
    for (int i = tid; i < N; i += NT) cmap[i] = -1;
    __syncthreads();
    for (int c = tid; c < nxc; c += NT) cmap[pm.xpos[c]] = c;
    T lk[M];
    LaneTw<T> tw;
    lane_twiddles<T, N>(roots, lane, lk, tw);
    __syncthreads();
    int cm[M];
#pragma unroll
    for (int n1 = 0; n1 < M; ++n1) cm[n1] = cmap[32 * n1 + lane];
    R acc[RW][M];
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int k1 = 0; k1 < M; ++k1) acc[r][k1] = R(0);
    for (int b = g; b < nbc; b += nsplit) {
        const R wb = R(w[b]);
        __syncthreads();  // the previous band's rows are read
        for (int i = tid; i < nxc * LD; i += NT) A[i] = zero_c<T>();
        __syncthreads();
        const T* plane = sb + (size_t(b) * nz + sz) * pm.nst;
        for (int s = tid; s < pm.nst; s += NT) A[pm.xc[s] * LD + pm.sy[s]] = plane[s];
        __syncthreads();
        for (int c = warp; c < nxc; c += kPlaneWarps) {
            T u[M];
            T* col = A + c * LD;
#pragma unroll
            for (int n1 = 0; n1 < M; ++n1) u[n1] = col[32 * n1 + lane];
            regfft_inv_dif<T, M>(u, lk, tw, lane);
#pragma unroll
            for (int k1 = 0; k1 < M; ++k1) col[32 * k1 + lane] = u[k1];
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RW; ++r) {
            const int sy = warp + r * kPlaneWarps;
            T u[M];
#pragma unroll
            for (int n1 = 0; n1 < M; ++n1) u[n1] = cm[n1] >= 0 ? A[cm[n1] * LD + sy] : zero_c<T>();
            regfft_inv_dif<T, M>(u, lk, tw, lane);
#pragma unroll
            for (int k1 = 0; k1 < M; ++k1) acc[r][k1] = fma(wb, fma(u[k1].x, u[k1].x, u[k1].y * u[k1].y), acc[r][k1]);
        }
    }
    if (!first && g >= nbc) return;  // nothing added to this partial plane
    R* out = ws + (size_t(g) * nz + sz) * N * N;
#pragma unroll
    for (int r = 0; r < RW; ++r) {
        const int sy = warp + r * kPlaneWarps;
#pragma unroll
        for (int k1 = 0; k1 < M; ++k1) {
            R* o = out + sy * N + 32 * k1 + lane;
            *o = first ? acc[r][k1] : *o + acc[r][k1];
        }
    }
}

// ---- stick buffer of the register-transform grids (nz = 32*M): the planes are stored by slot (plane slot sz
// holds z = sz/32 + M*bitrev5(sz mod 32)), V_eff is permuted along z as well, and the forward z pass takes
// the slots back to natural z (the z passes: plane_t.cuh, k_zinv_t / k_zfwd_t).
// Src gives the k-point entry of a block: one k-point (OneK) or a batch indexed by blockIdx.z (ManyK).
struct OneK {
    KBatchEntry e;
    __device__ __forceinline__ const KBatchEntry& get(int) const { return e; }
};
struct ManyK {
    KBatchArgs a;
    __device__ __forceinline__ const KBatchEntry& get(int q) const { return a.e[q]; }
};

__device__ __forceinline__ int perm_slot(int s, int m) { return (s >> 5) + m * int(__brev(unsigned(s & 31)) >> 27); }
// the same for lines of P = 2^lp lanes and q values per lane: slot s holds index s/P + q * bitrev_lp(s mod P)
__device__ __forceinline__ int perm_slot_p(int s, int lp, int q) {
    return (s >> lp) + q * int(__brev(unsigned(s & ((1 << lp) - 1))) >> (32 - lp));
}

template <typename R>
__global__ void k_permute_veff(int nz, int n, int lp, int mz, const R* __restrict__ in, R* __restrict__ out) {
    const long total = long(nz) * n * n;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int sx = int(i % n);
        const long r = i / n;
        const int sy = int(r % n);
        const int sz = int(r / n);
        const int q = n >> lp;
        out[i] = in[(long(perm_slot(sz, mz)) * n + perm_slot_p(sy, lp, q)) * n + perm_slot_p(sx, lp, q)];
    }
}

// rho (x, y, z natural, z fastest) += sum over g of the partial planes (slot order), in a fixed order
template <typename R>
__global__ void k_rho_reduce(int nz, int n, int m, int mz, int nsplit, const R* __restrict__ ws, R* __restrict__ rho) {
    const long total = long(nz) * n * n;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int sx = int(i % n);
        const int sy = int((i / n) % n);
        const int sz = int(i / (long(n) * n));
        R sum = ws[i];
        for (int g = 1; g < nsplit; ++g) sum += ws[size_t(g) * total + i];
        const int x = perm_slot(sx, m), y = perm_slot(sy, m), z = perm_slot(sz, mz);
        rho[(size_t(x) * n + y) * nz + z] += sum;
    }
}


// ---- k-point batched z passes: one launch covers every k-point of a batch (blockIdx.z = k slot) ----
template <typename T, int NZ>
__global__ void __launch_bounds__(kZWarps * 32) k_zinv_wb(KBatchArgs args, int b0, int nbc, const T* __restrict__ twz,
                                                         T* __restrict__ sb) {
    constexpr int LDZ = NZ | 1;
    __shared__ T A[kStickTile * LDZ];
    const KBatchEntry& e = args.e[blockIdx.z];
    const StickMapView sm = e.sm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int s0 = blockIdx.x * kStickTile;
    if (s0 >= sm.nst) return;
    const int ns = min(kStickTile, sm.nst - s0);
    const int band = blockIdx.y;
    for (int i = tid; i < kStickTile * LDZ; i += kZWarps * 32) A[i] = zero_c<T>();
    __syncthreads();
    const T* p = reinterpret_cast<const T*>(e.psi) + size_t(b0 + band) * e.ld;
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    for (int j = j0 + tid; j < j1; j += kZWarps * 32) {
        const int pk = sm.gpk[j];
        A[((pk >> 10) - s0) * LDZ + (pk & 1023)] = p[sm.glist[j]];
    }
    __syncthreads();
    for (int sl = warp; sl < ns; sl += kZWarps) fft_warp<T, +1, NZ>(A + sl * LDZ, lane, twz);
    __syncthreads();
    T* out = sb + (size_t(blockIdx.z) * nbc + band) * NZ * sm.nst;
    for (int i = tid; i < ns * NZ; i += kZWarps * 32) {
        const int z = i / ns;
        const int sl = i - z * ns;
        out[size_t(z) * sm.nst + s0 + sl] = A[sl * LDZ + z];
    }
}

template <typename T, typename R, int NZ>
__global__ void __launch_bounds__(kZWarps * 32) k_zfwd_wb(KBatchArgs args, int b0, int nbc, const T* __restrict__ twz,
                                                         const T* __restrict__ sb, R tpiba2, R invn) {
    constexpr int LDZ = NZ | 1;
    __shared__ T A[kStickTile * LDZ];
    const KBatchEntry& e = args.e[blockIdx.z];
    const StickMapView sm = e.sm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int s0 = blockIdx.x * kStickTile;
    if (s0 >= sm.nst) return;
    const int ns = min(kStickTile, sm.nst - s0);
    const int band = blockIdx.y;
    const T* in = sb + (size_t(blockIdx.z) * nbc + band) * NZ * sm.nst;
    for (int i = tid; i < ns * NZ; i += kZWarps * 32) {
        const int z = i / ns;
        const int sl = i - z * ns;
        A[sl * LDZ + z] = in[size_t(z) * sm.nst + s0 + sl];
    }
    __syncthreads();
    for (int sl = warp; sl < ns; sl += kZWarps) fft_warp<T, -1, NZ>(A + sl * LDZ, lane, twz);
    __syncthreads();
    const T* p = reinterpret_cast<const T*>(e.psi) + size_t(b0 + band) * e.ld;
    T* h = reinterpret_cast<T*>(e.hpsi) + size_t(b0 + band) * e.ld;
    const R* gk2 = reinterpret_cast<const R*>(e.gk2);
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    for (int j = j0 + tid; j < j1; j += kZWarps * 32) {
        const int pk = sm.gpk[j];
        const int g = sm.glist[j];
        T v = cscale(A[((pk >> 10) - s0) * LDZ + (pk & 1023)], invn);
        v = cadd(v, cscale(p[g], gk2[g] * tpiba2));
        h[g] = v;
    }
    if (blockIdx.x == 0)
        for (int g = e.npw + tid; g < e.ld; g += kZWarps * 32) h[g] = zero_c<T>();
}

template <typename T> const T* twp(const FftAxis& a);
template <> const double2* twp<double2>(const FftAxis& a) { return a.tw64.ptr; }
template <> const float2* twp<float2>(const FftAxis& a) { return a.tw32.ptr; }
template <typename T> const T* rtp(const FftAxis& a);
template <> const double2* rtp<double2>(const FftAxis& a) { return a.rt64.ptr; }
template <> const float2* rtp<float2>(const FftAxis& a) { return a.rt32.ptr; }

template <typename K> void smem_attr(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) B200_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
}

template <typename T, typename R, int NZ>
void zpasses(bool inv, const PWGrid& g, int ik, int nb, int ld, const T* psi, T* hpsi, T* sb, double tpiba2,
             int accumulate, cudaStream_t s) {
    const dim3 grid(ceil_div(g.nst, kStickTile), nb);
    if (inv) {
        k_zinv_w<T, NZ><<<grid, kZWarps * 32, 0, s>>>(g.stick_view(ik), twp<T>(g.az), psi, ld, sb);
        note_launch();
    } else {
        const KMap& km = g.kmaps[ik];
        const R* gk2 = std::is_same<R, double>::value ? (const R*)km.gk2.ptr : (const R*)km.gk2f.ptr;
        k_zfwd_w<T, R, NZ><<<grid, kZWarps * 32, 0, s>>>(g.stick_view(ik), twp<T>(g.az), sb, psi, hpsi, ld, km.npw,
                                                        gk2, R(tpiba2), R(1.0 / double(g.nxyz())), accumulate);
        note_launch();
    }
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R>
bool zpass_dispatch(bool inv, const PWGrid& g, int ik, int nb, int ld, const T* psi, T* hpsi, T* sb, double tpiba2,
                    int accumulate, cudaStream_t s) {
    switch (g.nz) {
        case 18: zpasses<T, R, 18>(inv, g, ik, nb, ld, psi, hpsi, sb, tpiba2, accumulate, s); return true;
        case 36: zpasses<T, R, 36>(inv, g, ik, nb, ld, psi, hpsi, sb, tpiba2, accumulate, s); return true;
        case 45: zpasses<T, R, 45>(inv, g, ik, nb, ld, psi, hpsi, sb, tpiba2, accumulate, s); return true;
        case 90: zpasses<T, R, 90>(inv, g, ik, nb, ld, psi, hpsi, sb, tpiba2, accumulate, s); return true;
        case 96: zpasses<T, R, 96>(inv, g, ik, nb, ld, psi, hpsi, sb, tpiba2, accumulate, s); return true;
        case 125: zpasses<T, R, 125>(inv, g, ik, nb, ld, psi, hpsi, sb, tpiba2, accumulate, s); return true;
        case 128: zpasses<T, R, 128>(inv, g, ik, nb, ld, psi, hpsi, sb, tpiba2, accumulate, s); return true;
        default: return false;
    }
}

template <typename T, typename R, int N>
bool plane_launch(const PWGrid& g, int nb, const R* veff, T* sb, cudaStream_t s) {
    const size_t smem = (size_t(kPlaneWarps) * N + size_t(g.nxc) * (N | 1)) * sizeof(T);
    if (smem > 227 * 1024) return false;
    smem_attr(k_plane_w<T, R, N, N>, smem);
    k_plane_w<T, R, N, N><<<dim3(nb, g.nz), kPlaneWarps * 32, smem, s>>>(g.plane_view(), g.nz, twp<T>(g.ax),
                                                                         twp<T>(g.ay), veff, sb);
    note_launch();
    B200_CUDA(cudaGetLastError());
    return true;
}

// Plane pass with the two-pass register transforms (plane_t.cuh): N = R1 * R2, NT threads, RB rows per
// x batch, at least MINB CTAs per SM.  vt: V_eff arranged for it (launch_arrange_veff).
template <typename T, typename R, int N, int R1, int R2, int NT, int RB, int MINB>
bool plane_launch_t(const PWGrid& g, int nb, const R* vt, T* sb, cudaStream_t s) {
    const size_t smem = plane_t::smem_bytes<T>(R1, R2, RB, N, g.nxc);
    if (smem > 227 * 1024) return false;
    auto kern = plane_t::k_plane_t<T, R, N, R1, R2, NT, RB, MINB>;
    smem_attr(kern, smem);
    kern<<<dim3(nb, g.nz), NT, smem, s>>>(g.plane_view(), g.nz, rtp<T>(g.ax), vt, sb);
    note_launch();
    B200_CUDA(cudaGetLastError());
    return true;
}

// the register-transform plane pass of variant `var` (1: one warp per line with warp-shuffle lane stages;
// 2-5: two-pass transforms in four launch shapes; 0: the default shape)
template <typename T, typename R, int N>
bool plane_launch_var(const PWGrid& g, int var, int nb, const R* vperm, T* sb, cudaStream_t s) {
    constexpr bool f64 = std::is_same<T, double2>::value;
    const R* vt = vperm + g.nxyz();
    if (var == 1) {
        const size_t smem = size_t(g.nxc) * (N | 1) * sizeof(T) + size_t(N) * sizeof(int);
        if (smem > 227 * 1024) return false;
        // FP64: two CTAs of 8 warps per SM (up to 128 registers a thread); FP32: four of 8 warps
        constexpr int P = plane_lanes<T, N>();
        if constexpr (f64) {
            smem_attr(k_plane_p<T, R, N, P, 8, 2>, smem);
            k_plane_p<T, R, N, P, 8, 2><<<dim3(nb, g.nz), 8 * 32, smem, s>>>(g.plane_view(), g.nz, rtp<T>(g.ax), vperm, sb);
        } else {
            smem_attr(k_plane_p<T, R, N, P, 8, 4>, smem);
            k_plane_p<T, R, N, P, 8, 4><<<dim3(nb, g.nz), 8 * 32, smem, s>>>(g.plane_view(), g.nz, rtp<T>(g.ax), vperm, sb);
        }
        note_launch();
        B200_CUDA(cudaGetLastError());
        return true;
    }
    constexpr int R2 = 8, R1 = N / 8;
    // thread counts that are multiples of R1 and R2 (each thread keeps its twiddles in registers): 24 | NT for
    // N = 96, 16 | NT for 128, 8 | NT for 64.  An FP64 plane of 128 takes ~146 KB of shared memory (one CTA
    // per SM) and its 16-point transforms ~230 registers a thread, so its CTAs stay at 256 threads.
    constexpr bool big64 = f64 && N == 128;
    constexpr int NTL = N == 96 ? 384 : (big64 ? 256 : 512);  // large CTA, one per SM
    constexpr int NTS = N == 96 ? 192 : 256;                   // small CTA, two (FP32: more) per SM
    constexpr int M2 = f64 ? 1 : 2;  // FP32 planes take half the shared memory: twice the CTAs per SM
    constexpr int MS = big64 ? 1 : 2 * M2;
    switch (var) {
        case 3: return plane_launch_t<T, R, N, R1, R2, NTL, 32, 1>(g, nb, vt, sb, s);
        case 4: return plane_launch_t<T, R, N, R1, R2, NTS, 32, big64 ? 1 : M2>(g, nb, vt, sb, s);
        case 5: return plane_launch_t<T, R, N, R1, R2, NTL, 16, 1>(g, nb, vt, sb, s);
        default: return plane_launch_t<T, R, N, R1, R2, NTS, 16, MS>(g, nb, vt, sb, s);
    }
}

// the default plane variant of a precision and plane size, from CUDA-event timings of the local pass on B200
// (64-atom cell at 96^2, 216-atom cell at 128^2, band chunks of 18 and 160): FP64 the two-pass transforms
// (96: 2.14 ms against 2.22 for the warp-shuffle pass per 160 bands; 128: 3.21 against 3.57 per 96 bands);
// FP32 the warp-shuffle pass (1.12 against 1.19 ms; 1.57 against 1.64 ms)
template <typename T> constexpr int default_plane_variant(int n) {
    return std::is_same<T, double2>::value ? (n == 128 ? 4 : 2) : 1;
}

template <typename T, typename R, int N>
bool plane_launch_r(const PWGrid& g, int nb, const R* vperm, T* sb, cudaStream_t s) {
    int var = std::is_same<T, double2>::value ? g.plane_variant64 : g.plane_variant32;
    if (var == 0) var = default_plane_variant<T>(N);
    if (plane_launch_var<T, R, N>(g, var, nb, vperm, sb, s)) return true;
    return var != 1 && plane_launch_var<T, R, N>(g, 1, nb, vperm, sb, s);  // shapes whose plane does not fit
}

template <typename T, typename R>
bool plane_dispatch(const PWGrid& g, int nb, const R* veff, const R* vperm, T* sb, cudaStream_t s) {
    if (g.nx != g.ny) return false;
    (void)vperm;
    switch (g.nx) {
        case 18: return plane_launch<T, R, 18>(g, nb, veff, sb, s);
        case 36: return plane_launch<T, R, 36>(g, nb, veff, sb, s);
        case 45: return plane_launch<T, R, 45>(g, nb, veff, sb, s);
        case 96: return plane_launch<T, R, 96>(g, nb, veff, sb, s);
        case 125: return plane_launch<T, R, 125>(g, nb, veff, sb, s);
        case 128: return plane_launch<T, R, 128>(g, nb, veff, sb, s);
        default: return false;
    }
}

bool supported_z(int n) { return n == 18 || n == 36 || n == 45 || n == 90 || n == 96 || n == 125 || n == 128; }
bool supported_xy(int nx, int ny) {
    return nx == ny && (nx == 18 || nx == 36 || nx == 45 || nx == 96 || nx == 125 || nx == 128);
}

template <typename T, typename R, int NZ>
void zbatch(bool inv, const PWGrid& g, const KBatchArgs& args, int nk, int b0, int nbc, T* sb, double tpiba2, cudaStream_t s) {
    const dim3 grid(ceil_div(g.nst, kStickTile), nbc, nk);
    if (inv) {
        k_zinv_wb<T, NZ><<<grid, kZWarps * 32, 0, s>>>(args, b0, nbc, twp<T>(g.az), sb);
    } else {
        k_zfwd_wb<T, R, NZ><<<grid, kZWarps * 32, 0, s>>>(args, b0, nbc, twp<T>(g.az), sb, R(tpiba2),
                                                         R(1.0 / double(g.nxyz())));
    }
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R>
bool zbatch_dispatch(bool inv, const PWGrid& g, const KBatchArgs& args, int nk, int b0, int nbc, T* sb, double tpiba2,
                     cudaStream_t s) {
    switch (g.nz) {
        case 18: zbatch<T, R, 18>(inv, g, args, nk, b0, nbc, sb, tpiba2, s); return true;
        case 36: zbatch<T, R, 36>(inv, g, args, nk, b0, nbc, sb, tpiba2, s); return true;
        case 45: zbatch<T, R, 45>(inv, g, args, nk, b0, nbc, sb, tpiba2, s); return true;
        case 90: zbatch<T, R, 90>(inv, g, args, nk, b0, nbc, sb, tpiba2, s); return true;
        case 96: zbatch<T, R, 96>(inv, g, args, nk, b0, nbc, sb, tpiba2, s); return true;
        case 125: zbatch<T, R, 125>(inv, g, args, nk, b0, nbc, sb, tpiba2, s); return true;
        case 128: zbatch<T, R, 128>(inv, g, args, nk, b0, nbc, sb, tpiba2, s); return true;
        default: return false;
    }
}

}  // namespace

template <typename T, typename R, int NZ, typename Src>
void zpass_r(bool inv, const PWGrid& g, const Src& src, int nk, int b0, int nbc, T* sb, double tpiba2, int accumulate,
             cudaStream_t s) {
    // two-pass register transforms (both plane-pass families read and write this stick layout): 32 sticks per
    // CTA, 8 warps.  Twiddles come from the L1-resident roots table; at 41-84 registers three or more CTAs
    // share an SM, which hides the latency of the sphere gathers and scatters better than one 12-warp CTA
    // keeping its twiddles in registers (116 registers at nz = 96) or the one-warp-per-stick shuffle passes
    constexpr int R2 = 8, R1 = NZ / 8, TS = 32, NT = 256;
    const dim3 grid(ceil_div(g.nst, TS), nbc, nk);
    constexpr size_t smem = plane_t::zpass_smem_bytes<T>(R1, R2, TS);
    if (inv) {
        auto kern = plane_t::k_zinv_t<T, NZ, R1, R2, TS, NT, Src>;
        smem_attr(kern, smem);
        kern<<<grid, NT, smem, s>>>(src, b0, nbc, rtp<T>(g.az), sb);
    } else {
        auto kern = plane_t::k_zfwd_t<T, R, NZ, R1, R2, TS, NT, Src>;
        smem_attr(kern, smem);
        kern<<<grid, NT, smem, s>>>(src, b0, nbc, rtp<T>(g.az), sb, R(tpiba2), R(1.0 / double(g.nxyz())), accumulate);
    }
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R, typename Src>
bool zpass_r_dispatch(bool inv, const PWGrid& g, const Src& src, int nk, int b0, int nbc, T* sb, double tpiba2,
                      int accumulate, cudaStream_t s) {
    switch (g.nz) {
        case 64: zpass_r<T, R, 64>(inv, g, src, nk, b0, nbc, sb, tpiba2, accumulate, s); return true;
        case 96: zpass_r<T, R, 96>(inv, g, src, nk, b0, nbc, sb, tpiba2, accumulate, s); return true;
        case 128: zpass_r<T, R, 128>(inv, g, src, nk, b0, nbc, sb, tpiba2, accumulate, s); return true;
        default: return false;
    }
}

template <typename T, typename R>
bool plane_r_dispatch(const PWGrid& g, int nb, const R* vperm, T* sb, cudaStream_t s) {
    switch (g.nx) {
        case 64: return plane_launch_r<T, R, 64>(g, nb, vperm, sb, s);
        case 96: return plane_launch_r<T, R, 96>(g, nb, vperm, sb, s);
        case 128: return plane_launch_r<T, R, 128>(g, nb, vperm, sb, s);
        default: return false;
    }
}

// all three passes with register transforms (grids with plane_perm_supported); false if the plane does not fit
template <typename T, typename R, typename Src>
bool local_r(const PWGrid& g, const Src& src, int nk, int b0, int nbc, const R* vperm, T* sb, double tpiba2,
             int accumulate, cudaStream_t s) {
    const size_t smem = size_t(g.nxc) * (g.nx | 1) * sizeof(T) + size_t(g.nx) * sizeof(int);
    if (smem > 227 * 1024) return false;  // neither plane pass fits (the two-pass one needs more)
    zpass_r_dispatch<T, R>(true, g, src, nk, b0, nbc, sb, tpiba2, accumulate, s);
    plane_r_dispatch<T, R>(g, nk * nbc, vperm, sb, s);
    zpass_r_dispatch<T, R>(false, g, src, nk, b0, nbc, sb, tpiba2, accumulate, s);
    return true;
}

template <typename T, typename R>
bool launch_hpsi_local_kbatch(const PWGrid& g, const KBatchArgs& args, int nk, int nb, const R* veff_zyx,
                              const R* veff_perm, T* stickbuf, int chunk, double tpiba2, cudaStream_t s) {
    if (veff_perm && plane_perm_supported(g)) {
        ManyK src;
        src.a = args;
        bool ok = true;
        for (int b0 = 0; b0 < nb && ok; b0 += chunk) {
            const int nbc = nb - b0 < chunk ? nb - b0 : chunk;
            ok = local_r<T, R>(g, src, nk, b0, nbc, veff_perm, stickbuf, tpiba2, 0, s);
        }
        if (ok) return true;
    }
    if (!supported_z(g.nz) || !supported_xy(g.nx, g.ny)) return false;
    const size_t smem = (size_t(kPlaneWarps) * g.nx + size_t(g.nxc) * (g.ny | 1)) * sizeof(T);
    if (smem > 227 * 1024) return false;
    for (int b0 = 0; b0 < nb; b0 += chunk) {
        const int nbc = nb - b0 < chunk ? nb - b0 : chunk;
        zbatch_dispatch<T, R>(true, g, args, nk, b0, nbc, stickbuf, tpiba2, s);
        plane_dispatch<T, R>(g, nk * nbc, veff_zyx, veff_perm, stickbuf, s);
        zbatch_dispatch<T, R>(false, g, args, nk, b0, nbc, stickbuf, tpiba2, s);
    }
    return true;
}

namespace {
}  // namespace

template bool launch_hpsi_local_kbatch<double2, double>(const PWGrid&, const KBatchArgs&, int, int, const double*,
                                                        const double*, double2*, int, double, cudaStream_t);
template bool launch_hpsi_local_kbatch<float2, float>(const PWGrid&, const KBatchArgs&, int, int, const float*,
                                                      const float*, float2*, int, double, cudaStream_t);

template <typename T, typename R>
bool launch_hpsi_local_fast(const PWGrid& g, int ik, const R* veff_zyx, const R* veff_perm, int nb, int ld,
                            const T* psi, T* hpsi, T* stickbuf, double tpiba2, int accumulate, cudaStream_t s) {
    if (veff_perm && plane_perm_supported(g)) {
        const KMap& km = g.kmaps[ik];
        OneK src;
        src.e.sm = g.stick_view(ik);
        src.e.psi = psi;
        src.e.hpsi = hpsi;
        src.e.ld = ld;
        src.e.npw = km.npw;
        src.e.gk2 = std::is_same<T, double2>::value ? (const void*)km.gk2.ptr : (const void*)km.gk2f.ptr;
        if (local_r<T, R>(g, src, 1, 0, nb, veff_perm, stickbuf, tpiba2, accumulate, s)) return true;
    }
    if (!supported_z(g.nz) || !supported_xy(g.nx, g.ny)) return false;
    const size_t smem = (size_t(kPlaneWarps) * g.nx + size_t(g.nxc) * (g.ny | 1)) * sizeof(T);
    if (smem > 227 * 1024) return false;
    zpass_dispatch<T, R>(true, g, ik, nb, ld, psi, hpsi, stickbuf, tpiba2, accumulate, s);
    plane_dispatch<T, R>(g, nb, veff_zyx, veff_perm, stickbuf, s);
    zpass_dispatch<T, R>(false, g, ik, nb, ld, psi, hpsi, stickbuf, tpiba2, accumulate, s);
    return true;
}

template bool launch_hpsi_local_fast<double2, double>(const PWGrid&, int, const double*, const double*, int, int,
                                                      const double2*, double2*, double2*, double, int, cudaStream_t);
template bool launch_hpsi_local_fast<float2, float>(const PWGrid&, int, const float*, const float*, int, int,
                                                    const float2*, float2*, float2*, double, int, cudaStream_t);

bool plane_perm_supported(const PWGrid& g) {
    auto ok = [](int n) { return n == 64 || n == 96 || n == 128; };
    return g.nx == g.ny && ok(g.nx) && ok(g.nz) && g.nz < 1024;
}

template <typename R>
bool launch_permute_veff(const PWGrid& g, const R* veff_zyx, R* out, cudaStream_t s) {
    if (!plane_perm_supported(g)) return false;
    // x and y in the slot order of the plane pass's P-lane transforms, z in that of the 32-lane z passes
    using T = typename std::conditional<std::is_same<R, double>::value, double2, float2>::type;
    int P = 8;
    switch (g.nx) {
        case 64: P = plane_lanes<T, 64>(); break;
        case 96: P = plane_lanes<T, 96>(); break;
        default: P = plane_lanes<T, 128>(); break;
    }
    const int lp = P == 8 ? 3 : P == 16 ? 4 : 5;
    k_permute_veff<R><<<1184, 256, 0, s>>>(g.nz, g.nx, lp, g.nz / 32, veff_zyx, out);
    note_launch();
    B200_CUDA(cudaGetLastError());
    return true;
}
template bool launch_permute_veff<double>(const PWGrid&, const double*, double*, cudaStream_t);
template bool launch_permute_veff<float>(const PWGrid&, const float*, float*, cudaStream_t);

template <typename R>
bool launch_arrange_veff(const PWGrid& g, const R* veff_zyx, R* out, cudaStream_t s) {
    if (!plane_perm_supported(g)) return false;
    plane_t::k_arrange_veff<R><<<1184, 256, 0, s>>>(g.nz, g.nx, g.nx / 8, 8, veff_zyx, out);
    note_launch();
    B200_CUDA(cudaGetLastError());
    return true;
}
template bool launch_arrange_veff<double>(const PWGrid&, const double*, double*, cudaStream_t);
template bool launch_arrange_veff<float>(const PWGrid&, const float*, float*, cudaStream_t);

bool rho_r_supported(const PWGrid& g) {
    const size_t smem = size_t(g.nxc) * (g.nx | 1) * sizeof(double2) + size_t(g.nx) * sizeof(int);
    return plane_perm_supported(g) && smem <= 227 * 1024;
}

template <typename T, typename R, int N>
void rho_plane_launch(const PWGrid& g, const T* sb, int nbc, const double* w, int nsplit, R* ws, int first,
                      cudaStream_t s) {
    const size_t smem = size_t(g.nxc) * (N | 1) * sizeof(T) + size_t(N) * sizeof(int);
    smem_attr(k_rho_plane_r<T, R, N>, smem);
    k_rho_plane_r<T, R, N><<<dim3(g.nz, nsplit), kPlaneWarps * 32, smem, s>>>(g.plane_view(), g.nz, rtp<T>(g.ax), sb,
                                                                               nbc, w, nsplit, ws, first);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R>
void launch_rho_chunk_r(const PWGrid& g, int ik, int b0, int nbc, int ld, const T* psi, const double* w_chunk,
                        T* sb, int nsplit, R* ws, int first, cudaStream_t s) {
    OneK src;
    src.e.sm = g.stick_view(ik);
    src.e.psi = psi;
    src.e.hpsi = nullptr;
    src.e.ld = ld;
    src.e.npw = g.kmaps[ik].npw;
    src.e.gk2 = nullptr;
    const bool zok = zpass_r_dispatch<T, R>(true, g, src, 1, b0, nbc, sb, 0.0, 0, s);
    B200_CHECK(zok, kInvalidArgument, "psi -> rho: nz has no register transform");
    switch (g.nx) {
        case 64: rho_plane_launch<T, R, 64>(g, sb, nbc, w_chunk, nsplit, ws, first, s); break;
        case 96: rho_plane_launch<T, R, 96>(g, sb, nbc, w_chunk, nsplit, ws, first, s); break;
        case 128: rho_plane_launch<T, R, 128>(g, sb, nbc, w_chunk, nsplit, ws, first, s); break;
        default: B200_CHECK(false, kInvalidArgument, "psi -> rho: nx has no register transform");
    }
}

template <typename R>
void launch_rho_reduce_r(const PWGrid& g, int nsplit, const R* ws, R* rho, cudaStream_t s) {
    k_rho_reduce<R><<<1184, 256, 0, s>>>(g.nz, g.nx, g.nx / 32, g.nz / 32, nsplit, ws, rho);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template void launch_rho_chunk_r<double2, double>(const PWGrid&, int, int, int, int, const double2*, const double*,
                                                  double2*, int, double*, int, cudaStream_t);
template void launch_rho_chunk_r<float2, float>(const PWGrid&, int, int, int, int, const float2*, const double*,
                                                float2*, int, float*, int, cudaStream_t);
template void launch_rho_reduce_r<double>(const PWGrid&, int, const double*, double*, cudaStream_t);
template void launch_rho_reduce_r<float>(const PWGrid&, int, const float*, float*, cudaStream_t);

}  // namespace b200
