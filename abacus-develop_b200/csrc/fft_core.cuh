// Batched mixed-radix (2/3/4/5) complex FFT on shared memory, for sm_100a.
//
// Self-sorting Stockham passes: pass j with radix R and p = R_0*...*R_{j-1}
// reads element i + r*(n/R), twiddles it by w^(r*k) with k = i mod p and
// w = exp(-+2 pi i / (p R)), does an R-point DFT and writes element
// (i - k)*R + k + q*p.  Data ping-pongs between two shared-memory buffers of
// the same geometry (element stride `es`, batch stride `bs`); the result is
// always left in the first buffer.  DIR = -1 is the forward transform
// exp(-i G r) (FFTW_FORWARD), DIR = +1 the un-normalised backward transform
// exp(+i G r) (FFTW_BACKWARD), the conventions of ABACUS's
// PW_Basis_K::real_to_recip / recip_to_real (pw_transform_k.cpp:26-213).
//
// Twiddles are computed on the host in double precision (stored for the
// forward sign; the backward pass conjugates them), so no device math library
// routine is involved.
#pragma once
#include <cuda_runtime.h>

namespace b200 {

template <typename T> struct RealOf;
template <> struct RealOf<double2> { using type = double; };
template <> struct RealOf<float2> { using type = float; };

template <typename T> __host__ __device__ __forceinline__ T cmake(typename RealOf<T>::type x, typename RealOf<T>::type y) {
    T r;
    r.x = x;
    r.y = y;
    return r;
}
template <typename T> __device__ __forceinline__ T cadd(T a, T b) { return cmake<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ T csub(T a, T b) { return cmake<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ T cmul(T a, T b) {
    return cmake<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename T> __device__ __forceinline__ T cmulc(T a, T b) {
    return cmake<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T> __device__ __forceinline__ T cscale(T a, typename RealOf<T>::type s) { return cmake<T>(a.x * s, a.y * s); }
// multiply by s*i, s = +1 or -1
template <typename T, int S> __device__ __forceinline__ T cmul_si(T a) {
    return S > 0 ? cmake<T>(-a.y, a.x) : cmake<T>(a.y, -a.x);
}

constexpr int kMaxPass = 12;

// One 1-D transform length: radix sequence and twiddle offsets (host-built).
struct FftPlan1D {
    int n;
    int npass;
    int radix[kMaxPass];
    int p[kMaxPass];
    int twoff[kMaxPass];  // offset of this pass's table inside the twiddle array
};

template <typename T, int DIR> __device__ __forceinline__ void dft2(T* u) {
    const T a = u[0];
    u[0] = cadd(a, u[1]);
    u[1] = csub(a, u[1]);
}

template <typename T, int DIR> __device__ __forceinline__ void dft3(T* u) {
    using R = typename RealOf<T>::type;
    const R s60 = R(0.86602540378443864676372317075294);  // sin(2 pi / 3)
    const T t1 = cadd(u[1], u[2]);
    const T t2 = cscale(cmul_si<T, DIR>(csub(u[1], u[2])), s60);
    const T m = csub(u[0], cscale(t1, R(0.5)));
    u[0] = cadd(u[0], t1);
    u[1] = cadd(m, t2);
    u[2] = csub(m, t2);
}

template <typename T, int DIR> __device__ __forceinline__ void dft4(T* u) {
    const T a0 = cadd(u[0], u[2]);
    const T a1 = csub(u[0], u[2]);
    const T b0 = cadd(u[1], u[3]);
    const T b1 = cmul_si<T, DIR>(csub(u[1], u[3]));
    u[0] = cadd(a0, b0);
    u[2] = csub(a0, b0);
    u[1] = cadd(a1, b1);
    u[3] = csub(a1, b1);
}

template <typename T, int DIR> __device__ __forceinline__ void dft5(T* u) {
    using R = typename RealOf<T>::type;
    const R c1 = R(0.30901699437494742410229341718282);   // cos(2 pi / 5)
    const R c2 = R(-0.80901699437494742410229341718282);  // cos(4 pi / 5)
    const R s1 = R(0.95105651629515357211643933337938);   // sin(2 pi / 5)
    const R s2 = R(0.58778525229247312916870595463907);   // sin(4 pi / 5)
    const T a1 = cadd(u[1], u[4]), b1 = csub(u[1], u[4]);
    const T a2 = cadd(u[2], u[3]), b2 = csub(u[2], u[3]);
    const T m1 = cadd(u[0], cadd(cscale(a1, c1), cscale(a2, c2)));
    const T m2 = cadd(u[0], cadd(cscale(a1, c2), cscale(a2, c1)));
    const T n1 = cmul_si<T, DIR>(cadd(cscale(b1, s1), cscale(b2, s2)));
    const T n2 = cmul_si<T, DIR>(csub(cscale(b1, s2), cscale(b2, s1)));
    u[0] = cadd(u[0], cadd(a1, a2));
    u[1] = cadd(m1, n1);
    u[4] = csub(m1, n1);
    u[2] = cadd(m2, n2);
    u[3] = csub(m2, n2);
}

template <typename T, int DIR, int R> __device__ __forceinline__ void dftR(T* u) {
    if constexpr (R == 2) dft2<T, DIR>(u);
    else if constexpr (R == 3) dft3<T, DIR>(u);
    else if constexpr (R == 4) dft4<T, DIR>(u);
    else dft5<T, DIR>(u);
}

// One Stockham pass over `howmany` transforms of length n.
template <typename T, int DIR, int R>
__device__ __forceinline__ void fft_pass(const T* __restrict__ src, T* __restrict__ dst, int n, int howmany, int es,
                                         int bs, int p, const T* __restrict__ tw, int tid, int nthr) {
    const int m = n / R;
    const int total = howmany * m;
    for (int t = tid; t < total; t += nthr) {
        const int b = t / m;
        const int i = t - b * m;
        const int k = i % p;
        const T* s = src + b * bs;
        T* d = dst + b * bs;
        T u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = s[(i + r * m) * es];
        if (p > 1) {
            const T* w = tw + k * (R - 1);
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const T wr = __ldg(w + r - 1);
                u[r] = DIR < 0 ? cmul(u[r], wr) : cmulc(u[r], wr);
            }
        }
        dftR<T, DIR, R>(u);
        const int j = (i - k) * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) d[(j + q * p) * es] = u[q];
    }
}

// `howmany` transforms of length pl.n stored at buf[b*bs + e*es]; tmp has the same geometry.
// Every thread of the block must call this (it contains __syncthreads).
template <typename T, int DIR>
__device__ void fft_batch(T* buf, T* tmp, int howmany, int es, int bs, const FftPlan1D& pl, const T* __restrict__ tw,
                          int tid, int nthr) {
    T* src = buf;
    T* dst = tmp;
    for (int ps = 0; ps < pl.npass; ++ps) {
        const T* t = tw + pl.twoff[ps];
        switch (pl.radix[ps]) {
            case 2: fft_pass<T, DIR, 2>(src, dst, pl.n, howmany, es, bs, pl.p[ps], t, tid, nthr); break;
            case 3: fft_pass<T, DIR, 3>(src, dst, pl.n, howmany, es, bs, pl.p[ps], t, tid, nthr); break;
            case 4: fft_pass<T, DIR, 4>(src, dst, pl.n, howmany, es, bs, pl.p[ps], t, tid, nthr); break;
            default: fft_pass<T, DIR, 5>(src, dst, pl.n, howmany, es, bs, pl.p[ps], t, tid, nthr); break;
        }
        __syncthreads();
        T* x = src;
        src = dst;
        dst = x;
    }
    if (src != buf) {
        const int total = howmany * pl.n;
        for (int t = tid; t < total; t += nthr) {
            const int b = t / pl.n;
            const int e = t - b * pl.n;
            buf[b * bs + e * es] = src[b * bs + e * es];
        }
        __syncthreads();
    }
}

}  // namespace b200
