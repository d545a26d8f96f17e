// Plane pass of the fused local H|psi> on two-pass register transforms (square planes N = R1 * R2).
//
// Each 1-D transform of length N = R1 * R2 is done in two register passes with one exchange through
// shared memory between them ("four-step" inside a CTA):
//   pass A  (R2 threads per line)  thread t holds f[R2*n1 + t], n1 < R1: an R1-point DFT in registers,
//                                  then the twiddle W_N^(t*k1);
//   pass B  (R1 threads per line)  thread k1 holds the R2 values (k1, t), t < R2: an R2-point DFT in
//                                  registers gives X[k1 + R1*k2], k2 < R2.
// Inverse (exp(+i)):  X[k1 + R1 k2] = sum_t W_R2^(-t k2) W_N^(-t k1) sum_n1 W_R1^(-n1 k1) f[R2 n1 + t].
// The forward transform (exp(-i)) is the same factorisation run backwards (pass B, then pass A), so the
// r-space values stay in the (k1, k2) order of pass B in between and V_eff(r) multiplies them there.
//
// Per (band, z slot) CTA: the occupied x-columns of the plane in shared memory, column-major, every
// column in "block" order: position p = R2*k + t' of a column lives at k*(R2+1) + t' (a pad every R2
// entries, so that pass B's threads, R2+1 entries apart, fall on different banks).  The inverse y
// transform's pass A reads the plane's sticks straight from the stick buffer through the (column, y) ->
// stick map (zero where a column has no stick) and the forward y transform's pass A writes them back the
// same way, so the plane enters and leaves shared memory only in transformed form.  The y transforms run
// in place on the columns: after the inverse, position p of a column holds y = p/R2 + R1*(p mod R2).  The
// x transforms take rows of RB positions at a time through a row buffer laid out [row][k1][t] with the
// same padding; the forward x transform writes back the occupied columns only.  V_eff comes pre-arranged
// as vt[z slot][p][k1][k2] = V(z, y(p), x = k1 + R1*k2), so pass B reads its R2 values contiguously.
//
// Small DFTs: Q = A*B point transforms composed from 2/3/4-point ones with the twiddles W_Q^j as exact
// constants (cos / sin of multiples of 7.5 degrees, the algebraic values); multiplications by 1, -1, +-i
// are folded away at compile time.  Twiddles W_N^j of the length-N transform come from the host-built
// root table (W_N^j = exp(-2 pi i j / N)).
#pragma once
#include "fft_core.cuh"
#include "pw_grid.h"

namespace b200 {
namespace plane_t {

// cos(k * 7.5 degrees), k integer
constexpr double cos48_q(int k) {  // first quadrant, k in [0, 12]
    return k == 0 ? 1.0
         : k == 3 ? 0.92387953251128675612818318939679   // cos 22.5
         : k == 4 ? 0.86602540378443864676372317075294   // cos 30
         : k == 6 ? 0.70710678118654752440084436210485   // cos 45
         : k == 8 ? 0.5                                   // cos 60
         : k == 9 ? 0.38268343236508977172845998403040   // cos 67.5
         : k == 12 ? 0.0
         : 2.0;  // not used (flags an unsupported angle)
}
constexpr double cos48(int k) {
    k %= 48;
    if (k < 0) k += 48;
    if (k <= 12) return cos48_q(k);
    if (k <= 24) return -cos48_q(24 - k);
    if (k <= 36) return -cos48_q(k - 24);
    return cos48_q(48 - k);
}
constexpr double sin48(int k) { return cos48(12 - k); }
// W_Q^j = exp(-2 pi i j / Q) as (re, im); Q divides 48
constexpr double wre(int Q, int j) { return cos48(j * (48 / Q)); }
constexpr double wim(int Q, int j) { return -sin48(j * (48 / Q)); }

// u * W_Q^(DIR<0 ? j : -j), with the trivial cases folded
template <typename T, int DIR, int Q, int J>
__device__ __forceinline__ T twc(T u) {
    using R = typename RealOf<T>::type;
    constexpr int j = ((J % Q) + Q) % Q;
    constexpr int e = DIR < 0 ? j : (Q - j) % Q;  // exponent of W_Q = exp(-2 pi i / Q)
    constexpr int q4 = (4 * e) % Q == 0 ? (4 * e) / Q : -1;  // quarter turns, if e is one
    if constexpr (e == 0) {
        return u;
    } else if constexpr (q4 == 1) {  // -i
        return cmake<T>(u.y, -u.x);
    } else if constexpr (q4 == 2) {
        return cmake<T>(-u.x, -u.y);
    } else if constexpr (q4 == 3) {  // +i
        return cmake<T>(-u.y, u.x);
    } else {
        constexpr double c = wre(Q, e), s = wim(Q, e);
        if constexpr (c == s) {  // (x + iy)(c + ic): two adds, two multiplies
            return cmake<T>((u.x - u.y) * R(c), (u.x + u.y) * R(c));
        } else if constexpr (c == -s) {  // (x + iy)(c - ic)
            return cmake<T>((u.x + u.y) * R(c), (u.y - u.x) * R(c));
        } else {
            return cmake<T>(fma(u.x, R(c), -u.y * R(s)), fma(u.x, R(s), u.y * R(c)));
        }
    }
}

// y[n2][k1] *= W_Q^(n2 k1) (DIR < 0) or its conjugate, for I = n2*A + k1 from I0 on
template <typename T, int DIR, int Q, int A, int B, int I>
__device__ __forceinline__ void tw_all(T (*y)[A]) {
    if constexpr (I < A * B) {
        y[I / A][I % A] = twc<T, DIR, Q, (I / A) * (I % A)>(y[I / A][I % A]);
        tw_all<T, DIR, Q, A, B, I + 1>(y);
    }
}

// Q-point DFT in registers, natural order in and out; DIR = -1: exp(-i), +1: exp(+i)
template <typename T, int DIR, int Q>
__device__ __forceinline__ void dft(T* u) {
    if constexpr (Q <= 5) {
        dftR<T, DIR, Q>(u);
    } else {
        constexpr int A = (Q % 4 == 0) ? 4 : (Q % 3 == 0 ? 3 : 2);
        constexpr int B = Q / A;
        T y[B][A];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) {
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) y[n2][n1] = u[B * n1 + n2];
            dftR<T, DIR, A>(y[n2]);
        }
        tw_all<T, DIR, Q, A, B, 0>(y);  // y[n2][k1] *= W_Q^(+-n2 k1), compile-time exponents
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            T z[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) z[n2] = y[n2][k1];
            dft<T, DIR, B>(z);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) u[k1 + A * k2] = z[k2];
        }
    }
}

template <int R1, int R2> struct Geom {
    static constexpr int RS = R2 + 1;                 // stride of a k block (R2 entries + pad)
    static constexpr int LDC = (R1 * RS) | 1;         // column pitch (odd: x neighbours on distinct banks)
    __host__ __device__ static constexpr int pos(int p) { return (p / R2) * RS + p % R2; }
};

template <typename T>
__host__ __device__ constexpr size_t smem_bytes(int R1, int R2, int RB, int N, int nxc) {
    return (size_t(nxc) * size_t((R1 * (R2 + 1)) | 1) + size_t(RB) * R1 * (R2 + 1)) * sizeof(T) + size_t(N) * sizeof(int);
}

// z slot -> z of the register z passes (slot s holds z = s/32 + m*bitrev5(s mod 32), m = nz/32)
__device__ __forceinline__ int zslot_to_z(int s, int m) { return (s >> 5) + m * int(__brev(unsigned(s & 31)) >> 27); }

// vt[zs][p][k1][k2] = veff_zyx[z(zs)][y(p)][k1 + R1*k2], y(p) = p/R2 + R1*(p mod R2)
template <typename R>
__global__ void k_arrange_veff(int nz, int n, int r1, int r2, const R* __restrict__ vzyx, R* __restrict__ vt) {
    const long total = long(nz) * n * n;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int k2 = int(i % r2);
        const int k1 = int((i / r2) % r1);
        const int p = int((i / n) % n);
        const int zs = int(i / (long(n) * n));
        const int z = zslot_to_z(zs, nz / 32);
        const int y = p / r2 + r1 * (p % r2);
        vt[i] = vzyx[(long(z) * n + y) * n + k1 + r1 * k2];
    }
}

// The twiddles W_N^(t*k1) of one thread: with NT a multiple of R1 and R2, a thread keeps the same t in every
// pass-A item and the same k1 in every pass-B item, so it loads its R1-1 (pass A) and R2-1 (pass B) twiddles
// once; otherwise they are read per item from the (L1-resident) root table.
template <typename T, int N, int R1, int R2, int NT> struct Twiddles {
    static constexpr bool kFixed = NT % R1 == 0 && NT % R2 == 0;
    T a[kFixed ? R1 : 1], b[kFixed ? R2 : 1];
    __device__ __forceinline__ void load(const T* __restrict__ roots, int tid) {
        if constexpr (kFixed) {
            const int t = tid % R2, k1 = tid % R1;
#pragma unroll
            for (int j = 1; j < R1; ++j) a[j] = __ldg(roots + (t * j) % N);
#pragma unroll
            for (int j = 1; j < R2; ++j) b[j] = __ldg(roots + (j * k1) % N);
        }
    }
    // W_N^(t*j) for pass A (thread's t, j = k1) and pass B (j = t, thread's k1)
    __device__ __forceinline__ T wa(const T* __restrict__ roots, int t, int j) const {
        if constexpr (kFixed) return a[j];
        else return __ldg(roots + (t * j) % N);
    }
    __device__ __forceinline__ T wb(const T* __restrict__ roots, int k1, int j) const {
        if constexpr (kFixed) return b[j];
        else return __ldg(roots + (j * k1) % N);
    }
};

// One CTA per (band, z slot): inverse y and x transforms, x V_eff(r), forward x and y transforms.
template <typename T, typename R, int N, int R1, int R2, int NT, int RB, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_plane_t(PlaneMapView pm, int nz, const T* __restrict__ roots,
                                                      const R* __restrict__ vt, T* __restrict__ sb) {
    static_assert(R1 * R2 == N && N % RB == 0, "plane geometry");
    using G = Geom<R1, R2>;
    constexpr int RS = G::RS, LDC = G::LDC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nxc = pm.nxc;
    T* A = reinterpret_cast<T*>(smem_raw);
    T* buf = A + size_t(nxc) * LDC;
    int* cmap = reinterpret_cast<int*>(buf + RB * R1 * RS);
    const int tid = threadIdx.x;
    const int band = blockIdx.x, zs = blockIdx.y;
    const T zero = cmake<T>(0, 0);
    Twiddles<T, N, R1, R2, NT> tw;
    tw.load(roots, tid);

    for (int i = tid; i < N; i += NT) cmap[i] = -1;
    __syncthreads();
    for (int c = tid; c < nxc; c += NT) cmap[pm.xpos[c]] = c;
    T* plane = sb + (size_t(band) * nz + zs) * pm.nst;

    // ---- inverse y: pass A on (column, t) straight from the plane's sticks (y without a stick is zero), pass B
    // on (column, k1) ----
    for (int i = tid; i < nxc * R2; i += NT) {
        const int c = i / R2, t = i % R2;
        const int* sm = pm.smap + c * N + t;
        int si[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) si[n1] = __ldg(sm + n1 * R2);
        T u[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) u[n1] = si[n1] >= 0 ? plane[si[n1]] : zero;
        dft<T, +1, R1>(u);
#pragma unroll
        for (int k1 = 1; k1 < R1; ++k1) u[k1] = cmulc(u[k1], tw.wa(roots, t, k1));
        T* col = A + c * LDC + t;
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) col[k1 * RS] = u[k1];
    }
    __syncthreads();
    for (int i = tid; i < nxc * R1; i += NT) {
        const int c = i / R1, k1 = i % R1;
        T* blk = A + c * LDC + k1 * RS;
        T v[R2];
#pragma unroll
        for (int t = 0; t < R2; ++t) v[t] = blk[t];
        dft<T, +1, R2>(v);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) blk[k2] = v[k2];
    }
    __syncthreads();

    // ---- x: rows of RB positions; inverse, x V_eff, forward ----
    // FP64: a thread's pass-A items all have t = tid % R2 (NT is a multiple of R2), so its R1 column indices
    // cmap[R2 n1 + t] are read once, packed one byte each (0xFF: no occupied column), instead of from shared
    // memory in every pass-A item of every row batch (FP32 CTAs, four per SM, have no registers to spare)
    static_assert(NT % R2 == 0, "x pass A: one t per thread");
    constexpr bool kPack = sizeof(T) == 16;
    constexpr int NPK = kPack ? (R1 + 3) / 4 : 1;
    unsigned cpk[NPK];
    if constexpr (kPack) {
        const int tx = tid % R2;
#pragma unroll
        for (int w = 0; w < NPK; ++w) cpk[w] = 0;
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) {
            const int cm = cmap[R2 * n1 + tx];
            cpk[n1 / 4] |= unsigned(cm < 0 ? 0xFF : cm) << (8 * (n1 % 4));
        }
    }
    auto col_of = [&](int n1, int t) -> int {
        if constexpr (kPack) {
            const unsigned b = (cpk[n1 / 4] >> (8 * (n1 % 4))) & 0xFFu;
            return b == 0xFFu ? -1 : int(b);
        } else {
            return cmap[R2 * n1 + t];
        }
    };
    const R* vz = vt + size_t(zs) * N * N;
    for (int p0 = 0; p0 < N; p0 += RB) {
        for (int i = tid; i < RB * R2; i += NT) {
            const int r = i / R2, t = i % R2;
            const int pp = G::pos(p0 + r);
            T u[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) {
                const int cm = col_of(n1, t);
                u[n1] = cm >= 0 ? A[cm * LDC + pp] : zero;
            }
            dft<T, +1, R1>(u);
#pragma unroll
            for (int k1 = 1; k1 < R1; ++k1) u[k1] = cmulc(u[k1], tw.wa(roots, t, k1));
            T* b = buf + r * R1 * RS + t;
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) b[k1 * RS] = u[k1];
        }
        __syncthreads();
        for (int i = tid; i < RB * R1; i += NT) {
            const int r = i / R1, k1 = i % R1;
            // V_eff of the item first: its loads are in flight during the inverse transform
            const R* vv = vz + (size_t(p0 + r) * R1 + k1) * R2;
            R vr[R2];
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) vr[k2] = __ldg(vv + k2);
            T* b = buf + (r * R1 + k1) * RS;
            T v[R2];
#pragma unroll
            for (int t = 0; t < R2; ++t) v[t] = b[t];
            dft<T, +1, R2>(v);
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) v[k2] = cscale(v[k2], vr[k2]);
            dft<T, -1, R2>(v);
#pragma unroll
            for (int t = 1; t < R2; ++t) v[t] = cmul(v[t], tw.wb(roots, k1, t));
#pragma unroll
            for (int t = 0; t < R2; ++t) b[t] = v[t];
        }
        __syncthreads();
        for (int i = tid; i < RB * R2; i += NT) {
            const int r = i / R2, t = i % R2;
            const int pp = G::pos(p0 + r);
            const T* b = buf + r * R1 * RS + t;
            T u[R1];
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) u[k1] = b[k1 * RS];
            dft<T, -1, R1>(u);
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) {
                const int cm = col_of(n1, t);
                if (cm >= 0) A[cm * LDC + pp] = u[n1];
            }
        }
        __syncthreads();
    }

    // ---- forward y: pass B on (column, k1), pass A on (column, t) ----
    for (int i = tid; i < nxc * R1; i += NT) {
        const int c = i / R1, k1 = i % R1;
        T* blk = A + c * LDC + k1 * RS;
        T v[R2];
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[k2] = blk[k2];
        dft<T, -1, R2>(v);
#pragma unroll
        for (int t = 1; t < R2; ++t) v[t] = cmul(v[t], tw.wb(roots, k1, t));
#pragma unroll
        for (int t = 0; t < R2; ++t) blk[t] = v[t];
    }
    __syncthreads();
    for (int i = tid; i < nxc * R2; i += NT) {
        const int c = i / R2, t = i % R2;
        const T* col = A + c * LDC + t;
        T u[R1];
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) u[k1] = col[k1 * RS];
        dft<T, -1, R1>(u);
        // straight back to the plane's sticks
        const int* sm = pm.smap + c * N + t;
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) {
            const int si = __ldg(sm + n1 * R2);
            if (si >= 0) plane[si] = u[n1];
        }
    }
}

}  // namespace plane_t
}  // namespace b200

namespace b200 {
namespace plane_t {

// One complex value global -> shared memory as an asynchronous copy (cp.async, 8 or 16 bytes): the value does
// not pass through a register, so a thread has all its copies of a loop in flight at once; cp_async_wait_all
// then __syncthreads make them visible to the CTA.
template <typename T> __device__ __forceinline__ void cp_async_value(T* dst_shared, const T* src_global) {
    static_assert(sizeof(T) == 8 || sizeof(T) == 16, "complex float or double");
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst_shared));
    if constexpr (sizeof(T) == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src_global) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src_global) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---- z passes on the two-pass transforms (nz = R1 * R2), TS sticks per CTA, NT threads ----
// The stick buffer keeps the layout of the warp-shuffle z passes: plane slot s holds z = zslot_to_z(s), so
// the plane passes and psi -> rho see the same buffer whichever z pass wrote it.  In shared memory a stick
// is in block order: natural z = R2*n1 + t at n1*(R2+1) + t before the inverse transform; after it, output
// z = k1 + R1*k2 sits at k1*(R2+1) + k2.
template <int R1, int R2> __host__ __device__ constexpr int zpos_natural(int z) { return (z / R2) * (R2 + 1) + z % R2; }
template <int R1, int R2> __host__ __device__ constexpr int zpos_output(int z) { return (z % R1) * (R2 + 1) + z / R1; }
template <typename T> constexpr size_t zpass_smem_bytes(int R1, int R2, int TS) { return size_t(TS) * ((R1 * (R2 + 1)) | 1) * sizeof(T); }

template <typename T, int NZ, int R1, int R2, int TS, int NT, typename Src>
__global__ void __launch_bounds__(NT) k_zinv_t(Src src, int b0, int nbc, const T* __restrict__ roots, T* __restrict__ sb) {
    static_assert(R1 * R2 == NZ && NZ % 32 == 0, "z geometry");
    constexpr int RS = R2 + 1, LDZ = (R1 * RS) | 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);  // TS sticks of LDZ
    const KBatchEntry& e = src.get(blockIdx.z);
    const StickMapView sm = e.sm;
    const int tid = threadIdx.x;
    const int s0 = blockIdx.x * TS;
    if (s0 >= sm.nst) return;
    const int ns = min(TS, sm.nst - s0);
    const int band = blockIdx.y;
    const T zero = cmake<T>(0, 0);
    Twiddles<T, NZ, R1, R2, NT> tw;
    tw.load(roots, tid);
    for (int i = tid; i < ns * LDZ; i += NT) A[i] = zero;
    __syncthreads();
    const T* p = reinterpret_cast<const T*>(e.psi) + size_t(b0 + band) * e.ld;
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    // the sphere's values straight into their stick positions, every copy of the loop in flight at once
    for (int j = j0 + tid; j < j1; j += NT) {
        const int pk = sm.gpk[j];
        cp_async_value(A + ((pk >> 10) - s0) * LDZ + zpos_natural<R1, R2>(pk & 1023), p + sm.glist[j]);
    }
    cp_async_wait_all();
    __syncthreads();
    for (int i = tid; i < ns * R2; i += NT) {
        const int sl = i / R2, t = i % R2;
        T* st = A + sl * LDZ + t;
        T u[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) u[n1] = st[n1 * RS];
        dft<T, +1, R1>(u);
#pragma unroll
        for (int k1 = 1; k1 < R1; ++k1) u[k1] = cmulc(u[k1], tw.wa(roots, t, k1));
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) st[k1 * RS] = u[k1];
    }
    __syncthreads();
    for (int i = tid; i < ns * R1; i += NT) {
        const int sl = i / R1, k1 = i % R1;
        T* blk = A + sl * LDZ + k1 * RS;
        T v[R2];
#pragma unroll
        for (int t = 0; t < R2; ++t) v[t] = blk[t];
        dft<T, +1, R2>(v);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) blk[k2] = v[k2];
    }
    __syncthreads();
    T* out = sb + (size_t(blockIdx.z) * nbc + band) * NZ * sm.nst;
    for (int i = tid; i < ns * NZ; i += NT) {
        const int sz = i / ns;
        const int sl = i - sz * ns;
        out[size_t(sz) * sm.nst + s0 + sl] = A[sl * LDZ + zpos_output<R1, R2>(zslot_to_z(sz, NZ / 32))];
    }
}

template <typename T, typename R, int NZ, int R1, int R2, int TS, int NT, typename Src>
__global__ void __launch_bounds__(NT) k_zfwd_t(Src src, int b0, int nbc, const T* __restrict__ roots,
                                               const T* __restrict__ sb, R tpiba2, R invn, int accumulate) {
    static_assert(R1 * R2 == NZ && NZ % 32 == 0, "z geometry");
    constexpr int RS = R2 + 1, LDZ = (R1 * RS) | 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);  // TS sticks of LDZ
    const KBatchEntry& e = src.get(blockIdx.z);
    const StickMapView sm = e.sm;
    const int tid = threadIdx.x;
    const int s0 = blockIdx.x * TS;
    if (s0 >= sm.nst) return;
    const int ns = min(TS, sm.nst - s0);
    const int band = blockIdx.y;
    Twiddles<T, NZ, R1, R2, NT> tw;
    tw.load(roots, tid);
    const T* in = sb + (size_t(blockIdx.z) * nbc + band) * NZ * sm.nst;
    // the stick planes of this tile (ns sticks of every z slot) as asynchronous copies, all in flight at once
    for (int i = tid; i < ns * NZ; i += NT) {
        const int sz = i / ns;
        const int sl = i - sz * ns;
        cp_async_value(A + sl * LDZ + zpos_output<R1, R2>(zslot_to_z(sz, NZ / 32)), in + size_t(sz) * sm.nst + s0 + sl);
    }
    cp_async_wait_all();
    __syncthreads();
    for (int i = tid; i < ns * R1; i += NT) {
        const int sl = i / R1, k1 = i % R1;
        T* blk = A + sl * LDZ + k1 * RS;
        T v[R2];
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[k2] = blk[k2];
        dft<T, -1, R2>(v);
#pragma unroll
        for (int t = 1; t < R2; ++t) v[t] = cmul(v[t], tw.wb(roots, k1, t));
#pragma unroll
        for (int t = 0; t < R2; ++t) blk[t] = v[t];
    }
    __syncthreads();
    for (int i = tid; i < ns * R2; i += NT) {
        const int sl = i / R2, t = i % R2;
        T* st = A + sl * LDZ + t;
        T u[R1];
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) u[k1] = st[k1 * RS];
        dft<T, -1, R1>(u);
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) st[n1 * RS] = u[n1];
    }
    __syncthreads();
    const T* p = reinterpret_cast<const T*>(e.psi) + size_t(b0 + band) * e.ld;
    T* h = reinterpret_cast<T*>(e.hpsi) + size_t(b0 + band) * e.ld;
    const R* gk2 = reinterpret_cast<const R*>(e.gk2);
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    for (int j = j0 + tid; j < j1; j += NT) {
        const int pk = sm.gpk[j];
        const int g = sm.glist[j];
        T v = cscale(A[((pk >> 10) - s0) * LDZ + zpos_natural<R1, R2>(pk & 1023)], invn);
        v = cadd(v, cscale(p[g], gk2[g] * tpiba2));
        if (accumulate) v = cadd(v, h[g]);
        h[g] = v;
    }
    if (!accumulate && blockIdx.x == 0)
        for (int g = e.npw + tid; g < e.ld; g += NT) h[g] = cmake<T>(0, 0);
}

}  // namespace plane_t
}  // namespace b200
