// sm_100a bodies of ABACUS's DEVICE_GPU op functors on the H|psi> path.
//
// Each launcher has the argument meaning of the reference functor it replaces:
//   ekinetic_pw_op ....... source/module_hamilt_pw/hamilt_pwdft/kernels/ekinetic_op.h:38-48
//   veff_pw_op (npol 1/2)  source/module_hamilt_pw/hamilt_pwdft/kernels/veff_op.h:57-66
//   nonlocal_pw_op ....... source/module_hamilt_pw/hamilt_pwdft/kernels/nonlocal_op.h:82-113
//   set_3d_fft_box_op, set_recip_to_real_output_op, set_real_to_recip_output_op
//                          source/module_basis/module_pw/kernels/pw_op.h
// Grids are sized in multiples of the 148 SMs (grid-stride loops) so that
// large launches fill both dies and small ones stay a single wave.
#include "functors.h"

namespace b200 {

namespace {
constexpr int kThreads = 256;
inline int grid_for(long n) {
    const long blocks = (n + kThreads - 1) / kThreads;
    return int(blocks < 148L * 16 ? (blocks < 1 ? 1 : blocks) : 148L * 16);
}
}  // namespace

template <typename T, typename R>
__global__ void k_ekinetic(int nband, int npw, int max_npw, R tpiba2, const R* __restrict__ gk2, T* __restrict__ hpsi,
                           const T* __restrict__ psi) {
    const long total = long(nband) * npw;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int ib = int(t / npw);
        const int ig = int(t - long(ib) * npw);
        const long i = long(ib) * max_npw + ig;
        hpsi[i] = cadd(hpsi[i], cscale(psi[i], gk2[ig] * tpiba2));
    }
}

template <typename T, typename R>
__global__ void k_veff(long size, T* __restrict__ out, const R* __restrict__ v) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < size; i += long(gridDim.x) * blockDim.x)
        out[i] = cscale(out[i], v[i]);
}

template <typename T, typename R>
__global__ void k_veff_npol2(long size, T* __restrict__ out, T* __restrict__ out1, const R* __restrict__ v0,
                             const R* __restrict__ v1, const R* __restrict__ v2, const R* __restrict__ v3) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < size; i += long(gridDim.x) * blockDim.x) {
        const T a = out[i], b = out1[i];
        // sup = a (v0 + v3) + b (v1 - i v2); sdown = b (v0 - v3) + a (v1 + i v2)  (veff_op.cpp:27-35)
        const T m1 = cmake<T>(v1[i], -v2[i]);
        const T m2 = cmake<T>(v1[i], v2[i]);
        out[i] = cadd(cscale(a, v0[i] + v3[i]), cmul(b, m1));
        out1[i] = cadd(cscale(b, v0[i] - v3[i]), cmul(a, m2));
    }
}

// ps[(sum+ii*l3+kk)*l2 + jj] += sum_xx deeq[((spin*dx+iat+ii)*dy+xx)*dz+kk] * becp[jj*nkb+sum+ii*l3+xx]
template <typename T, typename R>
__global__ void k_nonlocal(int l1, int l2, int l3, int sum, int iat, int spin, int nkb, int dx, int dy, int dz,
                           const R* __restrict__ deeq, T* __restrict__ ps, const T* __restrict__ becp) {
    const long total = long(l1) * l2 * l3;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int jj = int(t % l2);  // band fastest: consecutive threads write consecutive ps entries
        const long r = t / l2;
        const int kk = int(r % l3);
        const int ii = int(r / l3);
        const R* d = deeq + (long(spin * dx + iat + ii) * dy) * dz + kk;
        const T* b = becp + long(jj) * nkb + sum + ii * l3;
        T acc = cmake<T>(0, 0);
        for (int xx = 0; xx < l3; ++xx) acc = cadd(acc, cscale(b[xx], d[long(xx) * dz]));
        T* o = ps + long(sum + ii * l3 + kk) * l2 + jj;
        *o = cadd(*o, acc);
    }
}

template <typename T>
__global__ void k_nonlocal_nc(int l1, int l2, int l3, int sum, int iat, int nkb, int dx, int dy, int dz,
                              const T* __restrict__ dnc, T* __restrict__ ps, const T* __restrict__ becp) {
    const int half = l2 / 2;
    const long total = long(l1) * half * l3;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int jj = 2 * int(t % half);
        const long r = t / half;
        const int kk = int(r % l3);
        const int ii = int(r / l3);
        const int ia = iat + ii;
        T a0 = cmake<T>(0, 0), a1 = cmake<T>(0, 0);
        for (int xx = 0; xx < l3; ++xx) {
            const long bi = long(jj) * nkb + sum + ii * l3 + xx;
            const T b1 = becp[bi], b2 = becp[bi + nkb];
            const long o = (long(ia) * dy + kk) * dz + xx;
            const long sstride = long(dx) * dy * dz;
            a0 = cadd(a0, cadd(cmul(dnc[o], b1), cmul(dnc[sstride + o], b2)));
            a1 = cadd(a1, cadd(cmul(dnc[2 * sstride + o], b1), cmul(dnc[3 * sstride + o], b2)));
        }
        const long psind = long(sum + ii * l3 + kk) * l2 + jj;
        ps[psind] = cadd(ps[psind], a0);
        ps[psind + 1] = cadd(ps[psind + 1], a1);
    }
}

template <typename T>
__global__ void k_set_box(int npwk, const int* __restrict__ idx, const T* __restrict__ in, T* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npwk; i += gridDim.x * blockDim.x) out[idx[i]] = in[i];
}

template <typename T, typename R>
__global__ void k_r2r_out(long nrxx, int add, R factor, const T* __restrict__ in, T* __restrict__ out) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < nrxx; i += long(gridDim.x) * blockDim.x)
        out[i] = add ? cadd(out[i], cscale(in[i], factor)) : in[i];
}

template <typename T, typename R>
__global__ void k_r2g_out(int npw, int add, R scale, const int* __restrict__ idx, const T* __restrict__ in,
                          T* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npw; i += gridDim.x * blockDim.x) {
        const T v = cscale(in[idx[i]], scale);
        out[i] = add ? cadd(out[i], v) : v;
    }
}

// ---------------------------------------------------------------- launchers
template <typename T, typename R>
void ekinetic_pw(int nband, int npw, int max_npw, R tpiba2, const R* gk2, T* hpsi, const T* psi, cudaStream_t s) {
    if (nband <= 0 || npw <= 0) return;
    k_ekinetic<T, R><<<grid_for(long(nband) * npw), kThreads, 0, s>>>(nband, npw, max_npw, tpiba2, gk2, hpsi, psi);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R> void veff_pw(long size, T* out, const R* in, cudaStream_t s) {
    if (size <= 0) return;
    k_veff<T, R><<<grid_for(size), kThreads, 0, s>>>(size, out, in);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R>
void veff_pw_npol2(long size, T* out, T* out1, const R* const in[4], cudaStream_t s) {
    if (size <= 0) return;
    k_veff_npol2<T, R><<<grid_for(size), kThreads, 0, s>>>(size, out, out1, in[0], in[1], in[2], in[3]);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R>
void nonlocal_pw(int l1, int l2, int l3, int& sum, int& iat, int spin, int nkb, int dx, int dy, int dz, const R* deeq,
                 T* ps, const T* becp, cudaStream_t s) {
    const long total = long(l1) * l2 * l3;
    if (total > 0) {
        k_nonlocal<T, R><<<grid_for(total), kThreads, 0, s>>>(l1, l2, l3, sum, iat, spin, nkb, dx, dy, dz, deeq, ps, becp);
        note_launch();
        B200_CUDA(cudaGetLastError());
    }
    sum += l1 * l3;
    iat += l1;
}

template <typename T>
void nonlocal_pw_nc(int l1, int l2, int l3, int& sum, int& iat, int nkb, int dx, int dy, int dz, const T* dnc, T* ps,
                    const T* becp, cudaStream_t s) {
    const long total = long(l1) * (l2 / 2) * l3;
    if (total > 0) {
        k_nonlocal_nc<T><<<grid_for(total), kThreads, 0, s>>>(l1, l2, l3, sum, iat, nkb, dx, dy, dz, dnc, ps, becp);
        note_launch();
        B200_CUDA(cudaGetLastError());
    }
    iat += l1;
    sum += l1 * l3;
}

template <typename T> void set_3d_fft_box(int npwk, const int* idx, const T* in, T* out, cudaStream_t s) {
    if (npwk <= 0) return;
    k_set_box<T><<<grid_for(npwk), kThreads, 0, s>>>(npwk, idx, in, out);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R>
void set_recip_to_real_output(long nrxx, int add, R factor, const T* in, T* out, cudaStream_t s) {
    if (nrxx <= 0) return;
    k_r2r_out<T, R><<<grid_for(nrxx), kThreads, 0, s>>>(nrxx, add, factor, in, out);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R>
void set_real_to_recip_output(int npw, long nxyz, int add, R factor, const int* idx, const T* in, T* out, cudaStream_t s) {
    if (npw <= 0) return;
    const R scale = add ? R(factor / R(nxyz)) : R(R(1) / R(nxyz));
    k_r2g_out<T, R><<<grid_for(npw), kThreads, 0, s>>>(npw, add, scale, idx, in, out);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

#define B200_INST(T, R)                                                                                              \
    template void ekinetic_pw<T, R>(int, int, int, R, const R*, T*, const T*, cudaStream_t);                         \
    template void veff_pw<T, R>(long, T*, const R*, cudaStream_t);                                                   \
    template void veff_pw_npol2<T, R>(long, T*, T*, const R* const[4], cudaStream_t);                                \
    template void nonlocal_pw<T, R>(int, int, int, int&, int&, int, int, int, int, int, const R*, T*, const T*,      \
                                    cudaStream_t);                                                                   \
    template void nonlocal_pw_nc<T>(int, int, int, int&, int&, int, int, int, int, const T*, T*, const T*,           \
                                    cudaStream_t);                                                                   \
    template void set_3d_fft_box<T>(int, const int*, const T*, T*, cudaStream_t);                                    \
    template void set_recip_to_real_output<T, R>(long, int, R, const T*, T*, cudaStream_t);                          \
    template void set_real_to_recip_output<T, R>(int, long, int, R, const int*, const T*, T*, cudaStream_t);
B200_INST(double2, double)
B200_INST(float2, float)
#undef B200_INST

}  // namespace b200
