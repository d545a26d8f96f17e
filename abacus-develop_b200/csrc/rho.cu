// psi -> rho: ElecStatePW::psiToRho (module_elecstate/elecstate_pw.cpp:78-121, band loop :160-216) and its
// functor elecstate_pw_op (module_elecstate/kernels/elecstate_op.cpp:6-83).
//
// The functor entry points mirror the reference (rho is an array of nspin device pointers, host side).  The
// product path b200_pw_basis_psi_to_rho computes the reference's sum rho(r) += w1_b |psi_b(r)|^2 over the
// bands with a non-zero weight: on grids with register transforms (nx = ny and nx, nz in {64, 96, 128})
// fused into two passes per band chunk (inverse z transform of the sticks; per z plane the inverse y and x
// transforms with |psi|^2 summed in registers) and one final reduction; elsewhere by the reference's loop,
// the drop-in transform recip_to_real into a full box and elecstate_pw_op per band.  Nothing goes back to
// the host between bands.  One call at a time per basis handle (its scratch is shared).
#include <algorithm>
#include <vector>

#include "capi_guard.h"
#include "../../include/abacus_b200.h"
#include "capi_handles.h"

namespace b200 {
namespace {

template <typename T, typename R>
__global__ void k_elecstate(long nrxx, R w1, R* __restrict__ rho, const T* __restrict__ wfcr) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < nrxx; i += long(gridDim.x) * blockDim.x) {
        const T v = wfcr[i];
        rho[i] += w1 * (v.x * v.x + v.y * v.y);
    }
}

// the nspin = 4 overload: rho[0] += w1 (|a|^2 + |b|^2); with DOMAG the magnetisation components
// 2 Re(a* b), 2 Im(a* b) (as written there: ar*bi - br*ai) and |a|^2 - |b|^2; with DOMAG_Z only the last,
// the other two set to zero; otherwise rho[1..3] set to zero (elecstate_op.cpp:27-80)
template <typename T, typename R>
__global__ void k_elecstate_nc(int domag, int domag_z, long nrxx, R w1, R* __restrict__ r0, R* __restrict__ r1,
                               R* __restrict__ r2, R* __restrict__ r3, const T* __restrict__ a,
                               const T* __restrict__ b) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < nrxx; i += long(gridDim.x) * blockDim.x) {
        const T u = a[i], v = b[i];
        const R nu = u.x * u.x + u.y * u.y, nv = v.x * v.x + v.y * v.y;
        r0[i] += w1 * (nu + nv);
        if (domag) {
            r1[i] += w1 * R(2) * (u.x * v.x + u.y * v.y);
            r2[i] += w1 * R(2) * (u.x * v.y - v.x * u.y);
            r3[i] += w1 * (nu - nv);
        } else if (domag_z) {
            r1[i] = R(0);
            r2[i] = R(0);
            r3[i] += w1 * (nu - nv);
        } else {
            r1[i] = R(0);
            r2[i] = R(0);
            r3[i] = R(0);
        }
    }
}

inline int blocks_for(long n) {
    long b = (n + 255) / 256;
    return int(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

template <typename T, typename R>
void elecstate_call(int spin, int nrxx, R w1, R* const* rho, const T* wfcr, cudaStream_t s) {
    B200_CHECK(rho && wfcr && spin >= 0 && nrxx >= 0, kInvalidArgument, "bad argument");
    B200_CHECK(rho[spin] != nullptr, kInvalidArgument, "NULL rho[spin]");
    if (nrxx == 0) return;
    k_elecstate<T, R><<<blocks_for(nrxx), 256, 0, s>>>(nrxx, w1, rho[spin], wfcr);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R>
void elecstate_nc_call(int domag, int domag_z, int nrxx, R w1, R* const* rho, const T* a, const T* b, cudaStream_t s) {
    B200_CHECK(rho && a && b && nrxx >= 0, kInvalidArgument, "bad argument");
    B200_CHECK(rho[0] && rho[1] && rho[2] && rho[3], kInvalidArgument, "NULL rho component");
    if (nrxx == 0) return;
    k_elecstate_nc<T, R><<<blocks_for(nrxx), 256, 0, s>>>(domag, domag_z, nrxx, w1, rho[0], rho[1], rho[2], rho[3], a,
                                                          b);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

}  // namespace
}  // namespace b200

namespace {
using b200::guarded;

template <typename T, typename R>
void psi_to_rho(b200_pw_basis* b, b200::DeviceArray<T>& box, b200::DeviceArray<T>& aux, b200::DeviceArray<T>& sbuf,
                b200::DeviceArray<R>& ws, int ik, int nbands, int ld, const T* psi, const double* w1, R* rho,
                cudaStream_t s) {
    b200::PWGrid& g = b->grid;
    B200_CHECK(ik >= 0 && ik < int(g.kmaps.size()), b200::kInvalidArgument, "k-point index out of range");
    B200_CHECK(nbands >= 0 && ld >= g.kmaps[ik].npw, b200::kInvalidArgument, "ld smaller than npwk");
    B200_CHECK(psi && w1 && rho, b200::kInvalidArgument, "NULL argument");
    g.ensure_device();
    if (nbands > 0 && b200::rho_r_supported(g)) {
        // the same sum on the register transforms: runs of consecutive bands with a non-zero weight (the
        // reference skips the others, elecstate_pw.cpp:211), in chunks whose stick buffer is about 48 MB
        b->rho_w.resize(size_t(nbands));
        B200_CUDA(cudaMemcpyAsync(b->rho_w.ptr, w1, size_t(nbands) * sizeof(double), cudaMemcpyHostToDevice, s));
        const size_t per_band = size_t(g.nz) * g.nst;
        const int chunk = int(std::max<size_t>(1, (size_t(48) << 20) / (per_band * sizeof(T))));
        sbuf.resize(size_t(std::min(chunk, nbands)) * per_band);
        const int nsplit = std::max(1, std::min(8, (2 * 148 + g.nz - 1) / g.nz));  // about two CTAs per SM
        ws.resize(size_t(nsplit) * size_t(g.nxyz()));
        int first = 1;
        for (int b0 = 0; b0 < nbands;) {
            if (w1[b0] == 0.0) {
                ++b0;
                continue;
            }
            int b1 = b0;
            while (b1 < nbands && w1[b1] != 0.0 && b1 - b0 < chunk) ++b1;
            b200::launch_rho_chunk_r<T, R>(g, ik, b0, b1 - b0, ld, psi, b->rho_w.ptr + b0, sbuf.ptr, nsplit, ws.ptr,
                                           first, s);
            first = 0;
            b0 = b1;
        }
        if (!first) b200::launch_rho_reduce_r<R>(g, nsplit, ws.ptr, rho, s);
        return;
    }
    const long N = g.nxyz();
    box.resize(size_t(N));
    aux.resize(size_t(N));
    for (int ib = 0; ib < nbands; ++ib) {
        if (w1[ib] == 0.0) continue;  // only occupied bands (elecstate_pw.cpp:211)
        b200::launch_recip_to_real<T>(g, ik, psi + size_t(ib) * ld, box.ptr, aux.ptr, 0, 1.0, s);
        b200::k_elecstate<T, R><<<b200::blocks_for(N), 256, 0, s>>>(N, R(w1[ib]), rho, box.ptr);
        b200::note_launch();
        B200_CUDA(cudaGetLastError());
    }
}
}  // namespace

extern "C" {

int b200_elecstate_pw_op_f64(int spin, int nrxx, double w1, double* const* rho, const void* wfcr_d, void* stream) {
    return guarded([&] {
        b200::elecstate_call<double2, double>(spin, nrxx, w1, rho, (const double2*)wfcr_d, (cudaStream_t)stream);
    });
}
int b200_elecstate_pw_op_f32(int spin, int nrxx, float w1, float* const* rho, const void* wfcr_d, void* stream) {
    return guarded([&] {
        b200::elecstate_call<float2, float>(spin, nrxx, w1, rho, (const float2*)wfcr_d, (cudaStream_t)stream);
    });
}
int b200_elecstate_pw_op_nc_f64(int domag, int domag_z, int nrxx, double w1, double* const* rho, const void* wfcr_d,
                                const void* wfcr_another_spin_d, void* stream) {
    return guarded([&] {
        b200::elecstate_nc_call<double2, double>(domag, domag_z, nrxx, w1, rho, (const double2*)wfcr_d,
                                                 (const double2*)wfcr_another_spin_d, (cudaStream_t)stream);
    });
}
int b200_elecstate_pw_op_nc_f32(int domag, int domag_z, int nrxx, float w1, float* const* rho, const void* wfcr_d,
                                const void* wfcr_another_spin_d, void* stream) {
    return guarded([&] {
        b200::elecstate_nc_call<float2, float>(domag, domag_z, nrxx, w1, rho, (const float2*)wfcr_d,
                                               (const float2*)wfcr_another_spin_d, (cudaStream_t)stream);
    });
}

int b200_pw_basis_psi_to_rho_f64(b200_pw_basis* b, int ik, int nbands, int ld, const void* psi_d, const double* w1,
                                 double* rho_d, void* stream) {
    return guarded([&] {
        B200_CHECK(b != nullptr, b200::kInvalidArgument, "NULL basis");
        psi_to_rho<double2, double>(b, b->rho_box64, b->aux64, b->rho_sb64, b->rho_ws64, ik, nbands, ld,
                                    (const double2*)psi_d, w1, rho_d, (cudaStream_t)stream);
    });
}
int b200_pw_basis_psi_to_rho_f32(b200_pw_basis* b, int ik, int nbands, int ld, const void* psi_d, const double* w1,
                                 float* rho_d, void* stream) {
    return guarded([&] {
        B200_CHECK(b != nullptr, b200::kInvalidArgument, "NULL basis");
        psi_to_rho<float2, float>(b, b->rho_box32, b->aux32, b->rho_sb32, b->rho_ws32, ik, nbands, ld,
                                  (const float2*)psi_d, w1, rho_d, (cudaStream_t)stream);
    });
}

}  // extern "C"
