// psi -> rho: ElecStatePW::psiToRho (module_elecstate/elecstate_pw.cpp:78-121, band loop :160-216) and its
// functor elecstate_pw_op (module_elecstate/kernels/elecstate_op.cpp:6-83).
//
// The functor entry points mirror the reference (rho is an array of nspin device pointers, host side).  The
// product path b200_pw_basis_psi_to_rho runs the reference's loop on the device: for every band with a
// non-zero weight, the drop-in transform recip_to_real into a full box, then rho[spin](r) += w1*|psi(r)|^2;
// nothing goes back to the host between bands.
#include <vector>

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
template <typename F> int guarded_r(F&& f) {
    try {
        f();
        b200::set_last_error("");
        return B200_STATUS_OK;
    } catch (const b200::Error& e) {
        b200::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        b200::set_last_error(e.what());
        return B200_STATUS_INVALID_ARGUMENT;
    }
}

template <typename T, typename R>
void psi_to_rho(b200_pw_basis* b, b200::DeviceArray<T>& box, b200::DeviceArray<T>& aux, int ik, int nbands, int ld,
                const T* psi, const double* w1, R* rho, cudaStream_t s) {
    b200::PWGrid& g = b->grid;
    B200_CHECK(ik >= 0 && ik < int(g.kmaps.size()), b200::kInvalidArgument, "k-point index out of range");
    B200_CHECK(nbands >= 0 && ld >= g.kmaps[ik].npw, b200::kInvalidArgument, "ld smaller than npwk");
    B200_CHECK(psi && w1 && rho, b200::kInvalidArgument, "NULL argument");
    g.ensure_device();
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
    return guarded_r([&] {
        b200::elecstate_call<double2, double>(spin, nrxx, w1, rho, (const double2*)wfcr_d, (cudaStream_t)stream);
    });
}
int b200_elecstate_pw_op_f32(int spin, int nrxx, float w1, float* const* rho, const void* wfcr_d, void* stream) {
    return guarded_r([&] {
        b200::elecstate_call<float2, float>(spin, nrxx, w1, rho, (const float2*)wfcr_d, (cudaStream_t)stream);
    });
}
int b200_elecstate_pw_op_nc_f64(int domag, int domag_z, int nrxx, double w1, double* const* rho, const void* wfcr_d,
                                const void* wfcr_another_spin_d, void* stream) {
    return guarded_r([&] {
        b200::elecstate_nc_call<double2, double>(domag, domag_z, nrxx, w1, rho, (const double2*)wfcr_d,
                                                 (const double2*)wfcr_another_spin_d, (cudaStream_t)stream);
    });
}
int b200_elecstate_pw_op_nc_f32(int domag, int domag_z, int nrxx, float w1, float* const* rho, const void* wfcr_d,
                                const void* wfcr_another_spin_d, void* stream) {
    return guarded_r([&] {
        b200::elecstate_nc_call<float2, float>(domag, domag_z, nrxx, w1, rho, (const float2*)wfcr_d,
                                               (const float2*)wfcr_another_spin_d, (cudaStream_t)stream);
    });
}

int b200_pw_basis_psi_to_rho_f64(b200_pw_basis* b, int ik, int nbands, int ld, const void* psi_d, const double* w1,
                                 double* rho_d, void* stream) {
    return guarded_r([&] {
        B200_CHECK(b != nullptr, b200::kInvalidArgument, "NULL basis");
        psi_to_rho<double2, double>(b, b->rho_box64, b->aux64, ik, nbands, ld, (const double2*)psi_d, w1, rho_d,
                                    (cudaStream_t)stream);
    });
}
int b200_pw_basis_psi_to_rho_f32(b200_pw_basis* b, int ik, int nbands, int ld, const void* psi_d, const double* w1,
                                 float* rho_d, void* stream) {
    return guarded_r([&] {
        B200_CHECK(b != nullptr, b200::kInvalidArgument, "NULL basis");
        psi_to_rho<float2, float>(b, b->rho_box32, b->aux32, ik, nbands, ld, (const float2*)psi_d, w1, rho_d,
                                  (cudaStream_t)stream);
    });
}

}  // extern "C"
