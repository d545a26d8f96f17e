// Projector generation on the device: pseudopot_cell_vnl::getvnl (VNL_in_pw.cpp:412-540) and the three
// functors it composes, cal_ylm_real_op (module_base/kernels/math_op.cpp:27-130), cal_sk_op
// (kernels/wf_op.cpp:6-77) and cal_vnl_op (kernels/vnl_op.cpp:8-108).
//
// The functor entry points mirror the reference signatures (device pointers for the per-G and table data,
// host arrays for the per-type counts).  The product path is one fused kernel, k_getvnl: one thread per
// (G, atom) computes k+G, Y_lm by the same Legendre recursion, the 4-point Lagrange interpolation of the
// radial table, the structure factor e^{-i 2 pi (k+G).tau} and the (-i)^l prefactor, and writes that atom's
// nh projector rows in FP64 and FP32 in one pass: no Y_lm, vkb1 or sk arrays in HBM, one write of the
// projectors (the bound: nkb * npwx * 24 bytes).
#include <cmath>
#include <string>

#include "capi_guard.h"
#include "../../include/abacus_b200.h"
#include "capi_handles.h"

namespace b200 {

namespace {

__host__ __device__ inline double fact_d(int n) {
    double f = 1.0;
    for (int i = n; i > 1; --i) f *= i;
    return f;
}
__host__ __device__ inline int semi_fact(int n) {
    int f = 1;
    for (int i = n; i > 2; i -= 2) f *= i;
    return f;
}

// Real Y_lm at one direction, (lmax+1)^2 values in the reference order (per l: m = 0, then cos/sin pairs);
// the recursion of cal_ylm_real_op, with the polar angle from atan exactly as there.
template <typename R>
__device__ __forceinline__ void ylm_point(int lmax, R gx, R gy, R gz, R* ylm) {
    const R pi = R(3.14159265358979323846);
    if (lmax == 0) {
        ylm[0] = R(0.28209479177387814);
        return;
    }
    const R gmod = sqrt(gx * gx + gy * gy + gz * gz);
    const R cost = gmod < R(1.0e-9) ? R(0) : gz / gmod;
    R phi;
    if (gx > R(1.0e-9))
        phi = atan(gy / gx);
    else if (gx < R(-1.0e-9))
        phi = atan(gy / gx) + pi;
    else
        phi = R(1.5707963267948966) * (gy >= R(0) ? R(1) : R(-1));
    R p[kVnlMaxL + 1][kVnlMaxL + 1];  // p[m][l]
    int lm = -1;
#pragma unroll
    for (int l = 0; l <= kVnlMaxL; ++l) {
        if (l > lmax) break;
        const R c = sqrt(R(2 * l + 1) / R(12.566370614359172));
        if (l == 0) {
            p[0][0] = R(1);
        } else if (l == 1) {
            p[0][1] = cost;
            p[1][1] = -sqrt(max(R(0), R(1) - cost * cost));
        } else {
            const int l1 = l - 1, l2 = l - 2, l3 = 2 * l - 1;
#pragma unroll
            for (int m = 0; m <= kVnlMaxL - 2; ++m)
                if (m <= l2) p[m][l] = (cost * R(l3) * p[m][l1] - R(l1 + m) * p[m][l2]) / R(l - m);
            p[l1][l] = cost * R(l3) * p[l1][l1];
            const R x2 = max(R(0), R(1) - cost * cost);
            p[l][l] = R(semi_fact(l3)) * pow(x2, R(l) / R(2));
            if (l % 2 == 1) p[l][l] = -p[l][l];
        }
        ylm[++lm] = c * p[0][l];
#pragma unroll
        for (int m = 1; m <= kVnlMaxL; ++m) {
            if (m > l) break;
            const R same = c * sqrt(R(fact_d(l - m) / fact_d(l + m))) * R(1.4142135623730951);
            R sp, cp;
            sincos(R(m) * phi, &sp, &cp);
            ylm[++lm] = same * p[m][l] * cp;
            ylm[++lm] = same * p[m][l] * sp;
        }
    }
}

// _polynomial_interpolation (vnl_tools.hpp:6-28); iq is clamped so the four taps stay inside the row
template <typename R>
__device__ __forceinline__ R interp4(const R* __restrict__ tab, int it, int ib, int tab_2, int tab_3, R dq, R x) {
    const R pos = x / dq;
    int iq = int(pos);
    if (iq > tab_3 - 4) iq = tab_3 - 4;
    if (iq < 0) iq = 0;
    const R x0 = pos - R(iq);
    const R x1 = R(1) - x0, x2 = R(2) - x0, x3 = R(3) - x0;
    const R* t = tab + (long(it) * tab_2 + ib) * tab_3 + iq;
    return t[0] * x1 * x2 * x3 / R(6) + t[1] * x0 * x2 * x3 / R(2) - t[2] * x1 * x0 * x3 / R(2) +
           t[3] * x1 * x2 * x0 / R(6);
}

// (-i)^n
template <typename T> __device__ __forceinline__ T times_neg_i_pow(T z, int n) {
    switch (n & 3) {
        case 0: return z;
        case 1: return cmake<T>(z.y, -z.x);
        case 2: return cmake<T>(-z.x, -z.y);
        default: return cmake<T>(-z.y, z.x);
    }
}

// ---- functor kernels (reference layouts)
template <typename R>
__global__ void k_ylm_real(int ng, int lmax, const R* __restrict__ g, R* __restrict__ ylm) {
    const int ig = blockIdx.x * blockDim.x + threadIdx.x;
    if (ig >= ng) return;
    R y[(kVnlMaxL + 1) * (kVnlMaxL + 1)];
    ylm_point<R>(lmax, g[3 * ig], g[3 * ig + 1], g[3 * ig + 2], y);
    const int nlm = (lmax + 1) * (lmax + 1);
    for (int lm = 0; lm < nlm; ++lm) ylm[long(lm) * ng + ig] = y[lm];
}

struct SkArgs {
    int ik, nx, ny, nz, rho_nx, rho_ny, rho_nz, npw, npwx, fftny, e1, e2, e3;
};
template <typename R, typename T>
__global__ void k_cal_sk(SkArgs a, R two_pi, const int* __restrict__ igl2isz, const int* __restrict__ is2fftixy,
                         const R* __restrict__ kvec_c, const R* __restrict__ tau, const T* __restrict__ eig1,
                         const T* __restrict__ eig2, const T* __restrict__ eig3, T* __restrict__ sk) {
    const int igl = blockIdx.x * blockDim.x + threadIdx.x;
    const int iat = blockIdx.y;
    if (igl >= a.npw) return;
    R arg = R(0);
    for (int i = 0; i < 3; ++i) arg += kvec_c[a.ik * 3 + i] * tau[iat * 3 + i];
    arg *= two_pi;
    R sp, cp;
    sincos(arg, &sp, &cp);
    const T kph = cmake<T>(cp, -sp);
    const int isz = igl2isz[long(a.ik) * a.npwx + igl];
    int iz = isz % a.nz;
    const int ixy = is2fftixy[isz / a.nz];
    int ix = ixy / a.fftny, iy = ixy % a.fftny;
    if (ix >= a.nx / 2 + 1) ix -= a.nx;
    if (iy >= a.ny / 2 + 1) iy -= a.ny;
    if (iz >= a.nz / 2 + 1) iz -= a.nz;
    ix += a.rho_nx;
    iy += a.rho_ny;
    iz += a.rho_nz;
    sk[long(iat) * a.npw + igl] =
        cmul(cmul(cmul(kph, eig1[long(iat) * a.e1 + ix]), eig2[long(iat) * a.e2 + iy]), eig3[long(iat) * a.e3 + iz]);
}

struct VnlCounts {
    int ntype, npw, npwx, nhm, tab_2, tab_3;
    int na[kVnlMaxTypes], nb[kVnlMaxTypes], nh[kVnlMaxTypes];
};
template <typename R, typename T>
__global__ void k_cal_vnl(VnlCounts c, R dq, R tpiba, const R* __restrict__ gk, const R* __restrict__ ylm,
                          const R* __restrict__ indv, const R* __restrict__ nhtol, const R* __restrict__ nhtolm,
                          const R* __restrict__ tab, const T* __restrict__ sk, T* __restrict__ vkb) {
    const int ig = blockIdx.x * blockDim.x + threadIdx.x;
    if (ig >= c.npw) return;
    const R gx = gk[3 * ig], gy = gk[3 * ig + 1], gz = gk[3 * ig + 2];
    const R gnorm = sqrt(gx * gx + gy * gy + gz * gz) * tpiba;
    int jkb = 0, iat = 0;
    for (int it = 0; it < c.ntype; ++it) {
        for (int ia = 0; ia < c.na[it]; ++ia) {
            const T s = sk[long(iat) * c.npw + ig];
            for (int ih = 0; ih < c.nh[it]; ++ih) {
                const int ib = int(indv[it * c.nhm + ih]);
                const int lm = int(nhtolm[it * c.nhm + ih]);
                const R v = ylm[long(lm) * c.npw + ig] * interp4<R>(tab, it, ib, c.tab_2, c.tab_3, dq, gnorm);
                vkb[long(jkb) * c.npwx + ig] = times_neg_i_pow(cscale(s, v), int(nhtol[it * c.nhm + ih]));
                ++jkb;
            }
            ++iat;
        }
    }
}

// ---- fused getvnl: one thread per (G, atom); entries npw..ld-1 of each row are zeroed
__global__ void __launch_bounds__(256) k_getvnl(VnlParams P, int npw, const double* __restrict__ gk,
                                                const double* __restrict__ tab, const double* __restrict__ tau,
                                                double2* __restrict__ vkb, int npwx, float2* __restrict__ vkbf,
                                                int ldf) {
    const int ig = blockIdx.x * blockDim.x + threadIdx.x;
    const int iat = blockIdx.y;
    const int ncol = npwx > ldf ? npwx : ldf;
    if (ig >= ncol) return;
    int it = 0, a0 = 0, jkb0 = 0;
    while (it < P.ntype - 1 && iat >= a0 + P.na[it]) {
        a0 += P.na[it];
        jkb0 += P.na[it] * P.nh[it];
        ++it;
    }
    const int row0 = jkb0 + (iat - a0) * P.nh[it];
    const int nh = P.nh[it];
    if (ig >= npw) {
        for (int ih = 0; ih < nh; ++ih) {
            if (ig < npwx) vkb[long(row0 + ih) * npwx + ig] = make_double2(0.0, 0.0);
            if (vkbf && ig < ldf) vkbf[long(row0 + ih) * ldf + ig] = make_float2(0.f, 0.f);
        }
        return;
    }
    const double gx = gk[3 * ig], gy = gk[3 * ig + 1], gz = gk[3 * ig + 2];
    double ylm[(kVnlMaxL + 1) * (kVnlMaxL + 1)];
    ylm_point<double>(P.lmax, gx, gy, gz, ylm);
    const double gnorm = sqrt(gx * gx + gy * gy + gz * gz) * P.tpiba;
    const double* t = tau + 3 * iat;
    double sp, cp;
    sincospi(2.0 * (gx * t[0] + gy * t[1] + gz * t[2]), &sp, &cp);
    const double2 s = make_double2(cp, -sp);
    for (int ih = 0; ih < nh; ++ih) {
        const double v = ylm[P.nhtolm[it][ih]] * interp4<double>(tab, it, P.indv[it][ih], P.tab_2, P.tab_3, P.dq, gnorm);
        const double2 z = times_neg_i_pow(cscale(s, v), P.nhtol[it][ih]);
        vkb[long(row0 + ih) * npwx + ig] = z;
        if (vkbf) vkbf[long(row0 + ih) * ldf + ig] = make_float2(float(z.x), float(z.y));
    }
}

}  // namespace

void Hamilt::set_projectors(int ntype, const int* na, const int* nbeta, const int* nh, int nhm, int lmax,
                            const int* indv, const int* nhtol, const int* nhtolm, int tab_2, int tab_3, double dq,
                            const double* tab_h, const double* tau_h) {
    B200_CHECK(ntype >= 1 && ntype <= kVnlMaxTypes, kInvalidArgument, "1..8 atom types supported");
    B200_CHECK(nhm >= 1 && nhm <= kVnlMaxNh, kInvalidArgument, "nhm must be 1..32");
    B200_CHECK(lmax >= 0 && lmax <= kVnlMaxL, kInvalidArgument, "lmax must be 0..4");
    B200_CHECK(tab_3 >= 4 && tab_2 >= 1 && dq > 0.0, kInvalidArgument, "bad radial table shape");
    B200_CHECK(na && nbeta && nh && indv && nhtol && nhtolm && tab_h && tau_h, kInvalidArgument, "NULL argument");
    VnlParams p{};
    p.ntype = ntype;
    p.nhm = nhm;
    p.lmax = lmax;
    p.tab_2 = tab_2;
    p.tab_3 = tab_3;
    p.dq = dq;
    p.tpiba = grid->basis.tpiba;
    int nat = 0, nkb = 0;
    for (int it = 0; it < ntype; ++it) {
        B200_CHECK(na[it] >= 0 && nh[it] >= 0 && nh[it] <= nhm && nbeta[it] >= 0 && nbeta[it] <= tab_2,
                   kInvalidArgument, "bad per-type counts");
        p.na[it] = na[it];
        p.nbeta[it] = nbeta[it];
        p.nh[it] = nh[it];
        for (int ih = 0; ih < nh[it]; ++ih) {
            const int b = indv[it * nhm + ih], l = nhtol[it * nhm + ih], lm = nhtolm[it * nhm + ih];
            B200_CHECK(b >= 0 && b < nbeta[it] && l >= 0 && l <= lmax && lm >= l * l && lm < (l + 1) * (l + 1),
                       kInvalidArgument, "bad indv / nhtol / nhtolm entry");
            p.indv[it][ih] = (unsigned char)b;
            p.nhtol[it][ih] = (unsigned char)l;
            p.nhtolm[it][ih] = (unsigned char)lm;
        }
        nat += na[it];
        nkb += na[it] * nh[it];
    }
    B200_CHECK(nat >= 1, kInvalidArgument, "no atoms");
    p.nkb = nkb;
    // the interpolation reads iq..iq+3 with iq = |k+G|_max / dq: the table must reach past the cut-off
    const double qmax = std::sqrt(grid->basis.gk_ecut) * grid->basis.tpiba;
    B200_CHECK(int(qmax / dq) + 3 < tab_3, kInvalidArgument,
               "radial table too short for the cut-off: need tab_3 > " + std::to_string(int(qmax / dq) + 3));
    vnl.tab.upload(tab_h, size_t(ntype) * tab_2 * tab_3);
    vnl.tau.upload(tau_h, size_t(nat) * 3);
    vnl.p = p;
    vnl.nat = nat;
    vnl.set = true;
}

void Hamilt::build_vkb(int ik, cudaStream_t s) {
    B200_CHECK(vnl.set, kInvalidArgument, "projector tables not set");
    B200_CHECK(ik >= 0 && ik < int(nl.size()), kInvalidArgument, "k-point index out of range");
    const KMap& km = grid->kmaps[ik];
    NonlocalK& k = nl[ik];
    k.nkb = vnl.p.nkb;
    k.npwx = grid->basis.npwk_max;
    k.ldf = k.npwx + (k.npwx & 1);
    k.vkb.resize(size_t(k.nkb) * k.npwx);
    k.vkbf.resize(size_t(k.nkb) * k.ldf);
    const int ncol = k.ldf;
    k_getvnl<<<dim3(ceil_div(ncol, 256), vnl.nat), 256, 0, s>>>(vnl.p, km.npw, km.gkcar.ptr, vnl.tab.ptr, vnl.tau.ptr,
                                                                k.vkb.ptr, k.npwx, k.vkbf.ptr, k.ldf);
    note_launch();
    B200_CUDA(cudaGetLastError());
    fold_projectors(ik, s);
}

}  // namespace b200

namespace {
using b200::guarded;

template <typename R>
void ylm_call(int ng, int lmax, const R* g, R* ylm, cudaStream_t s) {
    B200_CHECK(ng >= 0 && lmax >= 0 && lmax <= b200::kVnlMaxL, b200::kInvalidArgument, "lmax must be 0..4");
    if (ng == 0) return;
    B200_CHECK(g && ylm, b200::kInvalidArgument, "NULL argument");
    b200::k_ylm_real<R><<<b200::ceil_div(ng, 256), 256, 0, s>>>(ng, lmax, g, ylm);
    b200::note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename R, typename T>
void sk_call(int ik, int ntype, int nx, int ny, int nz, int rho_nx, int rho_ny, int rho_nz, int npw, int npwx, int fftny,
             int e1, int e2, int e3, const int* atom_na, const int* igl2isz, const int* is2fftixy, R two_pi,
             const R* kvec_c, const R* tau, const T* eig1, const T* eig2, const T* eig3, T* sk, cudaStream_t s) {
    B200_CHECK(atom_na && ntype >= 0, b200::kInvalidArgument, "NULL atom_na");
    int nat = 0;
    for (int it = 0; it < ntype; ++it) nat += atom_na[it];
    if (npw == 0 || nat == 0) return;
    B200_CHECK(igl2isz && is2fftixy && kvec_c && tau && eig1 && eig2 && eig3 && sk, b200::kInvalidArgument,
               "NULL argument");
    b200::SkArgs a{ik, nx, ny, nz, rho_nx, rho_ny, rho_nz, npw, npwx, fftny, e1, e2, e3};
    b200::k_cal_sk<R, T><<<dim3(b200::ceil_div(npw, 256), nat), 256, 0, s>>>(a, two_pi, igl2isz, is2fftixy, kvec_c, tau,
                                                                           eig1, eig2, eig3, sk);
    b200::note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename R, typename T>
void vnl_call(int ntype, int npw, int npwx, int nhm, int tab_2, int tab_3, const int* na, const int* nb, const int* nh,
              R dq, R tpiba, const R* gk, const R* ylm, const R* indv, const R* nhtol, const R* nhtolm, const R* tab,
              const T* sk, T* vkb, cudaStream_t s) {
    B200_CHECK(ntype >= 0 && ntype <= b200::kVnlMaxTypes, b200::kInvalidArgument, "0..8 atom types supported");
    B200_CHECK(na && nb && nh, b200::kInvalidArgument, "NULL per-type counts");
    B200_CHECK(tab_3 >= 4, b200::kInvalidArgument, "tab_3 must be at least 4");
    b200::VnlCounts c{};
    c.ntype = ntype;
    c.npw = npw;
    c.npwx = npwx;
    c.nhm = nhm;
    c.tab_2 = tab_2;
    c.tab_3 = tab_3;
    for (int it = 0; it < ntype; ++it) {
        c.na[it] = na[it];
        c.nb[it] = nb[it];
        c.nh[it] = nh[it];
    }
    if (npw == 0) return;
    B200_CHECK(gk && ylm && indv && nhtol && nhtolm && tab && sk && vkb, b200::kInvalidArgument, "NULL argument");
    b200::k_cal_vnl<R, T><<<b200::ceil_div(npw, 256), 256, 0, s>>>(c, dq, tpiba, gk, ylm, indv, nhtol, nhtolm, tab, sk,
                                                                  vkb);
    b200::note_launch();
    B200_CUDA(cudaGetLastError());
}
}  // namespace

extern "C" {

int b200_cal_ylm_real_op_f64(int ng, int lmax, const double* g_d, double* ylm_d, void* stream) {
    return guarded([&] { ylm_call<double>(ng, lmax, g_d, ylm_d, (cudaStream_t)stream); });
}
int b200_cal_ylm_real_op_f32(int ng, int lmax, const float* g_d, float* ylm_d, void* stream) {
    return guarded([&] { ylm_call<float>(ng, lmax, g_d, ylm_d, (cudaStream_t)stream); });
}

int b200_cal_sk_op_f64(int ik, int ntype, int nx, int ny, int nz, int rho_nx, int rho_ny, int rho_nz, int npw, int npwx,
                       int fftny, int eigts1_nc, int eigts2_nc, int eigts3_nc, const int* atom_na,
                       const int* igl2isz_d, const int* is2fftixy_d, double two_pi, const double* kvec_c_d,
                       const double* atom_tau_d, const void* eigts1_d, const void* eigts2_d, const void* eigts3_d,
                       void* sk_d, void* stream) {
    return guarded([&] {
        sk_call<double, double2>(ik, ntype, nx, ny, nz, rho_nx, rho_ny, rho_nz, npw, npwx, fftny, eigts1_nc, eigts2_nc,
                                 eigts3_nc, atom_na, igl2isz_d, is2fftixy_d, two_pi, kvec_c_d, atom_tau_d,
                                 (const double2*)eigts1_d, (const double2*)eigts2_d, (const double2*)eigts3_d,
                                 (double2*)sk_d, (cudaStream_t)stream);
    });
}
int b200_cal_sk_op_f32(int ik, int ntype, int nx, int ny, int nz, int rho_nx, int rho_ny, int rho_nz, int npw, int npwx,
                       int fftny, int eigts1_nc, int eigts2_nc, int eigts3_nc, const int* atom_na,
                       const int* igl2isz_d, const int* is2fftixy_d, float two_pi, const float* kvec_c_d,
                       const float* atom_tau_d, const void* eigts1_d, const void* eigts2_d, const void* eigts3_d,
                       void* sk_d, void* stream) {
    return guarded([&] {
        sk_call<float, float2>(ik, ntype, nx, ny, nz, rho_nx, rho_ny, rho_nz, npw, npwx, fftny, eigts1_nc, eigts2_nc,
                               eigts3_nc, atom_na, igl2isz_d, is2fftixy_d, two_pi, kvec_c_d, atom_tau_d,
                               (const float2*)eigts1_d, (const float2*)eigts2_d, (const float2*)eigts3_d, (float2*)sk_d,
                               (cudaStream_t)stream);
    });
}

int b200_cal_vnl_op_f64(int ntype, int npw, int npwx, int nhm, int tab_2, int tab_3, const int* atom_na,
                        const int* atom_nb, const int* atom_nh, double dq, double tpiba, const double* gk_d,
                        const double* ylm_d, const double* indv_d, const double* nhtol_d, const double* nhtolm_d,
                        const double* tab_d, double* vkb1_d, const void* sk_d, void* vkb_d, void* stream) {
    (void)vkb1_d;
    return guarded([&] {
        vnl_call<double, double2>(ntype, npw, npwx, nhm, tab_2, tab_3, atom_na, atom_nb, atom_nh, dq, tpiba, gk_d, ylm_d,
                                  indv_d, nhtol_d, nhtolm_d, tab_d, (const double2*)sk_d, (double2*)vkb_d,
                                  (cudaStream_t)stream);
    });
}
int b200_cal_vnl_op_f32(int ntype, int npw, int npwx, int nhm, int tab_2, int tab_3, const int* atom_na,
                        const int* atom_nb, const int* atom_nh, float dq, float tpiba, const float* gk_d,
                        const float* ylm_d, const float* indv_d, const float* nhtol_d, const float* nhtolm_d,
                        const float* tab_d, float* vkb1_d, const void* sk_d, void* vkb_d, void* stream) {
    (void)vkb1_d;
    return guarded([&] {
        vnl_call<float, float2>(ntype, npw, npwx, nhm, tab_2, tab_3, atom_na, atom_nb, atom_nh, dq, tpiba, gk_d, ylm_d,
                                indv_d, nhtol_d, nhtolm_d, tab_d, (const float2*)sk_d, (float2*)vkb_d,
                                (cudaStream_t)stream);
    });
}

int b200_hamilt_set_projectors(b200_hamilt* h, int ntype, const int* na, const int* nbeta, const int* nh, int nhm,
                               int lmax, const int* indv, const int* nhtol, const int* nhtolm, int tab_2, int tab_3,
                               double dq, const double* tab, const double* tau) {
    return guarded([&] {
        B200_CHECK(h != nullptr, b200::kInvalidArgument, "NULL handle");
        h->h->set_projectors(ntype, na, nbeta, nh, nhm, lmax, indv, nhtol, nhtolm, tab_2, tab_3, dq, tab, tau);
    });
}

int b200_hamilt_build_vkb(b200_hamilt* h, int ik, void* stream) {
    return guarded([&] {
        B200_CHECK(h != nullptr, b200::kInvalidArgument, "NULL handle");
        h->h->build_vkb(ik, (cudaStream_t)stream);
    });
}

int b200_hamilt_copy_vkb(const b200_hamilt* h, int ik, void* vkb_d, void* stream) {
    return guarded([&] {
        B200_CHECK(h != nullptr && vkb_d != nullptr, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(ik >= 0 && ik < int(h->h->nl.size()), b200::kInvalidArgument, "k-point index out of range");
        const b200::NonlocalK& k = h->h->nl[ik];
        if (k.nkb <= 0) return;
        B200_CUDA(cudaMemcpyAsync(vkb_d, k.vkb.ptr, size_t(k.nkb) * k.npwx * sizeof(double2), cudaMemcpyDeviceToDevice,
                                  (cudaStream_t)stream));
    });
}

}  // extern "C"
