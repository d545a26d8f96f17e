// sm_100a kernels for the G-sphere <-> r-box transforms and the fused local H|psi>.
//
// Fused local H|psi> (the hot path, replaces the per-band loop of
// Veff::act + Ekinetic::act in ABACUS, veff_pw.cpp:38-109, ekinetic_pw.cpp:34-50):
//   1. k_zpass_inv : sphere scatter + inverse z FFT of a tile of sticks, written
//                    plane-major into the stick buffer;
//   2. k_plane     : per (band, z) plane: inverse y FFT of the occupied
//                    x-columns, then row by row inverse x FFT, multiply by
//                    V_eff(r), forward x FFT; forward y FFT; back into the
//                    stick buffer (the r box never touches HBM);
//   3. k_zpass_fwd : forward z FFT, gather of the sphere, 1/N scale, the
//                    kinetic term gk2*tpiba2*psi, store (or accumulate) hpsi.
// Drop-in transforms (PW_Basis_K::recip_to_real / real_to_recip,
// pw_transform_k.cpp:336-476) use k_box_zinv / k_box_y / k_box_x / k_box_zfwd
// on the full box in ABACUS's r order.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "pw_grid.h"

namespace b200 {

// ------------------------------------------------------------------ host plans
void FftAxis::build(int n) {
    B200_CHECK(n >= 1, kInvalidArgument, "FFT length must be positive");
    std::vector<int> rad;
    int m = n;
    while (m % 4 == 0) { rad.push_back(4); m /= 4; }
    while (m % 2 == 0) { rad.push_back(2); m /= 2; }
    while (m % 3 == 0) { rad.push_back(3); m /= 3; }
    while (m % 5 == 0) { rad.push_back(5); m /= 5; }
    B200_CHECK(m == 1, kInvalidArgument, "FFT length " + std::to_string(n) + " is not 2,3,5-smooth");
    B200_CHECK(int(rad.size()) <= kMaxPass, kInvalidArgument, "FFT length has too many factors");
    plan = FftPlan1D{};
    plan.n = n;
    plan.npass = int(rad.size());
    std::vector<double2> t64;
    int p = 1;
    for (int j = 0; j < plan.npass; ++j) {
        const int R = rad[j];
        plan.radix[j] = R;
        plan.p[j] = p;
        plan.twoff[j] = int(t64.size());
        const long L = long(p) * R;
        for (int k = 0; k < p; ++k)
            for (int r = 1; r < R; ++r) {
                const long num = (long(r) * k) % L;
                const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)num / (long double)L;
                t64.push_back(make_double2(double(std::cos(ang)), double(std::sin(ang))));
            }
        p *= R;
    }
    if (t64.empty()) t64.push_back(make_double2(1.0, 0.0));
    h_tw64 = t64;
}

void FftAxis::upload() {
    std::vector<float2> t32(h_tw64.size());
    for (size_t i = 0; i < h_tw64.size(); ++i) t32[i] = make_float2(float(h_tw64[i].x), float(h_tw64[i].y));
    tw64.upload(h_tw64.data(), h_tw64.size());
    tw32.upload(t32.data(), t32.size());
    const int n = plan.n;
    std::vector<double2> r64(n);
    std::vector<float2> r32(n);
    for (int j = 0; j < n; ++j) {
        const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / (long double)n;
        r64[j] = make_double2(double(std::cos(ang)), double(std::sin(ang)));
        r32[j] = make_float2(float(std::cos(ang)), float(std::sin(ang)));
    }
    rt64.upload(r64.data(), n);
    rt32.upload(r32.data(), n);
}

void PWGrid::build(const PWBasisK& b) {
    basis = b;
    nx = b.nx;
    ny = b.ny;
    nz = b.nz;
    nst = b.nst;
    on_device = false;
    B200_CHECK(nz < 1024, kInvalidArgument, "nz must be < 1024");
    ax.build(nx);
    ay.build(ny);
    az.build(nz);
    std::vector<int> sx(nst);
    h_sy.assign(nst, 0);
    h_sixy.assign(nst, 0);
    for (int s = 0; s < nst; ++s) {
        h_sixy[s] = b.is2fftixy[s];
        sx[s] = b.is2fftixy[s] / ny;
        h_sy[s] = b.is2fftixy[s] % ny;
    }
    h_xpos = sx;
    std::sort(h_xpos.begin(), h_xpos.end());
    h_xpos.erase(std::unique(h_xpos.begin(), h_xpos.end()), h_xpos.end());
    nxc = int(h_xpos.size());
    h_xc.assign(nst, 0);
    for (int s = 0; s < nst; ++s) h_xc[s] = int(std::lower_bound(h_xpos.begin(), h_xpos.end(), sx[s]) - h_xpos.begin());
    h_smap.assign(size_t(nxc) * ny, -1);
    for (int s = 0; s < nst; ++s) h_smap[size_t(h_xc[s]) * ny + h_sy[s]] = s;
    kmaps.clear();
    kmaps.resize(b.nks);
    const size_t L = size_t(b.npwk_max);
    for (int ik = 0; ik < b.nks; ++ik) {
        KMap& km = kmaps[ik];
        const int npw = b.npwk[ik];
        km.npw = npw;
        std::vector<int> stick(npw), zz(npw), order(npw);
        for (int g = 0; g < npw; ++g) {
            const int isz = b.igl2isz_k[ik * L + g];
            stick[g] = isz / nz;
            zz[g] = isz % nz;
        }
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return stick[a] < stick[c]; });
        km.h_gofs.assign(nst + 1, 0);
        km.h_gpk.assign(npw, 0);
        km.h_glist.assign(npw, 0);
        for (int g = 0; g < npw; ++g) km.h_gofs[stick[g] + 1]++;
        for (int s = 0; s < nst; ++s) km.h_gofs[s + 1] += km.h_gofs[s];
        for (int j = 0; j < npw; ++j) {
            const int g = order[j];
            km.h_gpk[j] = (stick[g] << 10) | zz[g];
            km.h_glist[j] = g;
        }
        km.h_precond.assign(npw, 0.0);
        for (int g = 0; g < npw; ++g) {
            // HSolverPW::update_precondition, precondition_type 2 (hsolver_pw.cpp:567-584)
            const double g2 = b.gk2[ik * L + g] * b.tpiba2;
            km.h_precond[g] = 1.0 + g2 + std::sqrt(1.0 + (g2 - 1.0) * (g2 - 1.0));
        }
    }
}

void PWGrid::ensure_device() {
    if (on_device) return;
    ax.upload();
    ay.upload();
    az.upload();
    st_xc.upload(h_xc.data(), nst);
    st_y.upload(h_sy.data(), nst);
    st_ixy.upload(h_sixy.data(), nst);
    xpos.upload(h_xpos.data(), nxc);
    smap.upload(h_smap.data(), h_smap.size());
    const size_t L = size_t(basis.npwk_max);
    for (int ik = 0; ik < basis.nks; ++ik) {
        KMap& km = kmaps[ik];
        const int npw = km.npw;
        km.gofs.upload(km.h_gofs.data(), nst + 1);
        km.gpk.upload(km.h_gpk.data(), npw);
        km.glist.upload(km.h_glist.data(), npw);
        km.ig2ixyz.upload(&basis.ig2ixyz_k[ik * L], npw);
        km.gk2.upload(&basis.gk2[ik * L], npw);
        std::vector<float> gf(npw);
        for (int g = 0; g < npw; ++g) gf[g] = float(basis.gk2[ik * L + g]);
        km.gk2f.upload(gf.data(), npw);
        km.precond.upload(km.h_precond.data(), npw);
        std::vector<double> gk(size_t(npw) * 3);
        for (int g = 0; g < npw; ++g)
            for (int j = 0; j < 3; ++j) gk[size_t(g) * 3 + j] = basis.gcar[(ik * L + g) * 3 + j] + basis.kvec_c[ik * 3 + j];
        km.gkcar.upload(gk.data(), size_t(npw) * 3);
    }
    B200_CUDA(cudaDeviceSynchronize());
    on_device = true;
}

size_t zpass_smem(const PWGrid& g, size_t elem) { return size_t(2) * kStickTile * odd_ld(g.nz) * elem; }
size_t plane_smem(const PWGrid& g, size_t elem) {
    return (size_t(g.nxc) * odd_ld(g.ny) + size_t(kPlaneCols) * odd_ld(g.ny) + size_t(2) * kPlaneRows * odd_ld(g.nx)) *
           elem;
}

// ------------------------------------------------------------------ kernels
template <typename T> __device__ __forceinline__ T czero() { return cmake<T>(0, 0); }

// (1) sphere -> sticks (inverse z FFT), one CTA per (stick tile, band)
template <typename T>
__global__ void __launch_bounds__(256) k_zpass_inv(StickMapView sm, FftPlan1D pz, const T* __restrict__ twz,
                                                   const T* __restrict__ psi, int ld, T* __restrict__ sb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);
    const int ldz = sm.nz | 1;
    T* B = A + kStickTile * ldz;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int s0 = blockIdx.x * kStickTile;
    const int ns = min(kStickTile, sm.nst - s0);
    const int band = blockIdx.y;
    for (int i = tid; i < kStickTile * ldz; i += nthr) A[i] = czero<T>();
    __syncthreads();
    const T* p = psi + size_t(band) * ld;
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    for (int j = j0 + tid; j < j1; j += nthr) {
        const int pk = sm.gpk[j];
        A[((pk >> 10) - s0) * ldz + (pk & 1023)] = p[sm.glist[j]];
    }
    __syncthreads();
    fft_batch<T, +1>(A, B, ns, 1, ldz, pz, twz, tid, nthr);
    T* out = sb + size_t(band) * sm.nz * sm.nst;
    for (int i = tid; i < ns * sm.nz; i += nthr) {
        const int z = i / ns;
        const int sl = i - z * ns;
        out[size_t(z) * sm.nst + s0 + sl] = A[sl * ldz + z];
    }
}

// (2) plane pass: inverse y, inverse x, V_eff, forward x, forward y. One CTA per (band, z).
template <typename T, typename R>
__global__ void __launch_bounds__(512) k_plane(PlaneMapView pm, int nx, int ny, int nz, FftPlan1D px, FftPlan1D py,
                                               const T* __restrict__ twx, const T* __restrict__ twy,
                                               const R* __restrict__ veff_zyx, T* __restrict__ sb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ldy = ny | 1, ldx = nx | 1;
    T* A = reinterpret_cast<T*>(smem_raw);        // nxc columns of length ny
    T* C = A + pm.nxc * ldy;                      // y-FFT scratch, kPlaneCols columns
    T* R1 = C + kPlaneCols * ldy;                 // kPlaneRows rows of length nx
    T* R2 = R1 + kPlaneRows * ldx;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int band = blockIdx.x;
    const int z = blockIdx.y;
    for (int i = tid; i < pm.nxc * ldy; i += nthr) A[i] = czero<T>();
    __syncthreads();
    T* plane = sb + (size_t(band) * nz + z) * pm.nst;
    for (int s = tid; s < pm.nst; s += nthr) A[pm.xc[s] * ldy + pm.sy[s]] = plane[s];
    __syncthreads();
    for (int c = 0; c < pm.nxc; c += kPlaneCols)
        fft_batch<T, +1>(A + c * ldy, C, min(kPlaneCols, pm.nxc - c), 1, ldy, py, twy, tid, nthr);
    const R* vz = veff_zyx + size_t(z) * ny * nx;
    for (int y0 = 0; y0 < ny; y0 += kPlaneRows) {
        const int nr = min(kPlaneRows, ny - y0);
        for (int i = tid; i < nr * ldx; i += nthr) R1[i] = czero<T>();
        __syncthreads();
        for (int e = tid; e < nr * pm.nxc; e += nthr) {
            const int r = e / pm.nxc;
            const int c = e - r * pm.nxc;
            R1[r * ldx + pm.xpos[c]] = A[c * ldy + y0 + r];
        }
        __syncthreads();
        fft_batch<T, +1>(R1, R2, nr, 1, ldx, px, twx, tid, nthr);
        for (int e = tid; e < nr * nx; e += nthr) {
            const int r = e / nx;
            const int x = e - r * nx;
            R1[r * ldx + x] = cscale(R1[r * ldx + x], vz[(y0 + r) * nx + x]);
        }
        __syncthreads();
        fft_batch<T, -1>(R1, R2, nr, 1, ldx, px, twx, tid, nthr);
        for (int e = tid; e < nr * pm.nxc; e += nthr) {
            const int r = e / pm.nxc;
            const int c = e - r * pm.nxc;
            A[c * ldy + y0 + r] = R1[r * ldx + pm.xpos[c]];
        }
        __syncthreads();
    }
    for (int c = 0; c < pm.nxc; c += kPlaneCols)
        fft_batch<T, -1>(A + c * ldy, C, min(kPlaneCols, pm.nxc - c), 1, ldy, py, twy, tid, nthr);
    for (int s = tid; s < pm.nst; s += nthr) plane[s] = A[pm.xc[s] * ldy + pm.sy[s]];
}

// ---- non-collinear (npol = 2) local pass: the plane pass split at the real-space product ----
// (2a) inverse y and x transforms of spinor column blockIdx.x at plane z = blockIdx.y; the real-space plane
// goes to r[col][z][y][x] (rows of nx)
template <typename T>
__global__ void __launch_bounds__(512) k_plane_inv_r(PlaneMapView pm, int nx, int ny, int nz, FftPlan1D px, FftPlan1D py,
                                                     const T* __restrict__ twx, const T* __restrict__ twy,
                                                     const T* __restrict__ sb, T* __restrict__ r) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ldy = ny | 1, ldx = nx | 1;
    T* A = reinterpret_cast<T*>(smem_raw);
    T* C = A + pm.nxc * ldy;
    T* R1 = C + kPlaneCols * ldy;
    T* R2 = R1 + kPlaneRows * ldx;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int col = blockIdx.x, z = blockIdx.y;
    for (int i = tid; i < pm.nxc * ldy; i += nthr) A[i] = czero<T>();
    __syncthreads();
    const T* plane = sb + (size_t(col) * nz + z) * pm.nst;
    for (int st = tid; st < pm.nst; st += nthr) A[pm.xc[st] * ldy + pm.sy[st]] = plane[st];
    __syncthreads();
    for (int c = 0; c < pm.nxc; c += kPlaneCols)
        fft_batch<T, +1>(A + c * ldy, C, min(kPlaneCols, pm.nxc - c), 1, ldy, py, twy, tid, nthr);
    T* out = r + (size_t(col) * nz + z) * size_t(ny) * nx;
    for (int y0 = 0; y0 < ny; y0 += kPlaneRows) {
        const int nr = min(kPlaneRows, ny - y0);
        for (int i = tid; i < nr * ldx; i += nthr) R1[i] = czero<T>();
        __syncthreads();
        for (int e = tid; e < nr * pm.nxc; e += nthr) {
            const int rr = e / pm.nxc;
            const int c = e - rr * pm.nxc;
            R1[rr * ldx + pm.xpos[c]] = A[c * ldy + y0 + rr];
        }
        __syncthreads();
        fft_batch<T, +1>(R1, R2, nr, 1, ldx, px, twx, tid, nthr);
        for (int e = tid; e < nr * nx; e += nthr) {
            const int rr = e / nx;
            const int x = e - rr * nx;
            out[size_t(y0 + rr) * nx + x] = R1[rr * ldx + x];
        }
        __syncthreads();
    }
}

// (2b) the 2x2 spin potential of veff_pw_op's npol = 2 form (veff_op.cpp:20-37) on spinor column
// blockIdx.x (component c = column & 1, partner column ^ 1) at plane z = blockIdx.y:
//   up' = up (V0 + V3) + dn (V1 - i V2),   dn' = dn (V0 - V3) + up (V1 + i V2),
// then the forward x and y transforms back into the column's sticks.  v4: the four components, (z, y, x).
template <typename T, typename R>
__global__ void __launch_bounds__(512) k_plane_fwd_nc(PlaneMapView pm, int nx, int ny, int nz, FftPlan1D px,
                                                      FftPlan1D py, const T* __restrict__ twx,
                                                      const T* __restrict__ twy, const R* __restrict__ v4,
                                                      const T* __restrict__ r, T* __restrict__ sb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ldy = ny | 1, ldx = nx | 1;
    T* A = reinterpret_cast<T*>(smem_raw);
    T* C = A + pm.nxc * ldy;
    T* R1 = C + kPlaneCols * ldy;
    T* R2 = R1 + kPlaneRows * ldx;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int col = blockIdx.x, z = blockIdx.y;
    const bool up = (col & 1) == 0;
    const size_t N = size_t(nx) * ny * nz, P = size_t(ny) * nx;
    const T* own = r + (size_t(col) * nz + z) * P;
    const T* oth = r + (size_t(col ^ 1) * nz + z) * P;
    const R* v0 = v4 + size_t(z) * P;
    for (int y0 = 0; y0 < ny; y0 += kPlaneRows) {
        const int nr = min(kPlaneRows, ny - y0);
        for (int e = tid; e < nr * nx; e += nthr) {
            const int rr = e / nx;
            const int x = e - rr * nx;
            const size_t i = size_t(y0 + rr) * nx + x;
            const T a = own[i], b = oth[i];
            const R va = v0[i], vb = v0[i + N], vc = v0[i + 2 * N], vd = v0[i + 3 * N];
            // own component: (V0 +- V3) a + (V1 -+ i V2) b
            const R d = up ? va + vd : va - vd;
            const R sg = up ? R(-1) : R(1);
            T o;
            o.x = d * a.x + vb * b.x - sg * vc * b.y;
            o.y = d * a.y + vb * b.y + sg * vc * b.x;
            R1[rr * ldx + x] = o;
        }
        __syncthreads();
        fft_batch<T, -1>(R1, R2, nr, 1, ldx, px, twx, tid, nthr);
        for (int e = tid; e < nr * pm.nxc; e += nthr) {
            const int rr = e / pm.nxc;
            const int c = e - rr * pm.nxc;
            A[c * ldy + y0 + rr] = R1[rr * ldx + pm.xpos[c]];
        }
        __syncthreads();
    }
    for (int c = 0; c < pm.nxc; c += kPlaneCols)
        fft_batch<T, -1>(A + c * ldy, C, min(kPlaneCols, pm.nxc - c), 1, ldy, py, twy, tid, nthr);
    T* plane = sb + (size_t(col) * nz + z) * pm.nst;
    for (int st = tid; st < pm.nst; st += nthr) plane[st] = A[pm.xc[st] * ldy + pm.sy[st]];
}

// (3) sticks -> sphere (forward z FFT), + kinetic term, store/accumulate hpsi
template <typename T, typename R>
__global__ void __launch_bounds__(256) k_zpass_fwd(StickMapView sm, FftPlan1D pz, const T* __restrict__ twz,
                                                   const T* __restrict__ sb, const T* __restrict__ psi,
                                                   T* __restrict__ hpsi, int ld, int npw, const R* __restrict__ gk2,
                                                   R tpiba2, R invn, int accumulate) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);
    const int ldz = sm.nz | 1;
    T* B = A + kStickTile * ldz;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int s0 = blockIdx.x * kStickTile;
    const int ns = min(kStickTile, sm.nst - s0);
    const int band = blockIdx.y;
    const T* in = sb + size_t(band) * sm.nz * sm.nst;
    for (int i = tid; i < ns * sm.nz; i += nthr) {
        const int z = i / ns;
        const int sl = i - z * ns;
        A[sl * ldz + z] = in[size_t(z) * sm.nst + s0 + sl];
    }
    __syncthreads();
    fft_batch<T, -1>(A, B, ns, 1, ldz, pz, twz, tid, nthr);
    const T* p = psi + size_t(band) * ld;
    T* h = hpsi + size_t(band) * ld;
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    for (int j = j0 + tid; j < j1; j += nthr) {
        const int pk = sm.gpk[j];
        const int g = sm.glist[j];
        T v = cscale(A[((pk >> 10) - s0) * ldz + (pk & 1023)], invn);
        v = cadd(v, cscale(p[g], gk2[g] * tpiba2));
        if (accumulate) v = cadd(v, h[g]);
        h[g] = v;
    }
    if (!accumulate && blockIdx.x == 0)
        for (int g = npw + tid; g < ld; g += nthr) h[g] = czero<T>();
}

// ---- drop-in box transforms ----
// sphere -> box columns (inverse z FFT), box pre-zeroed
template <typename T>
__global__ void __launch_bounds__(256) k_box_zinv(StickMapView sm, FftPlan1D pz, const T* __restrict__ twz,
                                                  const int* __restrict__ st_ixy, const T* __restrict__ in,
                                                  T* __restrict__ box) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);
    const int ldz = sm.nz | 1;
    T* B = A + kStickTile * ldz;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int s0 = blockIdx.x * kStickTile;
    const int ns = min(kStickTile, sm.nst - s0);
    for (int i = tid; i < kStickTile * ldz; i += nthr) A[i] = czero<T>();
    __syncthreads();
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    for (int j = j0 + tid; j < j1; j += nthr) {
        const int pk = sm.gpk[j];
        A[((pk >> 10) - s0) * ldz + (pk & 1023)] = in[sm.glist[j]];
    }
    __syncthreads();
    fft_batch<T, +1>(A, B, ns, 1, ldz, pz, twz, tid, nthr);
    for (int i = tid; i < ns * sm.nz; i += nthr) {
        const int sl = i / sm.nz;
        const int z = i - sl * sm.nz;
        box[size_t(st_ixy[s0 + sl]) * sm.nz + z] = A[sl * ldz + z];
    }
}

// y FFT of the box for the x values in xlist (in place); CTA = (x, z tile)
template <typename T, int DIR>
__global__ void __launch_bounds__(256) k_box_y(FftPlan1D py, const T* __restrict__ twy, const int* __restrict__ xlist,
                                               int ny, int nz, T* __restrict__ box) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ldy = ny | 1;
    T* A = reinterpret_cast<T*>(smem_raw);
    T* B = A + kBoxTile * ldy;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int x = xlist ? xlist[blockIdx.x] : blockIdx.x;
    const int z0 = blockIdx.y * kBoxTile;
    const int nzt = min(kBoxTile, nz - z0);
    T* base = box + size_t(x) * ny * nz + z0;
    for (int i = tid; i < ny * nzt; i += nthr) {
        const int y = i / nzt;
        const int zz = i - y * nzt;
        A[zz * ldy + y] = base[size_t(y) * nz + zz];
    }
    __syncthreads();
    fft_batch<T, DIR>(A, B, nzt, 1, ldy, py, twy, tid, nthr);
    for (int i = tid; i < ny * nzt; i += nthr) {
        const int y = i / nzt;
        const int zz = i - y * nzt;
        base[size_t(y) * nz + zz] = A[zz * ldy + y];
    }
}

// x FFT of the box; mode 0: dst = v, mode 1: dst += factor * v. CTA = (y, z tile)
template <typename T, typename R, int DIR>
__global__ void __launch_bounds__(256) k_box_x(FftPlan1D px, const T* __restrict__ twx, int nx, int ny, int nz,
                                               const T* src, T* dst, int mode, R factor) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ldx = nx | 1;
    T* A = reinterpret_cast<T*>(smem_raw);
    T* B = A + kBoxTile * ldx;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int y = blockIdx.x;
    const int z0 = blockIdx.y * kBoxTile;
    const int nzt = min(kBoxTile, nz - z0);
    const size_t off = size_t(y) * nz + z0;
    const size_t xs = size_t(ny) * nz;
    for (int i = tid; i < nx * nzt; i += nthr) {
        const int x = i / nzt;
        const int zz = i - x * nzt;
        A[zz * ldx + x] = src[x * xs + off + zz];
    }
    __syncthreads();
    fft_batch<T, DIR>(A, B, nzt, 1, ldx, px, twx, tid, nthr);
    for (int i = tid; i < nx * nzt; i += nthr) {
        const int x = i / nzt;
        const int zz = i - x * nzt;
        const T v = A[zz * ldx + x];
        T* d = dst + x * xs + off + zz;
        *d = mode ? cadd(*d, cscale(v, factor)) : v;
    }
}

// box columns -> sphere (forward z FFT), out (+)= scale * v
template <typename T, typename R>
__global__ void __launch_bounds__(256) k_box_zfwd(StickMapView sm, FftPlan1D pz, const T* __restrict__ twz,
                                                  const int* __restrict__ st_ixy, const T* __restrict__ box,
                                                  T* __restrict__ out, int add, R scale) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);
    const int ldz = sm.nz | 1;
    T* B = A + kStickTile * ldz;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int s0 = blockIdx.x * kStickTile;
    const int ns = min(kStickTile, sm.nst - s0);
    for (int i = tid; i < ns * sm.nz; i += nthr) {
        const int sl = i / sm.nz;
        const int z = i - sl * sm.nz;
        A[sl * ldz + z] = box[size_t(st_ixy[s0 + sl]) * sm.nz + z];
    }
    __syncthreads();
    fft_batch<T, -1>(A, B, ns, 1, ldz, pz, twz, tid, nthr);
    const int j0 = sm.gofs[s0], j1 = sm.gofs[s0 + ns];
    for (int j = j0 + tid; j < j1; j += nthr) {
        const int pk = sm.gpk[j];
        const int g = sm.glist[j];
        const T v = cscale(A[((pk >> 10) - s0) * ldz + (pk & 1023)], scale);
        out[g] = add ? cadd(out[g], v) : v;
    }
}

template <typename R>
__global__ void k_veff_zyx(int nx, int ny, int nz, const double* __restrict__ veff, R* __restrict__ out) {
    const long N = long(nx) * ny * nz;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < N; i += long(gridDim.x) * blockDim.x) {
        const int x = int(i % nx);
        const long t = i / nx;
        const int y = int(t % ny);
        const int z = int(t / ny);
        out[i] = R(veff[(long(x) * ny + y) * nz + z]);
    }
}

// ------------------------------------------------------------------ launchers
template <typename T> const T* tw_of(const FftAxis& a);
template <> const double2* tw_of<double2>(const FftAxis& a) { return a.tw64.ptr; }
template <> const float2* tw_of<float2>(const FftAxis& a) { return a.tw32.ptr; }

template <typename K> static void set_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) B200_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
}

template <typename T, typename R>
void launch_hpsi_local(const PWGrid& g, int ik, const R* veff_zyx, const R* veff_perm, int nb, int ld, const T* psi,
                       T* hpsi, T* stickbuf, double tpiba2, int accumulate, cudaStream_t s) {
    if (nb <= 0) return;
    B200_CHECK(nb <= 65535, kInvalidArgument, "too many bands in one launch");
    // compile-time warp transforms for the standard grid sizes; generic Stockham kernels otherwise
    if (launch_hpsi_local_fast<T, R>(g, ik, veff_zyx, veff_perm, nb, ld, psi, hpsi, stickbuf, tpiba2, accumulate, s))
        return;
    const size_t zs = zpass_smem(g, sizeof(T));
    const size_t ps = plane_smem(g, sizeof(T));
    B200_CHECK(ps <= 227 * 1024, kCapacityError, "plane pass does not fit in shared memory for this grid");
    const StickMapView sm = g.stick_view(ik);
    const dim3 gz(ceil_div(g.nst, kStickTile), nb);
    set_smem(k_zpass_inv<T>, zs);
    k_zpass_inv<T><<<gz, 256, zs, s>>>(sm, g.az.plan, tw_of<T>(g.az), psi, ld, stickbuf);
    note_launch();
    B200_CUDA(cudaGetLastError());
    set_smem(k_plane<T, R>, ps);
    k_plane<T, R><<<dim3(nb, g.nz), 512, ps, s>>>(g.plane_view(), g.nx, g.ny, g.nz, g.ax.plan, g.ay.plan, tw_of<T>(g.ax),
                                                  tw_of<T>(g.ay), veff_zyx, stickbuf);
    note_launch();
    B200_CUDA(cudaGetLastError());
    const KMap& km = g.kmaps[ik];
    const R* gk2 = std::is_same<R, double>::value ? (const R*)km.gk2.ptr : (const R*)km.gk2f.ptr;
    set_smem(k_zpass_fwd<T, R>, zs);
    k_zpass_fwd<T, R><<<gz, 256, zs, s>>>(sm, g.az.plan, tw_of<T>(g.az), stickbuf, psi, hpsi, ld, km.npw, gk2, R(tpiba2),
                                          R(1.0 / double(g.nxyz())), accumulate);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T, typename R>
void launch_hpsi_local_nc(const PWGrid& g, int ik, const R* veff4_zyx, int ncols, int ld, const T* psi, T* hpsi,
                          T* stickbuf, T* rbuf, double tpiba2, cudaStream_t s) {
    if (ncols <= 0) return;
    B200_CHECK(ncols <= 65535 && ncols % 2 == 0, kInvalidArgument, "npol = 2: an even number of spinor columns, at most 65535");
    const size_t zs = zpass_smem(g, sizeof(T));
    const size_t ps = plane_smem(g, sizeof(T));
    B200_CHECK(ps <= 227 * 1024, kCapacityError, "plane pass does not fit in shared memory for this grid");
    const StickMapView sm = g.stick_view(ik);
    const dim3 gz(ceil_div(g.nst, kStickTile), ncols);
    set_smem(k_zpass_inv<T>, zs);
    k_zpass_inv<T><<<gz, 256, zs, s>>>(sm, g.az.plan, tw_of<T>(g.az), psi, ld, stickbuf);
    note_launch();
    B200_CUDA(cudaGetLastError());
    set_smem(k_plane_inv_r<T>, ps);
    k_plane_inv_r<T><<<dim3(ncols, g.nz), 512, ps, s>>>(g.plane_view(), g.nx, g.ny, g.nz, g.ax.plan, g.ay.plan,
                                                       tw_of<T>(g.ax), tw_of<T>(g.ay), stickbuf, rbuf);
    note_launch();
    B200_CUDA(cudaGetLastError());
    set_smem(k_plane_fwd_nc<T, R>, ps);
    k_plane_fwd_nc<T, R><<<dim3(ncols, g.nz), 512, ps, s>>>(g.plane_view(), g.nx, g.ny, g.nz, g.ax.plan, g.ay.plan,
                                                           tw_of<T>(g.ax), tw_of<T>(g.ay), veff4_zyx, rbuf, stickbuf);
    note_launch();
    B200_CUDA(cudaGetLastError());
    const KMap& km = g.kmaps[ik];
    const R* gk2 = std::is_same<R, double>::value ? (const R*)km.gk2.ptr : (const R*)km.gk2f.ptr;
    set_smem(k_zpass_fwd<T, R>, zs);
    k_zpass_fwd<T, R><<<gz, 256, zs, s>>>(sm, g.az.plan, tw_of<T>(g.az), stickbuf, psi, hpsi, ld, km.npw, gk2, R(tpiba2),
                                          R(1.0 / double(g.nxyz())), 0);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T>
void launch_recip_to_real(const PWGrid& g, int ik, const T* in, T* out, T* aux, int add, double factor, cudaStream_t s) {
    using R = typename RealOf<T>::type;
    const size_t N = size_t(g.nxyz());
    B200_CUDA(cudaMemsetAsync(aux, 0, N * sizeof(T), s));
    const size_t zs = zpass_smem(g, sizeof(T));
    set_smem(k_box_zinv<T>, zs);
    k_box_zinv<T><<<ceil_div(g.nst, kStickTile), 256, zs, s>>>(g.stick_view(ik), g.az.plan, tw_of<T>(g.az), g.st_ixy.ptr,
                                                               in, aux);
    note_launch();
    B200_CUDA(cudaGetLastError());
    const size_t ys = size_t(2) * kBoxTile * odd_ld(g.ny) * sizeof(T);
    set_smem(k_box_y<T, +1>, ys);
    k_box_y<T, +1><<<dim3(g.nxc, ceil_div(g.nz, kBoxTile)), 256, ys, s>>>(g.ay.plan, tw_of<T>(g.ay), g.xpos.ptr, g.ny,
                                                                          g.nz, aux);
    note_launch();
    B200_CUDA(cudaGetLastError());
    const size_t xsm = size_t(2) * kBoxTile * odd_ld(g.nx) * sizeof(T);
    set_smem(k_box_x<T, R, +1>, xsm);
    k_box_x<T, R, +1><<<dim3(g.ny, ceil_div(g.nz, kBoxTile)), 256, xsm, s>>>(g.ax.plan, tw_of<T>(g.ax), g.nx, g.ny, g.nz,
                                                                             aux, out, add, R(factor));
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename T>
void launch_real_to_recip(const PWGrid& g, int ik, const T* in, T* out, T* aux, int add, double factor, cudaStream_t s) {
    using R = typename RealOf<T>::type;
    const size_t xsm = size_t(2) * kBoxTile * odd_ld(g.nx) * sizeof(T);
    set_smem(k_box_x<T, R, -1>, xsm);
    k_box_x<T, R, -1><<<dim3(g.ny, ceil_div(g.nz, kBoxTile)), 256, xsm, s>>>(g.ax.plan, tw_of<T>(g.ax), g.nx, g.ny, g.nz,
                                                                             in, aux, 0, R(1));
    note_launch();
    B200_CUDA(cudaGetLastError());
    const size_t ys = size_t(2) * kBoxTile * odd_ld(g.ny) * sizeof(T);
    set_smem(k_box_y<T, -1>, ys);
    k_box_y<T, -1><<<dim3(g.nxc, ceil_div(g.nz, kBoxTile)), 256, ys, s>>>(g.ay.plan, tw_of<T>(g.ay), g.xpos.ptr, g.ny,
                                                                          g.nz, aux);
    note_launch();
    B200_CUDA(cudaGetLastError());
    const size_t zs = zpass_smem(g, sizeof(T));
    set_smem(k_box_zfwd<T, R>, zs);
    // set_real_to_recip_output_op: out (+)= factor / nxyz * box (pw_op.cpp:46-66)
    const double scale = (add ? factor : 1.0) / double(g.nxyz());
    k_box_zfwd<T, R><<<ceil_div(g.nst, kStickTile), 256, zs, s>>>(g.stick_view(ik), g.az.plan, tw_of<T>(g.az),
                                                                  g.st_ixy.ptr, aux, out, add, R(scale));
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template <typename R>
void launch_transpose_veff(const PWGrid& g, const double* veff, R* out, cudaStream_t s) {
    k_veff_zyx<R><<<1184, 256, 0, s>>>(g.nx, g.ny, g.nz, veff, out);
    note_launch();
    B200_CUDA(cudaGetLastError());
}

template void launch_hpsi_local<double2, double>(const PWGrid&, int, const double*, const double*, int, int,
                                                 const double2*, double2*,
                                                 double2*, double, int, cudaStream_t);
template void launch_hpsi_local<float2, float>(const PWGrid&, int, const float*, const float*, int, int, const float2*,
                                               float2*, float2*,
                                               double, int, cudaStream_t);
template void launch_hpsi_local_nc<double2, double>(const PWGrid&, int, const double*, int, int, const double2*,
                                                    double2*, double2*, double2*, double, cudaStream_t);
template void launch_hpsi_local_nc<float2, float>(const PWGrid&, int, const float*, int, int, const float2*, float2*,
                                                  float2*, float2*, double, cudaStream_t);
template void launch_recip_to_real<double2>(const PWGrid&, int, const double2*, double2*, double2*, int, double, cudaStream_t);
template void launch_recip_to_real<float2>(const PWGrid&, int, const float2*, float2*, float2*, int, double, cudaStream_t);
template void launch_real_to_recip<double2>(const PWGrid&, int, const double2*, double2*, double2*, int, double, cudaStream_t);
template void launch_real_to_recip<float2>(const PWGrid&, int, const float2*, float2*, float2*, int, double, cudaStream_t);
template void launch_transpose_veff<double>(const PWGrid&, const double*, double*, cudaStream_t);
template void launch_transpose_veff<float>(const PWGrid&, const double*, float*, cudaStream_t);

}  // namespace b200
