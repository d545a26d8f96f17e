// Device-resident plane-wave grid: FFT plans, stick maps and per-k sphere maps.
//
// Layouts in HBM (one pool, one GPU):
//  * psi / hpsi: band b at psi + b*ld, G in the order of the basis (ABACUS's
//    igl2isz_k order: sticks by ixy = x*ny + y, z ascending from the bottom).
//  * stick buffer (fused H|psi>): per band nz planes of nst sticks,
//    element (band, z, s) at band*nz*nst + z*nst + s.  A z-plane is contiguous,
//    so the plane pass reads and writes whole planes with coalesced accesses.
//  * r box (drop-in transforms): ABACUS's order r = (ix*ny + iy)*nz + iz.
//  * V_eff for the fused path: transposed once to (z, y, x) so a plane row is
//    contiguous.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "common.h"
#include "fft_core.cuh"
#include "pw_basis.h"

namespace b200 {

// One FFT axis: plan plus twiddles in both precisions.
struct FftAxis {
    FftPlan1D plan{};
    std::vector<double2> h_tw64;
    DeviceArray<double2> tw64;
    DeviceArray<float2> tw32;
    DeviceArray<double2> rt64;  // the n roots W_n^j = exp(-2 pi i j / n), j < n (register/shuffle transforms)
    DeviceArray<float2> rt32;
    void build(int n);  // host plan + twiddles
    void upload();
};

// Sphere -> stick maps for one k-point.
struct KMap {
    int npw = 0;
    std::vector<int> h_gofs, h_gpk, h_glist;
    std::vector<double> h_precond;
    DeviceArray<int> gofs;   // nst+1 offsets of each stick's entries in the sorted list
    DeviceArray<int> gpk;    // packed (stick << 10) | z per sorted entry
    DeviceArray<int> glist;  // G index (position in psi) per sorted entry
    DeviceArray<int> ig2ixyz;
    DeviceArray<double> gk2;
    DeviceArray<float> gk2f;
    DeviceArray<double> precond;  // Davidson preconditioner 1 + g2 + sqrt(1 + (g2-1)^2)
    DeviceArray<double> gkcar;    // k+G cartesian (npw x 3, units of tpiba): PW_Basis_K::getgpluskcar
};

// Index maps handed to kernels by value.
struct StickMapView {
    int nst, nz;
    const int* gofs;
    const int* gpk;
    const int* glist;
};
struct PlaneMapView {
    int nst, nxc;
    const int* xc;    // per stick: compact x-column index
    const int* sy;    // per stick: y
    const int* xpos;  // per compact column: x
    const int* smap;  // per compact column c and y < ny: the stick at (xpos[c], y), or -1 (nxc x ny)
};

struct PWGrid {
    PWBasisK basis;
    int nx = 0, ny = 0, nz = 0, nst = 0, nxc = 0;
    FftAxis ax, ay, az;
    DeviceArray<int> st_xc, st_y, xpos, st_ixy, smap;
    std::vector<int> h_xpos, h_xc, h_sy, h_sixy, h_smap;
    std::vector<KMap> kmaps;
    bool on_device = false;
    // plane pass of the register transforms, per precision (0: default shape; see plane_launch_var)
    int plane_variant64 = 0, plane_variant32 = 0;

    void build(const PWBasisK& b);  // host-side plans and maps only (no GPU needed)
    void ensure_device();           // uploads plans and maps on first device use
    StickMapView stick_view(int ik) const {
        const KMap& k = kmaps[ik];
        return StickMapView{nst, nz, k.gofs.ptr, k.gpk.ptr, k.glist.ptr};
    }
    PlaneMapView plane_view() const { return PlaneMapView{nst, nxc, st_xc.ptr, st_y.ptr, xpos.ptr, smap.ptr}; }
    long nxyz() const { return long(nx) * ny * nz; }
};

// Shared-memory footprint helpers (bytes) for the launch shapes used by the kernels.
constexpr int kStickTile = 16;   // sticks per CTA in the z passes
constexpr int kPlaneCols = 8;    // y-FFT column chunk in the plane pass
constexpr int kPlaneRows = 8;    // x-FFT row chunk in the plane pass
constexpr int kBoxTile = 16;     // z-columns per CTA in the box x/y passes
inline int odd_ld(int n) { return n | 1; }
size_t zpass_smem(const PWGrid& g, size_t elem);
size_t plane_smem(const PWGrid& g, size_t elem);

// ---- launchers (fft_kernels.cu); all asynchronous on `s` ----
// Fused local part of H|psi> for nb bands (one chunk): hpsi = Ekin psi + V_loc psi (accumulate==0 zeroes padding).
template <typename T, typename R>
void launch_hpsi_local(const PWGrid& g, int ik, const R* veff_zyx, const R* veff_perm, int nb, int ld, const T* psi,
                       T* hpsi, T* stickbuf, double tpiba2, int accumulate, cudaStream_t s);
// Same, with warp-synchronous compile-time transforms; returns false (launching nothing) for
// grid sizes it does not cover.
template <typename T, typename R>
bool launch_hpsi_local_fast(const PWGrid& g, int ik, const R* veff_zyx, const R* veff_perm, int nb, int ld,
                            const T* psi, T* hpsi, T* stickbuf, double tpiba2, int accumulate, cudaStream_t s);
// k-point batch: one entry per k (its stick maps, psi / hpsi with leading dimension ld, npwk, gk2 in the
// precision of the call); passed by value so a launch needs no device-side argument buffer.
constexpr int kMaxKBatch = 128;
struct KBatchEntry {
    StickMapView sm;
    const void* psi;
    void* hpsi;
    int ld, npw;
    const void* gk2;
};
struct KBatchArgs {
    KBatchEntry e[kMaxKBatch];
};
// Kinetic + local part of H|psi> for nb bands of nk k-points in one launch per pass (per band chunk);
// returns false for grid sizes without compiled warp transforms.
template <typename T, typename R>
bool launch_hpsi_local_kbatch(const PWGrid& g, const KBatchArgs& args, int nk, int nb, const R* veff_zyx,
                              const R* veff_perm, T* stickbuf, int chunk, double tpiba2, cudaStream_t s);
// Drop-in transforms (PW_Basis_K::recip_to_real / real_to_recip on the GPU), one band.
// the local part of H|psi> for npol = 2 (Veff::act's spinor branch, veff_pw.cpp:73-104, with Ekinetic::act on both
// components): ncols spinor columns (band b's components at columns 2b, 2b+1, pitch ld), the four V_eff
// components in (z, y, x) order; stickbuf holds ncols stick sets, rbuf ncols real-space boxes
template <typename T, typename R>
void launch_hpsi_local_nc(const PWGrid& g, int ik, const R* veff4_zyx, int ncols, int ld, const T* psi, T* hpsi,
                          T* stickbuf, T* rbuf, double tpiba2, cudaStream_t s);
template <typename T>
void launch_recip_to_real(const PWGrid& g, int ik, const T* in, T* out, T* aux, int add, double factor, cudaStream_t s);
template <typename T>
void launch_real_to_recip(const PWGrid& g, int ik, const T* in, T* out, T* aux, int add, double factor, cudaStream_t s);
// V_eff (ABACUS r order) -> (z, y, x) transposed copy, in precision R.
template <typename R>
void launch_transpose_veff(const PWGrid& g, const double* veff, R* out, cudaStream_t s);
// Square xy planes of n = 32*m (m = 2, 3, 4) use register/shuffle transforms whose r-space values come out
// in a permuted order; V_eff is stored once in that order: out[z][sy][sx] = veff_zyx[z][p(sy)][p(sx)],
// p(s) = s/32 + m*bitrev5(s mod 32).  Returns false (nothing done) for other grids.
bool plane_perm_supported(const PWGrid& g);
// psi -> rho on the register transforms (grids with plane_perm_supported whose plane fits shared memory):
// bands [b0, b0 + nbc) of psi through the inverse z pass into sb, then w_chunk[b] |psi_b(r)|^2 summed into
// nsplit partial planes ws (slot order; first = 1 overwrites them); launch_rho_reduce_r adds them to rho
bool rho_r_supported(const PWGrid& g);
template <typename T, typename R>
void launch_rho_chunk_r(const PWGrid& g, int ik, int b0, int nbc, int ld, const T* psi, const double* w_chunk,
                        T* sb, int nsplit, R* ws, int first, cudaStream_t s);
template <typename R>
void launch_rho_reduce_r(const PWGrid& g, int nsplit, const R* ws, R* rho, cudaStream_t s);
template <typename R>
bool launch_permute_veff(const PWGrid& g, const R* veff_zyx, R* out, cudaStream_t s);
// The same grids: V_eff arranged for the two-pass plane transforms, out[z slot][p][k1][k2] =
// veff_zyx[z][y(p)][k1 + R1 k2] with N = 8 R1, y(p) = p/8 + R1 (p mod 8) (plane_t.cuh)
template <typename R>
bool launch_arrange_veff(const PWGrid& g, const R* veff_zyx, R* out, cudaStream_t s);
// Number of plane-pass variants the autotuner may choose from (1 .. kPlaneVariants)
constexpr int kPlaneVariants = 5;

}  // namespace b200
