// Device Hamiltonian: the Ekinetic -> Veff -> Nonlocal chain of HamiltPW
// (hamilt_pw.cpp:21-114) as one fused local pass plus the projector GEMMs.
#include <algorithm>

#include "functors.h"
#include "hamilt.h"

namespace b200 {

// rows x cols (row pitch lda) complex128 -> complex64 with row pitch ldb (the extra column zeroed)
__global__ void k_z2c_pitch(int rows, int cols, int lda, int ldb, const double2* __restrict__ a, float2* __restrict__ b) {
    const long n = long(rows) * ldb;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int r = int(i / ldb);
        const int c = int(i - long(r) * ldb);
        b[i] = c < cols ? make_float2(float(a[long(r) * lda + c].x), float(a[long(r) * lda + c].y)) : make_float2(0.f, 0.f);
    }
}

// The atom types of D as the folding kernel sees them (by value)
struct FoldTypes {
    int ntype;
    int sum0[kVnlMaxTypes + 1];  // first projector row of each type
    int iat0[kVnlMaxTypes];      // first atom of each type
    int nh[kVnlMaxTypes];
};

// out[sum + ia*nh + x][g] = sum_k D(spin, iat + ia, x, k) vkb[sum + ia*nh + k][g], in FP64, stored in To with
// row pitch ldo (the order of add_nonlocal_pp's ps = D becp, nonlocal_pw.cpp:64-110, moved onto the projectors)
template <typename To>
__global__ void k_fold_deeq(int nkb, int npwx, int ldo, FoldTypes ft, int spin, int dx, int dy, int dz,
                            const double* __restrict__ deeq, const double2* __restrict__ vkb, To* __restrict__ out) {
    const long total = long(nkb) * npwx;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int g = int(t % npwx);
        const int j = int(t / npwx);
        int it = 0;
        while (it + 1 < ft.ntype && j >= ft.sum0[it + 1]) ++it;
        const int nh = ft.nh[it];
        const int ia = (j - ft.sum0[it]) / nh;
        const int x = (j - ft.sum0[it]) - ia * nh;
        const int row0 = ft.sum0[it] + ia * nh;
        const double* d = deeq + (long(spin * dx + ft.iat0[it] + ia) * dy + x) * dz;
        double re = 0.0, im = 0.0;
        for (int k = 0; k < nh; ++k) {
            const double2 v = vkb[long(row0 + k) * npwx + g];
            re = fma(d[k], v.x, re);
            im = fma(d[k], v.y, im);
        }
        To o;
        o.x = re;
        o.y = im;
        out[long(j) * ldo + g] = o;
    }
}

// npol = 2: W_s[x][g] = sum_k D_s(iat, k, x) vkb[row0 + k][g] for the four spin blocks s (block s at rows
// s * nkb, row pitch ldo): add_nonlocal_pp's spinor form (nonlocal_op.cpp:43-74: ps_up = D0 becp_up +
// D1 becp_dn, ps_dn = D2 becp_up + D3 becp_dn, then H psi += vkb ps) moved onto the projectors
template <typename To>
__global__ void k_fold_deeq_nc(int nkb, int npwx, int ldo, FoldTypes ft, int dx, int dy, int dz,
                               const double2* __restrict__ dnc, const double2* __restrict__ vkb, To* __restrict__ out) {
    const long total = 4L * nkb * npwx;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int g = int(t % npwx);
        const long q = t / npwx;
        const int sblk = int(q / nkb);
        const int j = int(q - long(sblk) * nkb);
        int it = 0;
        while (it + 1 < ft.ntype && j >= ft.sum0[it + 1]) ++it;
        const int nh = ft.nh[it];
        const int ia = (j - ft.sum0[it]) / nh;
        const int x = (j - ft.sum0[it]) - ia * nh;
        const int row0 = ft.sum0[it] + ia * nh;
        const double2* d = dnc + (long(sblk * dx + ft.iat0[it] + ia) * dy) * dz + x;  // D_s(iat, k, x) at d[k dz]
        double re = 0.0, im = 0.0;
        for (int k = 0; k < nh; ++k) {
            const double2 c = d[long(k) * dz];
            const double2 v = vkb[long(row0 + k) * npwx + g];
            re = fma(c.x, v.x, fma(-c.y, v.y, re));
            im = fma(c.x, v.y, fma(c.y, v.x, im));
        }
        To o;
        o.x = re;
        o.y = im;
        out[q * ldo + g] = o;
    }
}

HpsiWork::HpsiWork() { B200_CUBLAS(cublasCreate(&cublas)); }
HpsiWork::~HpsiWork() {
    if (side) cudaStreamSynchronize(side);
    if (cublas) cublasDestroy(cublas);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
}
void HpsiWork::ensure_side() {
    if (!side) B200_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    if (!ev_fork) B200_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    if (!ev_join) B200_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
}

Hamilt::Hamilt(PWGrid* g, int prec) : grid(g), precision(prec) { nl.resize(g->kmaps.size()); }

Hamilt::~Hamilt() = default;

void Hamilt::set_veff(const double* veff_d) {
    const size_t N = size_t(grid->nxyz());
    veff_zyx.resize(N);
    launch_transpose_veff<double>(*grid, veff_d, veff_zyx.ptr, 0);
    veff_zyxf.resize(N);
    launch_transpose_veff<float>(*grid, veff_d, veff_zyxf.ptr, 0);
    has_perm = plane_perm_supported(*grid);
    if (has_perm) {
        // two layouts back to back: the warp-shuffle plane pass's, then the two-pass plane pass's
        veff_perm.resize(2 * N);
        veff_permf.resize(2 * N);
        launch_permute_veff<double>(*grid, veff_zyx.ptr, veff_perm.ptr, 0);
        launch_permute_veff<float>(*grid, veff_zyxf.ptr, veff_permf.ptr, 0);
        launch_arrange_veff<double>(*grid, veff_zyx.ptr, veff_perm.ptr + N, 0);
        launch_arrange_veff<float>(*grid, veff_zyxf.ptr, veff_permf.ptr + N, 0);
    }
    B200_CUDA(cudaStreamSynchronize(0));
    has_veff = true;
}

template <> const double* Hamilt::veff_of<double>() const { return veff_zyx.ptr; }
template <> const float* Hamilt::veff_of<float>() const { return veff_zyxf.ptr; }
template <> const double* Hamilt::veff_perm_of<double>() const { return has_perm ? veff_perm.ptr : nullptr; }
template <> const float* Hamilt::veff_perm_of<float>() const { return has_perm ? veff_permf.ptr : nullptr; }

void Hamilt::set_vkb(int ik, int nkb, int npwx, const double2* vkb_d) {
    B200_CHECK(ik >= 0 && ik < int(nl.size()), kInvalidArgument, "k-point index out of range");
    NonlocalK& k = nl[ik];
    k.nkb = nkb;
    k.npwx = npwx;
    if (nkb <= 0) return;
    B200_CHECK(npwx >= grid->kmaps[ik].npw, kInvalidArgument, "npwx smaller than npwk");
    const long n = long(nkb) * npwx;
    k.vkb.resize(n);
    B200_CUDA(cudaMemcpyAsync(k.vkb.ptr, vkb_d, n * sizeof(double2), cudaMemcpyDeviceToDevice, 0));
    k.ldf = npwx + (npwx & 1);
    k.vkbf.resize(size_t(nkb) * k.ldf);
    k_z2c_pitch<<<592, 256>>>(nkb, npwx, npwx, k.ldf, vkb_d, k.vkbf.ptr);
    note_launch();
    B200_CUDA(cudaGetLastError());
    fold_projectors(ik, 0);
    B200_CUDA(cudaStreamSynchronize(0));
}

void Hamilt::set_deeq(int ntype_, const int* na_, const int* nh_, int nspin_, int dx_, int dy_, int dz_,
                      const double* deeq_d) {
    B200_CHECK(ntype_ >= 0 && nspin_ >= 1, kInvalidArgument, "bad deeq shape");
    ntype = ntype_;
    na.assign(na_, na_ + ntype);
    nh.assign(nh_, nh_ + ntype);
    nspin = nspin_;
    dx = dx_;
    dy = dy_;
    dz = dz_;
    const long n = long(nspin) * dx * dy * dz;
    deeq.resize(n);
    B200_CUDA(cudaMemcpyAsync(deeq.ptr, deeq_d, n * sizeof(double), cudaMemcpyDeviceToDevice, 0));
    for (int ik = 0; ik < int(nl.size()); ++ik) fold_projectors(ik, 0);
    B200_CUDA(cudaStreamSynchronize(0));
}

void Hamilt::set_veff_nc(const double* veff4_d) {
    const size_t N = size_t(grid->nxyz());
    veff_nc_zyx.resize(4 * N);
    veff_nc_zyxf.resize(4 * N);
    for (int c = 0; c < 4; ++c) {
        launch_transpose_veff<double>(*grid, veff4_d + c * N, veff_nc_zyx.ptr + c * N, 0);
        launch_transpose_veff<float>(*grid, veff4_d + c * N, veff_nc_zyxf.ptr + c * N, 0);
    }
    B200_CUDA(cudaStreamSynchronize(0));
    has_veff_nc = true;
}

void Hamilt::set_deeq_nc(int ntype_, const int* na_, const int* nh_, int dx_, int dy_, int dz_,
                         const double2* deeq_nc_d) {
    B200_CHECK(ntype_ >= 0 && dx_ >= 0 && dy_ >= 0 && dz_ >= 0, kInvalidArgument, "bad deeq_nc shape");
    ntype = ntype_;
    na.assign(na_, na_ + ntype);
    nh.assign(nh_, nh_ + ntype);
    nc_dx = dx_;
    nc_dy = dy_;
    nc_dz = dz_;
    const long n = 4L * dx_ * dy_ * dz_;
    deeq_nc.resize(size_t(n));
    if (n) B200_CUDA(cudaMemcpyAsync(deeq_nc.ptr, deeq_nc_d, n * sizeof(double2), cudaMemcpyDeviceToDevice, 0));
    for (int ik = 0; ik < int(nl.size()); ++ik) fold_projectors(ik, 0);
    B200_CUDA(cudaStreamSynchronize(0));
}

// the atom types of D for the folding kernels (checked against the projector count)
static FoldTypes fold_types(int ntype, const std::vector<int>& na, const std::vector<int>& nh, int nkb, int natoms_max,
                            int nh_max) {
    B200_CHECK(ntype >= 1 && ntype <= kVnlMaxTypes, kInvalidArgument, "1..8 atom types supported by the projector fold");
    FoldTypes ft{};
    ft.ntype = ntype;
    int sum = 0, iat = 0;
    for (int it = 0; it < ntype; ++it) {
        ft.sum0[it] = sum;
        ft.iat0[it] = iat;
        ft.nh[it] = nh[it];
        B200_CHECK(nh[it] >= 1 && nh[it] <= nh_max, kInvalidArgument, "nh larger than D's nhm");
        sum += na[it] * nh[it];
        iat += na[it];
    }
    ft.sum0[ntype] = sum;
    B200_CHECK(sum == nkb, kInvalidArgument, "sum of na*nh over types differs from nkb");
    B200_CHECK(iat <= natoms_max, kInvalidArgument, "more atoms than D's first dimension");
    return ft;
}

// npol = 2: the spin blocks of D into the projectors of k-point ik (FP64, FP32, residue forms)
static void fold_nc(Hamilt& H, NonlocalK& k, int ik, cudaStream_t s) {
    k.nc_folded = false;
    if (k.nkb <= 0 || !H.deeq_nc.ptr || k.vkb.ptr == nullptr) return;
    const FoldTypes ft = fold_types(H.ntype, H.na, H.nh, k.nkb, H.nc_dx, std::min(H.nc_dy, H.nc_dz));
    const long total = 4L * k.nkb * k.npwx;
    const int blocks = int(std::min<long>((total + 255) / 256, 148L * 8));
    k.wnc.resize(size_t(total));
    k.wncf.resize(size_t(4) * k.nkb * k.ldf);
    if (k.ldf != k.npwx) B200_CUDA(cudaMemsetAsync(k.wncf.ptr, 0, k.wncf.n * sizeof(float2), s));
    k_fold_deeq_nc<double2><<<blocks, 256, 0, s>>>(k.nkb, k.npwx, k.npwx, ft, H.nc_dx, H.nc_dy, H.nc_dz, H.deeq_nc.ptr,
                                                  k.vkb.ptr, k.wnc.ptr);
    k_fold_deeq_nc<float2><<<blocks, 256, 0, s>>>(k.nkb, k.npwx, k.ldf, ft, H.nc_dx, H.nc_dy, H.nc_dz, H.deeq_nc.ptr,
                                                 k.vkb.ptr, k.wncf.ptr);
    note_launch(2);
    B200_CUDA(cudaGetLastError());
    if (H.fp64_gemm != 0) {
        const int npw = H.grid->kmaps[ik].npw;
        for (int half = 0; half < 2; ++half)
            oz_prepare_a('N', npw, 2 * k.nkb, k.wnc.ptr + size_t(half) * 2 * k.nkb * k.npwx, k.npwx, H.oz_mods,
                         k.wnc_oz[half], H.oz_setup, s);
    } else {
        k.wnc_oz[0] = OzOperand();
        k.wnc_oz[1] = OzOperand();
    }
    k.nc_folded = true;
}

void Hamilt::fold_projectors(int ik, cudaStream_t s) {
    NonlocalK& k = nl[ik];
    // vkb^H in residue form (becp of both spin forms) when the FP64 products run on the int8 tensor cores
    k.oz_ready = false;
    if (fp64_gemm != 0 && k.nkb > 0 && k.vkb.ptr)
        oz_prepare_a('C', k.nkb, grid->kmaps[ik].npw, k.vkb.ptr, k.npwx, oz_mods, k.vkb_oz, oz_setup, s);
    else
        k.vkb_oz = OzOperand();
    fold_nc(*this, k, ik, s);
    k.folded = false;
    if (k.nkb <= 0 || !deeq.ptr || k.vkb.ptr == nullptr) return;
    const FoldTypes ft = fold_types(ntype, na, nh, k.nkb, dx, std::min(dy, dz));
    const long total = long(k.nkb) * k.npwx;
    int blocks = int((total + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k.vkbd.resize(size_t(nspin) * total);
    k.vkbdf.resize(size_t(nspin) * k.nkb * k.ldf);
    if (k.ldf != k.npwx) B200_CUDA(cudaMemsetAsync(k.vkbdf.ptr, 0, k.vkbdf.n * sizeof(float2), s));
    for (int sp = 0; sp < nspin; ++sp) {
        k_fold_deeq<double2><<<blocks, 256, 0, s>>>(k.nkb, k.npwx, k.npwx, ft, sp, dx, dy, dz, deeq.ptr, k.vkb.ptr,
                                                    k.vkbd.ptr + size_t(sp) * total);
        k_fold_deeq<float2><<<blocks, 256, 0, s>>>(k.nkb, k.npwx, k.ldf, ft, sp, dx, dy, dz, deeq.ptr, k.vkb.ptr,
                                                   k.vkbdf.ptr + size_t(sp) * k.nkb * k.ldf);
        note_launch(2);
        B200_CUDA(cudaGetLastError());
    }
    if (fp64_gemm != 0) {
        const int npw = grid->kmaps[ik].npw;
        k.vkbd_oz.resize(size_t(nspin));
        for (int sp = 0; sp < nspin; ++sp)
            oz_prepare_a('N', npw, k.nkb, k.vkbd.ptr + size_t(sp) * total, k.npwx, oz_mods, k.vkbd_oz[sp], oz_setup, s);
        k.oz_ready = true;
    } else {
        k.vkbd_oz.clear();
    }
    k.folded = true;
}

void Hamilt::set_fp64_gemm(int mode, int nmods) {
    B200_CHECK(mode >= 0 && mode <= 2, kInvalidArgument,
               "FP64 GEMM mode must be 0 (cuBLAS), 1 (int8 tensor cores from 48 bands) or 2 (int8 always)");
    B200_CHECK(nmods >= kOzMinMods && nmods <= kOzMaxMods, kInvalidArgument, "number of moduli must be 12..16");
    fp64_gemm = mode;
    oz_mods = nmods;
    for (int ik = 0; ik < int(nl.size()); ++ik) fold_projectors(ik, 0);
    B200_CUDA(cudaStreamSynchronize(0));
}

int Hamilt::band_chunk(size_t elem) const {
    if (chunk_override > 0) return chunk_override;
    // keep one chunk's stick buffer (nst*nz per band) inside ~48 MB so the three passes hit L2
    const size_t per_band = size_t(grid->nst) * grid->nz * elem;
    size_t c = (size_t(48) << 20) / (per_band ? per_band : 1);
    if (c < 1) c = 1;
    if (c > 4096) c = 4096;
    return int(c);
}

namespace {
template <typename T> struct Blas;
// FP64 complex GEMMs go through cublasZgemm3m: on B200 (cuBLAS 12.9) it returns the same bits as
// cublasZgemm on the projector and subspace shapes and runs 18-20 % faster (42 vs 35 TFLOP/s)
template <> struct Blas<double2> {
    static cublasStatus_t gemm(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
                               const double2* alpha, const double2* A, int lda, const double2* B, int ldb,
                               const double2* beta, double2* C, int ldc) {
        return cublasZgemm3m(h, ta, tb, m, n, k, reinterpret_cast<const cuDoubleComplex*>(alpha),
                           reinterpret_cast<const cuDoubleComplex*>(A), lda, reinterpret_cast<const cuDoubleComplex*>(B),
                           ldb, reinterpret_cast<const cuDoubleComplex*>(beta), reinterpret_cast<cuDoubleComplex*>(C), ldc);
    }
};
}  // namespace

template <typename T>
void Hamilt::hpsi(int ik, int spin, int nb, int ld, const T* psi, T* hpsi, int mode, cudaStream_t s, HpsiWork* wk) {
    using R = typename RealOf<T>::type;
    HpsiWork& W = wk ? *wk : work;
    auto& sb64 = W.sb64;
    auto& sb32 = W.sb32;
    auto& becp64 = W.becp64;
    auto& becp32 = W.becp32;
    auto& psi_pad32 = W.psi_pad32;
    auto& tcw = W.tcw;
    cublasHandle_t cublas = W.cublas;
    constexpr bool f64 = std::is_same<T, double2>::value;
    B200_CHECK(ik >= 0 && ik < int(grid->kmaps.size()), kInvalidArgument, "k-point index out of range");
    const int npw = grid->kmaps[ik].npw;
    B200_CHECK(nb >= 0 && ld >= npw, kInvalidArgument, "ld smaller than npwk or negative band count");
    if (nb == 0) return;
    auto local_pass = [&](cudaStream_t st) {
        B200_CHECK(has_veff, kInvalidArgument, "V_eff not set");
        const R* veff = f64 ? (const R*)veff_zyx.ptr : (const R*)veff_zyxf.ptr;
        const int chunk = band_chunk(sizeof(T));
        const int nbc0 = nb < chunk ? nb : chunk;
        const size_t sbn = size_t(nbc0) * grid->nst * grid->nz;
        T* sb;
        if constexpr (f64) {
            sb64.resize(sbn);
            sb = sb64.ptr;
        } else {
            sb32.resize(sbn);
            sb = sb32.ptr;
        }
        for (int b0 = 0; b0 < nb; b0 += chunk) {
            const int nbc = nb - b0 < chunk ? nb - b0 : chunk;
            launch_hpsi_local<T, R>(*grid, ik, veff, veff_perm_of<R>(), nbc, ld, psi + size_t(b0) * ld,
                                    hpsi + size_t(b0) * ld, sb, grid->basis.tpiba2, 0, st);
        }
    };
    const NonlocalK& k = nl[ik];
    const bool with_nl = mode != 1 && k.nkb > 0;
    if (!with_nl) {
        if (mode != 2) local_pass(s);
        return;
    }
    const int nkb = k.nkb;
    B200_CHECK(deeq.ptr != nullptr, kInvalidArgument, "deeq not set");
    B200_CHECK(spin >= 0 && spin < nspin, kInvalidArgument, "spin out of range");
    const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
    // becp with an even leading dimension in FP32 (TMA row pitch of the second product)
    const int ldb_p = f64 ? nkb : nkb + (nkb & 1);
    T* becp;
    if constexpr (f64) {
        becp64.resize(size_t(ldb_p) * nb);
        becp = becp64.ptr;
    } else {
        becp32.resize(size_t(ldb_p) * nb);
        becp = becp32.ptr;
    }
    // Nonlocal::act (nonlocal_pw.cpp:211-304): becp = vkb^H psi, then H psi += vkb (D becp), here with D folded
    // into the projectors once per k-point and spin: H psi += vkbd becp (vkbd = D vkb per atom block)
    B200_CHECK(k.folded, kInvalidArgument, "projectors and D not both set for this k-point");
    const T* vkbd = f64 ? reinterpret_cast<const T*>(k.vkbd.ptr + size_t(spin) * nkb * k.npwx)
                        : reinterpret_cast<const T*>(k.vkbdf.ptr + size_t(spin) * nkb * k.ldf);
    const bool oz = f64 && k.oz_ready && (fp64_gemm == 2 || (fp64_gemm == 1 && nb >= kOzMinBands));
    if (oz) W.tcw.ensure();  // the int8 GEMM reports a bounded wait that ran out in the same error word
    auto projections = [&](cudaStream_t st) {
        if constexpr (f64) {
            if (oz) {
                oz_zgemm('C', nkb, nb, npw, one, k.vkb_oz, psi, ld, zero, becp, nkb, W.ozw, W.tcw.err.ptr, st);
                return;
            }
            B200_CUBLAS(cublasSetStream(cublas, st));
            B200_CUBLAS(Blas<T>::gemm(cublas, CUBLAS_OP_C, CUBLAS_OP_N, nkb, nb, npw, &one, (const T*)k.vkb.ptr, k.npwx,
                                      psi, ld, &zero, becp, nkb));
        } else {
            // mixed precision: both projector products on the tensor cores (3xTF32)
            const float2* psi_b = psi;
            int ldb = ld;
            if (ld & 1) {  // the TMA row pitch must be a multiple of 16 bytes: stage psi with an even pitch
                ldb = ld + 1;
                psi_pad32.resize(size_t(nb) * ldb);
                B200_CUDA(cudaMemcpy2DAsync(psi_pad32.ptr, size_t(ldb) * sizeof(float2), psi, size_t(ld) * sizeof(float2),
                                            size_t(npw) * sizeof(float2), nb, cudaMemcpyDeviceToDevice, st));
                psi_b = psi_pad32.ptr;
            }
            tc_cgemm('C', nkb, nb, npw, one, k.vkbf.ptr, k.ldf, psi_b, ldb, zero, becp, ldb_p, tcw, st);
        }
    };
    if (mode == 2) {
        projections(s);
    } else {
        // the projection runs on a second stream beside the local pass (it reads psi only); H psi += vkbd becp
        // waits for both
        W.ensure_side();
        B200_CUDA(cudaEventRecord(W.ev_fork, s));
        B200_CUDA(cudaStreamWaitEvent(W.side, W.ev_fork, 0));
        projections(W.side);
        B200_CUDA(cudaEventRecord(W.ev_join, W.side));
        local_pass(s);
        B200_CUDA(cudaStreamWaitEvent(s, W.ev_join, 0));
    }
    if constexpr (f64) {
        if (oz) {
            oz_zgemm('N', npw, nb, nkb, one, k.vkbd_oz[spin], becp, nkb, one, hpsi, ld, W.ozw, W.tcw.err.ptr, s);
        } else {
            B200_CUBLAS(cublasSetStream(cublas, s));
            B200_CUBLAS(Blas<T>::gemm(cublas, CUBLAS_OP_N, CUBLAS_OP_N, npw, nb, nkb, &one, vkbd, k.npwx, becp, nkb,
                                      &one, hpsi, ld));
        }
    } else {
        tc_cgemm('N', npw, nb, nkb, one, vkbd, k.ldf, becp, ldb_p, one, hpsi, ld, tcw, s);
    }
}

template <typename T>
void Hamilt::hpsi_nc(int ik, int nb, int ld, const T* psi, T* hpsi, cudaStream_t s, HpsiWork* wk) {
    using R = typename RealOf<T>::type;
    constexpr bool f64 = std::is_same<T, double2>::value;
    HpsiWork& W = wk ? *wk : work;
    B200_CHECK(ik >= 0 && ik < int(grid->kmaps.size()), kInvalidArgument, "k-point index out of range");
    const int npw = grid->kmaps[ik].npw;
    B200_CHECK(nb >= 0 && ld >= npw, kInvalidArgument, "ld smaller than npwk or negative band count");
    B200_CHECK(has_veff_nc, kInvalidArgument, "npol = 2: V_eff's four components not set");
    if (nb == 0) return;
    // local part, in chunks of bands whose real-space planes (two boxes per band) stay within 512 MB
    const size_t N = size_t(grid->nxyz());
    const size_t per_col = N * sizeof(T);
    int cb = int((size_t(512) << 20) / (2 * per_col));
    if (cb < 1) cb = 1;
    if (cb > nb) cb = nb;
    if (cb > 32767) cb = 32767;
    const R* v4 = f64 ? (const R*)veff_nc_zyx.ptr : (const R*)veff_nc_zyxf.ptr;
    T *sb, *rb;
    const size_t sbn = size_t(2) * cb * grid->nst * grid->nz, rbn = size_t(2) * cb * N;
    if constexpr (f64) {
        W.sb64.resize(sbn);
        W.rb64.resize(rbn);
        sb = W.sb64.ptr;
        rb = W.rb64.ptr;
    } else {
        W.sb32.resize(sbn);
        W.rb32.resize(rbn);
        sb = W.sb32.ptr;
        rb = W.rb32.ptr;
    }
    for (int b0 = 0; b0 < nb; b0 += cb) {
        const int nbc = nb - b0 < cb ? nb - b0 : cb;
        launch_hpsi_local_nc<T, R>(*grid, ik, v4, 2 * nbc, ld, psi + size_t(2) * b0 * ld, hpsi + size_t(2) * b0 * ld, sb,
                                   rb, grid->basis.tpiba2, s);
    }
    // Nonlocal::act with npol = 2 (nonlocal_pw.cpp:211-283 with add_nonlocal_pp's spinor form): becp of the 2 nb
    // spinor columns, read as [becp_up; becp_dn] (2 nkb x nb), then H psi_up += [W0 W1] becp, H psi_dn += [W2 W3] becp
    const NonlocalK& k = nl[ik];
    if (k.nkb <= 0) return;
    B200_CHECK(k.nc_folded, kInvalidArgument, "npol = 2: projectors and deeq_nc not both set for this k-point");
    const int nkb = k.nkb;
    const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
    T* becp;
    if constexpr (f64) {
        W.becp64.resize(size_t(2) * nkb * nb);
        becp = W.becp64.ptr;
        const bool oz = k.vkb_oz.res.ptr && k.wnc_oz[0].res.ptr && (fp64_gemm == 2 || (fp64_gemm == 1 && nb >= kOzMinBands));
        if (oz) {
            W.tcw.ensure();
            oz_zgemm('C', nkb, 2 * nb, npw, one, k.vkb_oz, psi, ld, zero, becp, nkb, W.ozw, W.tcw.err.ptr, s);
            for (int half = 0; half < 2; ++half)
                oz_zgemm('N', npw, nb, 2 * nkb, one, k.wnc_oz[half], becp, 2 * nkb, one, hpsi + size_t(half) * ld, 2 * ld,
                         W.ozw, W.tcw.err.ptr, s);
        } else {
            B200_CUBLAS(cublasSetStream(W.cublas, s));
            const cuDoubleComplex* o = reinterpret_cast<const cuDoubleComplex*>(&one);
            const cuDoubleComplex* z0 = reinterpret_cast<const cuDoubleComplex*>(&zero);
            B200_CUBLAS(cublasZgemm3m(W.cublas, CUBLAS_OP_C, CUBLAS_OP_N, nkb, 2 * nb, npw, o,
                                      reinterpret_cast<const cuDoubleComplex*>(k.vkb.ptr), k.npwx,
                                      reinterpret_cast<const cuDoubleComplex*>(psi), ld, z0,
                                      reinterpret_cast<cuDoubleComplex*>(becp), nkb));
            for (int half = 0; half < 2; ++half)
                B200_CUBLAS(cublasZgemm3m(W.cublas, CUBLAS_OP_N, CUBLAS_OP_N, npw, nb, 2 * nkb, o,
                                          reinterpret_cast<const cuDoubleComplex*>(k.wnc.ptr + size_t(half) * 2 * nkb * k.npwx),
                                          k.npwx, reinterpret_cast<const cuDoubleComplex*>(becp), 2 * nkb, o,
                                          reinterpret_cast<cuDoubleComplex*>(hpsi + size_t(half) * ld), 2 * ld));
        }
    } else {
        W.becp32.resize(size_t(2) * nkb * nb);
        becp = W.becp32.ptr;
        const float2* psi_b = psi;
        int ldb = ld;
        if (ld & 1) {  // the TMA row pitch must be a multiple of 16 bytes: stage psi with an even pitch
            ldb = ld + 1;
            W.psi_pad32.resize(size_t(2) * nb * ldb);
            B200_CUDA(cudaMemcpy2DAsync(W.psi_pad32.ptr, size_t(ldb) * sizeof(float2), psi, size_t(ld) * sizeof(float2),
                                        size_t(npw) * sizeof(float2), 2 * nb, cudaMemcpyDeviceToDevice, s));
            psi_b = W.psi_pad32.ptr;
        }
        tc_cgemm('C', nkb, 2 * nb, npw, one, k.vkbf.ptr, k.ldf, psi_b, ldb, zero, becp, nkb, W.tcw, s);
        for (int half = 0; half < 2; ++half)
            tc_cgemm('N', npw, nb, 2 * nkb, one, k.wncf.ptr + size_t(half) * 2 * nkb * k.ldf, k.ldf, becp, 2 * nkb, one,
                     hpsi + size_t(half) * ld, 2 * ld, W.tcw, s);
    }
}

template void Hamilt::hpsi_nc<double2>(int, int, int, const double2*, double2*, cudaStream_t, HpsiWork*);
template void Hamilt::hpsi_nc<float2>(int, int, int, const float2*, float2*, cudaStream_t, HpsiWork*);

template <typename T>
void Hamilt::hpsi_kbatch(int nk, const int* iks, int spin, int nb, int ld, const T* const* psis, T* const* hpsis,
                         cudaStream_t s, HpsiWork* wk) {
    using R = typename RealOf<T>::type;
    constexpr bool f64 = std::is_same<T, double2>::value;
    B200_CHECK(nk >= 1 && nk <= kMaxKBatch, kInvalidArgument, "k-point batch must hold 1..128 k-points");
    B200_CHECK(has_veff, kInvalidArgument, "V_eff not set");
    HpsiWork& W = wk ? *wk : work;
    KBatchArgs args;
    for (int q = 0; q < nk; ++q) {
        const int ik = iks[q];
        B200_CHECK(ik >= 0 && ik < int(grid->kmaps.size()), kInvalidArgument, "k-point index out of range");
        const KMap& km = grid->kmaps[ik];
        B200_CHECK(ld >= km.npw, kInvalidArgument, "ld smaller than npwk");
        args.e[q].sm = grid->stick_view(ik);
        args.e[q].psi = psis[q];
        args.e[q].hpsi = hpsis[q];
        args.e[q].ld = ld;
        args.e[q].npw = km.npw;
        args.e[q].gk2 = f64 ? (const void*)km.gk2.ptr : (const void*)km.gk2f.ptr;
    }
    const size_t per_band = size_t(grid->nst) * grid->nz * sizeof(T);
    int chunk = chunk_override > 0 ? chunk_override : int((size_t(48) << 20) / (per_band * nk));
    if (chunk < 1) chunk = 1;
    if (chunk > nb) chunk = nb;
    const R* veff = f64 ? (const R*)veff_zyx.ptr : (const R*)veff_zyxf.ptr;
    T* sb;
    if constexpr (f64) {
        W.sb64.resize(size_t(nk) * chunk * grid->nst * grid->nz);
        sb = W.sb64.ptr;
    } else {
        W.sb32.resize(size_t(nk) * chunk * grid->nst * grid->nz);
        sb = W.sb32.ptr;
    }
    if (!launch_hpsi_local_kbatch<T, R>(*grid, args, nk, nb, veff, veff_perm_of<R>(), sb, chunk, grid->basis.tpiba2,
                                        s)) {
        for (int q = 0; q < nk; ++q) hpsi<T>(iks[q], spin, nb, ld, psis[q], hpsis[q], 1, s, &W);
    }
    for (int q = 0; q < nk; ++q) hpsi<T>(iks[q], spin, nb, ld, psis[q], hpsis[q], 2, s, &W);
}

template void Hamilt::hpsi_kbatch<double2>(int, const int*, int, int, int, const double2* const*, double2* const*,
                                           cudaStream_t, HpsiWork*);
template void Hamilt::hpsi_kbatch<float2>(int, const int*, int, int, int, const float2* const*, float2* const*,
                                          cudaStream_t, HpsiWork*);
template void Hamilt::hpsi<double2>(int, int, int, int, const double2*, double2*, int, cudaStream_t, HpsiWork*);
template void Hamilt::hpsi<float2>(int, int, int, int, const float2*, float2*, int, cudaStream_t, HpsiWork*);

}  // namespace b200
