// Device Hamiltonian: the Ekinetic -> Veff -> Nonlocal chain of HamiltPW
// (hamilt_pw.cpp:21-114) as one fused local pass plus the projector GEMMs.
#include "functors.h"
#include "hamilt.h"

namespace b200 {

__global__ void k_d2f(long n, const double* __restrict__ a, float* __restrict__ b) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) b[i] = float(a[i]);
}
// rows x cols (row pitch lda) complex128 -> complex64 with row pitch ldb (the extra column zeroed)
__global__ void k_z2c_pitch(int rows, int cols, int lda, int ldb, const double2* __restrict__ a, float2* __restrict__ b) {
    const long n = long(rows) * ldb;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int r = int(i / ldb);
        const int c = int(i - long(r) * ldb);
        b[i] = c < cols ? make_float2(float(a[long(r) * lda + c].x), float(a[long(r) * lda + c].y)) : make_float2(0.f, 0.f);
    }
}

// ps in the K-major (becp) layout, ps[b*nkb + j] = sum_x D[x, k] becp[b*nkb + x] over the atom block of j:
// the same contraction as nonlocal_pw_op (nonlocal_op.cpp:8-41) with the output transposed for the GEMM that follows
template <typename T, typename R>
__global__ void k_nonlocal_kmajor(int l1, int nb, int l3, int sum, int iat, int spin, int nkb, int dx, int dy, int dz,
                                  const R* __restrict__ deeq, T* __restrict__ ps, const T* __restrict__ becp) {
    const long total = long(l1) * l3 * nb;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int kk = int(t % l3);
        const long r = t / l3;
        const int ii = int(r % l1);
        const int b = int(r / l1);
        const R* d = deeq + (long(spin * dx + iat + ii) * dy) * dz + kk;
        const T* bp = becp + long(b) * nkb + sum + ii * l3;
        T acc = cmake<T>(0, 0);
        for (int xx = 0; xx < l3; ++xx) acc = cadd(acc, cscale(bp[xx], d[long(xx) * dz]));
        ps[long(b) * nkb + sum + ii * l3 + kk] = acc;
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
        veff_perm.resize(N);
        veff_permf.resize(N);
        launch_permute_veff<double>(*grid, veff_zyx.ptr, veff_perm.ptr, 0);
        launch_permute_veff<float>(*grid, veff_zyxf.ptr, veff_permf.ptr, 0);
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
    deeqf.resize(n);
    k_d2f<<<592, 256>>>(n, deeq_d, deeqf.ptr);
    note_launch();
    B200_CUDA(cudaGetLastError());
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
template <> struct Blas<float2> {
    static cublasStatus_t gemm(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
                               const float2* alpha, const float2* A, int lda, const float2* B, int ldb,
                               const float2* beta, float2* C, int ldc) {
        return cublasCgemm(h, ta, tb, m, n, k, reinterpret_cast<const cuComplex*>(alpha),
                           reinterpret_cast<const cuComplex*>(A), lda, reinterpret_cast<const cuComplex*>(B), ldb,
                           reinterpret_cast<const cuComplex*>(beta), reinterpret_cast<cuComplex*>(C), ldc);
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
    auto& ps64 = W.ps64;
    auto& becp32 = W.becp32;
    auto& ps32 = W.ps32;
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
    T* becp;
    T* ps;
    if constexpr (f64) {
        becp64.resize(size_t(nkb) * nb);
        ps64.resize(size_t(nkb) * nb);
        becp = becp64.ptr;
        ps = ps64.ptr;
    } else {
        becp32.resize(size_t(nkb) * nb);
        ps32.resize(size_t(nkb) * nb);
        becp = becp32.ptr;
        ps = ps32.ptr;
    }
    const T one = cmake<T>(1, 0), zero = cmake<T>(0, 0);
    const R* d = f64 ? (const R*)deeq.ptr : (const R*)deeqf.ptr;
    B200_CHECK(d != nullptr, kInvalidArgument, "deeq not set");
    B200_CHECK(spin >= 0 && spin < nspin, kInvalidArgument, "spin out of range");
    const int ldps = f64 ? nkb : nkb + (nkb & 1);
    if constexpr (!f64) {
        if (ldps != nkb) {
            becp32.resize(size_t(ldps) * nb);
            ps32.resize(size_t(ldps) * nb);
            becp = becp32.ptr;
            ps = ps32.ptr;
        }
    }
    // first half of Nonlocal::act, which reads only psi: becp = vkb^H psi (nonlocal_pw.cpp:261-276) and
    // ps = D becp per atom type (add_nonlocal_pp, nonlocal_pw.cpp:64-110)
    auto projections = [&](cudaStream_t st) {
        if constexpr (f64) {
            const T* vkb = (const T*)k.vkb.ptr;
            B200_CUBLAS(cublasSetStream(cublas, st));
            B200_CUBLAS(Blas<T>::gemm(cublas, CUBLAS_OP_C, CUBLAS_OP_N, nkb, nb, npw, &one, vkb, k.npwx, psi, ld, &zero,
                                      becp, nkb));
            B200_CUDA(cudaMemsetAsync(ps, 0, size_t(nkb) * nb * sizeof(T), st));
            int sum = 0, iat = 0;
            for (int it = 0; it < ntype; ++it)
                nonlocal_pw<T, R>(na[it], nb, nh[it], sum, iat, spin, nkb, dx, dy, dz, d, ps, becp, st);
            B200_CHECK(sum == nkb, kInvalidArgument, "sum of na*nh over types differs from nkb");
        } else {
            // mixed precision: both projector products on the tensor cores (3xTF32), ps kept in becp's layout
            const float2* psi_b = psi;
            int ldb = ld;
            if (ld & 1) {  // the TMA row pitch must be a multiple of 16 bytes: stage psi with an even pitch
                ldb = ld + 1;
                psi_pad32.resize(size_t(nb) * ldb);
                B200_CUDA(cudaMemcpy2DAsync(psi_pad32.ptr, size_t(ldb) * sizeof(float2), psi, size_t(ld) * sizeof(float2),
                                            size_t(npw) * sizeof(float2), nb, cudaMemcpyDeviceToDevice, st));
                psi_b = psi_pad32.ptr;
            }
            tc_cgemm('C', nkb, nb, npw, one, k.vkbf.ptr, k.ldf, psi_b, ldb, zero, becp, ldps, tcw, st);
            int sum = 0, iat = 0;
            for (int it = 0; it < ntype; ++it) {
                const long total = long(na[it]) * nh[it] * nb;
                if (total > 0) {
                    int blocks = int((total + 255) / 256);
                    if (blocks > 148 * 8) blocks = 148 * 8;
                    k_nonlocal_kmajor<T, R><<<blocks, 256, 0, st>>>(na[it], nb, nh[it], sum, iat, spin, ldps, dx, dy, dz,
                                                                   d, ps, becp);
                    note_launch();
                    B200_CUDA(cudaGetLastError());
                }
                sum += na[it] * nh[it];
                iat += na[it];
            }
            B200_CHECK(sum == nkb, kInvalidArgument, "sum of na*nh over types differs from nkb");
        }
    };
    if (mode == 2) {
        projections(s);
    } else {
        // the projections run on a second stream beside the local pass (they read psi only); hpsi += vkb ps
        // waits for both
        W.ensure_side();
        B200_CUDA(cudaEventRecord(W.ev_fork, s));
        B200_CUDA(cudaStreamWaitEvent(W.side, W.ev_fork, 0));
        projections(W.side);
        B200_CUDA(cudaEventRecord(W.ev_join, W.side));
        local_pass(s);
        B200_CUDA(cudaStreamWaitEvent(s, W.ev_join, 0));
    }
    // hpsi += vkb ps^T (nonlocal_pw.cpp:190-205)
    if constexpr (f64) {
        B200_CUBLAS(cublasSetStream(cublas, s));
        B200_CUBLAS(Blas<T>::gemm(cublas, CUBLAS_OP_N, CUBLAS_OP_T, npw, nb, nkb, &one, (const T*)k.vkb.ptr, k.npwx, ps,
                                  nb, &one, hpsi, ld));
    } else {
        tc_cgemm('N', npw, nb, nkb, one, k.vkbf.ptr, k.ldf, ps, ldps, one, hpsi, ld, tcw, s);
    }
}

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
