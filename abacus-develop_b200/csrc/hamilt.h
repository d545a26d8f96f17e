// Device Hamiltonian for one pool: V_eff, projectors, D and workspaces.
#pragma once
#include <cublas_v2.h>

#include <vector>

#include "common.h"
#include "gemm_oz.h"
#include "gemm_tc.h"
#include "linalg_status.h"
#include "pw_grid.h"

namespace b200 {

struct NonlocalK {
    int nkb = 0, npwx = 0;
    DeviceArray<double2> vkb;   // nkb x npwx row-major (column-major npwx x nkb)
    DeviceArray<float2> vkbf;   // FP32 copy, leading dimension ldf = npwx rounded up to even (TMA row pitch)
    int ldf = 0;
    // D folded into the projectors for the second product of Nonlocal::act: row x of atom a is
    // sum_k D(spin, a, x, k) vkb_k, so that H psi += vkbd becp needs no ps = D becp step.  One block of
    // nkb rows per spin; rebuilt whenever the projectors or D change (set-up calls only, so H|psi> itself
    // only reads them and concurrent callers need no lock).
    DeviceArray<double2> vkbd;  // nspin x nkb x npwx
    DeviceArray<float2> vkbdf;  // nspin x nkb x ldf
    bool folded = false;
    // the FP64 products' projector operands in int8 residue form (gemm_oz.h), built with the fold when the
    // FP64 GEMMs run on the int8 tensor cores: vkb^H for becp (rows = projectors), vkbd per spin for
    // H psi += vkbd becp (rows = plane waves)
    OzOperand vkb_oz;
    std::vector<OzOperand> vkbd_oz;
    bool oz_ready = false;
    // npol = 2: the four 2x2 spin blocks of D folded into the projectors, W_s = vkb D_s per atom block; rows
    // [0, 2 nkb) = [W0; W1] (H psi_up += W0 becp_up + W1 becp_dn), rows [2 nkb, 4 nkb) = [W2; W3] (H psi_dn)
    DeviceArray<double2> wnc;  // 4 x nkb x npwx
    DeviceArray<float2> wncf;  // 4 x nkb x ldf
    OzOperand wnc_oz[2];       // residue forms of the two halves (FP64 products on the int8 tensor cores)
    bool nc_folded = false;
};

// Scratch of one H|psi> caller: stick buffer, becp, the padded-psi stage, a cuBLAS handle and the
// tensor-core GEMM workspace.  Callers that run H|psi> concurrently (different streams or threads) each
// own one; the Hamiltonian itself is read-only after set-up.
struct HpsiWork {
    DeviceArray<double2> sb64, becp64, rb64;
    DeviceArray<float2> sb32, becp32, psi_pad32, rb32;  // rb: real-space planes of the npol = 2 local pass
    cublasHandle_t cublas = nullptr;
    TcGemmWorkspace tcw;
    OzWorkspace ozw;  // the FP64 projector products on the int8 tensor cores (psi / becp residues, products)
    // second stream of an H|psi>: the projections (becp, D becp) run on it beside the local pass
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    void ensure_side();
    HpsiWork();
    ~HpsiWork();
    HpsiWork(const HpsiWork&) = delete;
    HpsiWork& operator=(const HpsiWork&) = delete;
};

// Projector tables of one cell, the inputs of pseudopot_cell_vnl::getvnl (VNL_in_pw.cpp:412-540):
// radial tables tab(it, ib, iq) on a q grid of step dq, per-type (ih -> beta, l, lm) maps and atom positions.
constexpr int kVnlMaxTypes = 8;
constexpr int kVnlMaxNh = 32;
constexpr int kVnlMaxL = 4;
struct VnlParams {  // handed to the kernel by value
    int ntype, nhm, lmax, tab_2, tab_3, nkb;
    double dq, tpiba;
    int na[kVnlMaxTypes], nbeta[kVnlMaxTypes], nh[kVnlMaxTypes];
    unsigned char indv[kVnlMaxTypes][kVnlMaxNh], nhtol[kVnlMaxTypes][kVnlMaxNh], nhtolm[kVnlMaxTypes][kVnlMaxNh];
};
struct VnlTables {
    bool set = false;
    VnlParams p{};
    int nat = 0;
    DeviceArray<double> tab;  // ntype * tab_2 * tab_3
    DeviceArray<double> tau;  // nat * 3, units of lat0, atoms grouped by type
};

struct Hamilt {
    PWGrid* grid = nullptr;
    int precision = 0;  // 0 = FP64, 1 = mixed
    DeviceArray<double> veff_zyx;
    DeviceArray<float> veff_zyxf;
    // grids with 32*m square planes: (z, y, x) in the warp-shuffle register-transform order, then (N more
    // values) the arrangement of the two-pass plane transforms
    DeviceArray<double> veff_perm;
    DeviceArray<float> veff_permf;
    bool has_perm = false;
    template <typename R> const R* veff_of() const;
    template <typename R> const R* veff_perm_of() const;
    bool has_veff = false;
    std::vector<NonlocalK> nl;
    int ntype = 0, nspin = 1, dx = 0, dy = 0, dz = 0;
    std::vector<int> na, nh;
    DeviceArray<double> deeq;
    // npol = 2 (non-collinear): V_eff's four components in (z, y, x) order, and D's four complex spin blocks
    // deeq_nc(4, dx, dy, dz) (nonlocal_op.cpp:43-74)
    DeviceArray<double> veff_nc_zyx;
    DeviceArray<float> veff_nc_zyxf;
    bool has_veff_nc = false;
    DeviceArray<double2> deeq_nc;
    int nc_dx = 0, nc_dy = 0, nc_dz = 0;
    HpsiWork work;  // default scratch for callers that do not bring their own
    int chunk_override = 0;  // bands per stick-buffer chunk chosen by the autotuner (0 = 48 MB rule)
    // FP64 projector products: 0 = cuBLAS ZGEMM; int8 tensor cores (exact modular emulation, oz_mods moduli)
    // 1 = for calls of at least kOzMinBands bands (each call reads the projectors' whole residue form, twice the
    // bytes of the FP64 projectors, so narrow calls go to cuBLAS, whose cost scales with the bands), 2 = always
    int fp64_gemm = 1;
    static constexpr int kOzMinBands = 48;
    int oz_mods = 16;
    OzWorkspace oz_setup;  // scratch of the projector residues built at fold time
    VnlTables vnl;           // projector tables for on-device getvnl

    void set_projectors(int ntype, const int* na, const int* nbeta, const int* nh, int nhm, int lmax, const int* indv,
                        const int* nhtol, const int* nhtolm, int tab_2, int tab_3, double dq, const double* tab_h,
                        const double* tau_h);
    // getvnl for k-point ik: the FP64 projectors and their FP32 copy, built on the device (stream s)
    void build_vkb(int ik, cudaStream_t s);

    explicit Hamilt(PWGrid* g, int prec);
    ~Hamilt();
    void set_veff(const double* veff_d);
    void set_vkb(int ik, int nkb, int npwx, const double2* vkb_d);
    void set_deeq(int ntype, const int* na, const int* nh, int nspin, int dx, int dy, int dz, const double* deeq_d);
    int band_chunk(size_t elem) const;
    // fold D into the projectors of k-point ik (all spins), on stream s; nothing if either is not set.  With
    // fp64_gemm = 1 also the int8 residue forms of vkb and vkbd.
    void fold_projectors(int ik, cudaStream_t s);
    // npol = 2 set-up: V_eff's four components (4 x nrxx, the reference's (x, y, z) order), D's spin blocks
    void set_veff_nc(const double* veff4_d);
    void set_deeq_nc(int ntype, const int* na, const int* nh, int dx, int dy, int dz, const double2* deeq_nc_d);
    // H|psi> with npol = 2 (hPsi's spinor branches: Ekinetic and Veff on both components, Nonlocal with deeq_nc):
    // band b's components at psi + (2 b + c) ld, c = 0, 1
    template <typename T>
    void hpsi_nc(int ik, int nb, int ld, const T* psi, T* hpsi, cudaStream_t s, HpsiWork* w = nullptr);
    // choose the FP64 projector products (0 cuBLAS, 1 int8 tensor cores from kOzMinBands bands, 2 int8 always;
    // nmods moduli) and re-fold
    void set_fp64_gemm(int mode, int nmods);
    // mode 0 = full H, 1 = kinetic + local only (overwrites hpsi), 2 = nonlocal only (accumulates)
    template <typename T>
    void hpsi(int ik, int spin, int nb, int ld, const T* psi, T* hpsi, int mode, cudaStream_t s, HpsiWork* w = nullptr);
    // H|psi> for nb bands of nk k-points: the local part in one launch per pass for all k (per band chunk),
    // the projectors per k.  psis / hpsis are host arrays of device pointers (leading dimension ld).
    template <typename T>
    void hpsi_kbatch(int nk, const int* iks, int spin, int nb, int ld, const T* const* psis, T* const* hpsis,
                     cudaStream_t s, HpsiWork* w = nullptr);
};

}  // namespace b200
