// Device Hamiltonian for one pool: V_eff, projectors, D and workspaces.
#pragma once
#include <cublas_v2.h>

#include <vector>

#include "common.h"
#include "gemm_tc.h"
#include "pw_grid.h"

namespace b200 {

#define B200_CUBLAS(call)                                                                                       \
    do {                                                                                                        \
        cublasStatus_t st_ = (call);                                                                            \
        if (st_ != CUBLAS_STATUS_SUCCESS)                                                                       \
            throw ::b200::Error(::b200::kCublasError, std::string(#call) + " failed with status " +           \
                                                          std::to_string(int(st_)));                           \
    } while (0)

struct NonlocalK {
    int nkb = 0, npwx = 0;
    DeviceArray<double2> vkb;   // nkb x npwx row-major (column-major npwx x nkb)
    DeviceArray<float2> vkbf;   // FP32 copy, leading dimension ldf = npwx rounded up to even (TMA row pitch)
    int ldf = 0;
};

struct Hamilt {
    PWGrid* grid = nullptr;
    int precision = 0;  // 0 = FP64, 1 = mixed
    DeviceArray<double> veff_zyx;
    DeviceArray<float> veff_zyxf;
    bool has_veff = false;
    std::vector<NonlocalK> nl;
    int ntype = 0, nspin = 1, dx = 0, dy = 0, dz = 0;
    std::vector<int> na, nh;
    DeviceArray<double> deeq;
    DeviceArray<float> deeqf;
    // workspaces
    DeviceArray<double2> sb64, becp64, ps64;
    DeviceArray<float2> sb32, becp32, ps32, psi_pad32;
    cublasHandle_t cublas = nullptr;
    TcGemmWorkspace tcw;  // tensor-core GEMM workspace (mixed precision projectors)

    explicit Hamilt(PWGrid* g, int prec);
    ~Hamilt();
    void set_veff(const double* veff_d);
    void set_vkb(int ik, int nkb, int npwx, const double2* vkb_d);
    void set_deeq(int ntype, const int* na, const int* nh, int nspin, int dx, int dy, int dz, const double* deeq_d);
    int band_chunk(size_t elem) const;
    // mode 0 = full H, 1 = kinetic + local only (overwrites hpsi), 2 = nonlocal only (accumulates)
    template <typename T> void hpsi(int ik, int spin, int nb, int ld, const T* psi, T* hpsi, int mode, cudaStream_t s);
};

}  // namespace b200
