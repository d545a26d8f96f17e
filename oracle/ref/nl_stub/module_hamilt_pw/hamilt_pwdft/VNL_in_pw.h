// Test infrastructure (oracle): stand-in for the reference's pseudopot_cell_vnl
// (module_hamilt_pw/hamilt_pwdft/VNL_in_pw.h) when its Nonlocal operator is compiled from its source.  The
// operator reads the projector count nkb, the projectors' leading dimension vkb.nc, the bounds of D
// (deeq.getBound2..4) and the data pointers of vkb, D and the non-collinear D; getvnl (which would rebuild
// vkb for k-point ik) leaves the projectors the caller set.
#ifndef VNL_IN_PW_H
#define VNL_IN_PW_H

#include <complex>

#include "module_basis/module_pw/pw_basis_k.h"
#include "module_cell/unitcell.h"

struct OracleBounds4 {
    int b1 = 0, b2 = 0, b3 = 0, b4 = 0;
    int getBound1() const { return b1; }
    int getBound2() const { return b2; }
    int getBound3() const { return b3; }
    int getBound4() const { return b4; }
};

struct OracleMatrixShape {
    int nr = 0, nc = 0;
};

class pseudopot_cell_vnl {
  public:
    int nkb = 0;
    OracleBounds4 deeq, deeq_nc;
    double* d_deeq = nullptr;
    mutable OracleMatrixShape vkb;
    double* deeq_data = nullptr;
    std::complex<double>* deeq_nc_data = nullptr;
    std::complex<double>* vkb_data = nullptr;

    template <typename FPTYPE> FPTYPE* get_deeq_data() const;
    template <typename FPTYPE> std::complex<FPTYPE>* get_deeq_nc_data() const;
    template <typename FPTYPE> std::complex<FPTYPE>* get_vkb_data() const;
    template <typename FPTYPE, typename Device>
    void getvnl(Device*, const int&, std::complex<FPTYPE>*) const {}
};

template <> inline double* pseudopot_cell_vnl::get_deeq_data<double>() const { return deeq_data; }
template <> inline float* pseudopot_cell_vnl::get_deeq_data<float>() const { return nullptr; }
template <> inline std::complex<double>* pseudopot_cell_vnl::get_deeq_nc_data<double>() const { return deeq_nc_data; }
template <> inline std::complex<float>* pseudopot_cell_vnl::get_deeq_nc_data<float>() const { return nullptr; }
template <> inline std::complex<double>* pseudopot_cell_vnl::get_vkb_data<double>() const { return vkb_data; }
template <> inline std::complex<float>* pseudopot_cell_vnl::get_vkb_data<float>() const { return nullptr; }

#endif
