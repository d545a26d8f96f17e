// Test infrastructure (oracle): a C entry point to the reference's own PW_Basis_K set-up
// (module_basis/module_pw/pw_init.cpp, pw_basis.cpp, pw_basis_k.cpp, pw_distributeg*.cpp, compiled from the
// reference sources by oracle/build_ref.py; FFTW plans through the stand-in of oracle/ref/fftw_stub.cpp, never
// executed), for comparing its plane-wave spheres and index maps with this library's.  The product never
// loads it.
//
// As ESolver_KS_PW sets the wavefunction basis up: the charge grid from ecutrho (initgrids(lat0, latvec,
// ecutrho), the 2,3,5-smooth rule) unless an explicit grid is given, then the wavefunction basis on that grid
// (initgrids(lat0, latvec, nx, ny, nz)), initparameters(gamma_only = false, ecutwfc, nks, kvec_d),
// setuptransform, collect_local_pw and get_ig2ixyz_k.
#include <algorithm>
#include <complex>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "module_base/matrix3.h"
#include "module_base/vector3.h"
#include "module_basis/module_pw/pw_basis.h"
#include "module_basis/module_pw/pw_basis_k.h"
#include "module_hamilt_pw/hamilt_pwdft/operator_pw/ekinetic_pw.h"
#include "module_hamilt_pw/hamilt_pwdft/operator_pw/veff_pw.h"

namespace {
std::string g_err_pw;

// the wavefunction basis as ESolver_KS_PW builds it (see the file comment)
std::unique_ptr<ModulePW::PW_Basis_K> make_basis(double lat0, const double* latvec, double ecutwfc, double ecutrho,
                                                 int nx, int ny, int nz, int nks, const double* kvec_d) {
    const ModuleBase::Matrix3 lv(latvec[0], latvec[1], latvec[2], latvec[3], latvec[4], latvec[5], latvec[6],
                                 latvec[7], latvec[8]);
    int gx = nx, gy = ny, gz = nz;
    if (gx <= 0 || gy <= 0 || gz <= 0) {
        ModulePW::PW_Basis rho;
        rho.initgrids(lat0, lv, ecutrho);
        gx = rho.nx;
        gy = rho.ny;
        gz = rho.nz;
    }
    std::vector<ModuleBase::Vector3<double>> kd(nks);
    for (int ik = 0; ik < nks; ++ik) kd[ik] = ModuleBase::Vector3<double>(kvec_d[3 * ik], kvec_d[3 * ik + 1], kvec_d[3 * ik + 2]);
    auto wfc = std::make_unique<ModulePW::PW_Basis_K>();
    wfc->initgrids(lat0, lv, gx, gy, gz);
    wfc->initparameters(false, ecutwfc, nks, kd.data());
    wfc->setuptransform();
    wfc->collect_local_pw();
    wfc->get_ig2ixyz_k();
    return wfc;
}
}  // namespace

extern "C" {

const char* ref_pw_basis_last_error() { return g_err_pw.c_str(); }

// latvec: 9 doubles, rows a1, a2, a3 in units of lat0; kvec_d: nks x 3.  Outputs: dims = (nx, ny, nz,
// npwk_max); npwk: nks; ig2ixyz and gk2: nks x cap entries (k-point ik at ik * cap), filled when
// cap >= npwk_max (otherwise only dims and npwk are written).  Returns 0 on success.
int ref_pw_basis_k(double lat0, const double* latvec, double ecutwfc, double ecutrho, int nx, int ny, int nz, int nks,
                   const double* kvec_d, int* dims, int* npwk, int cap, int* ig2ixyz, double* gk2) {
    try {
        auto b = make_basis(lat0, latvec, ecutwfc, ecutrho, nx, ny, nz, nks, kvec_d);
        ModulePW::PW_Basis_K& wfc = *b;
        dims[0] = wfc.nx;
        dims[1] = wfc.ny;
        dims[2] = wfc.nz;
        dims[3] = wfc.npwk_max;
        for (int ik = 0; ik < nks; ++ik) npwk[ik] = wfc.npwk[ik];
        if (cap >= wfc.npwk_max && ig2ixyz && gk2) {
            for (int ik = 0; ik < nks; ++ik)
                for (int ig = 0; ig < wfc.npwk[ik]; ++ig) {
                    ig2ixyz[ik * cap + ig] = wfc.ig2ixyz_k_[ik * wfc.npwk_max + ig];
                    gk2[ik * cap + ig] = wfc.gk2[ik * wfc.npwk_max + ig];
                }
        }
        g_err_pw.clear();
        return 0;
    } catch (const std::exception& e) {
        g_err_pw = e.what();
        return 1;
    }
}

// PW_Basis_K::recip2real (inverse != 0: npwk[ik] coefficients -> nx ny nz box, r order) or real2recip
// (inverse == 0: box -> coefficients) <double> of k-point ik, with add / factor as the reference
// (pw_transform_k.cpp:26-213), through its FFT class on the stand-in transforms of oracle/ref/fftw_stub.cpp.
int ref_pw_transform(double lat0, const double* latvec, double ecutwfc, double ecutrho, int nx, int ny, int nz,
                     int nks, const double* kvec_d, int ik, int inverse, const void* in, void* out, int add,
                     double factor) {
    try {
        auto b = make_basis(lat0, latvec, ecutwfc, ecutrho, nx, ny, nz, nks, kvec_d);
        using C = std::complex<double>;
        if (inverse)
            b->recip2real<double>(static_cast<const C*>(in), static_cast<C*>(out), ik, add != 0, factor);
        else
            b->real2recip<double>(static_cast<const C*>(in), static_cast<C*>(out), ik, add != 0, factor);
        g_err_pw.clear();
        return 0;
    } catch (const std::exception& e) {
        g_err_pw = e.what();
        return 1;
    }
}

// The kinetic and local parts of H|psi> for k-point ik by the reference's own operators, Ekinetic then Veff
// (operator_pw/ekinetic_pw.cpp, veff_pw.cpp with kernels/ekinetic_op.cpp, veff_op.cpp), chained as
// Operator::hPsi does for them (hpsi zeroed first, operator.cpp:39-88): psi and hpsi are nbands vectors at
// stride npwk_max; veff: the nx ny nz box in r order (one spin).
int ref_hpsi_local(double lat0, const double* latvec, double ecutwfc, double ecutrho, int nx, int ny, int nz, int nks,
                   const double* kvec_d, int ik, const double* veff, int nbands, const void* psi, void* hpsi) {
    try {
        using T = std::complex<double>;
        using Cpu = base_device::DEVICE_CPU;
        auto b = make_basis(lat0, latvec, ecutwfc, ecutrho, nx, ny, nz, nks, kvec_d);
        hamilt::Ekinetic<hamilt::OperatorPW<T, Cpu>> ek(b->tpiba2, b->gk2, b->nks, b->npwk_max);
        std::vector<int> isk(nks, 0);
        hamilt::Veff<hamilt::OperatorPW<T, Cpu>> ve(isk.data(), veff, 1, b->nrxx, b.get());
        ek.init(ik);
        ve.init(ik);
        const int ld = b->npwk_max;
        T* out = static_cast<T*>(hpsi);
        std::fill(out, out + static_cast<size_t>(nbands) * ld, T(0.0, 0.0));
        ek.act(nbands, ld, 1, static_cast<const T*>(psi), out, b->npwk[ik]);
        ve.act(nbands, ld, 1, static_cast<const T*>(psi), out, b->npwk[ik]);
        g_err_pw.clear();
        return 0;
    } catch (const std::exception& e) {
        g_err_pw = e.what();
        return 1;
    }
}

}  // extern "C"
