// Test infrastructure (oracle): a C entry point to the reference's own occupation code
// (module_elecstate/occupy.cpp: Occupy::gweights / efermig / sumkg / wgauss / w1gauss, compiled from the
// reference sources by oracle/build_ref.py), for the parity tests of the NSCF smearing weights.  The product
// never loads it.
#include <exception>
#include <string>
#include <vector>

#include "module_base/global_variable.h"
#include "module_base/matrix.h"
#include "module_elecstate/occupy.h"

namespace {
std::string g_err_occ;
}

extern "C" {

const char* ref_occupy_last_error() { return g_err_occ.c_str(); }

// ekb: nks x nband (row-major, Ry); wk: nks; ngauss: 0 Gaussian, n > 0 Methfessel-Paxton order n, -1 cold,
// -99 Fermi-Dirac; outputs the Fermi energy, the band-energy correction demet and wg (nks x nband).
int ref_gweights(int nks, const double* wk, int nband, double nelec, double sigma, int ngauss, const double* ekb,
                 double* ef, double* demet, double* wg) {
    try {
        GlobalV::NBANDS = nband;
        ModuleBase::matrix e(nks, nband), w(nks, nband);
        for (int i = 0; i < nks * nband; ++i) e.c[i] = ekb[i];
        std::vector<double> wkv(wk, wk + nks);
        std::vector<int> isk(nks, 0);
        Occupy::gweights(nks, wkv, nband, nelec, sigma, ngauss, e, *ef, *demet, w, -1, isk);
        for (int i = 0; i < nks * nband; ++i) wg[i] = w.c[i];
        g_err_occ.clear();
        return 0;
    } catch (const std::exception& ex) {
        g_err_occ = ex.what();
        return 1;
    }
}

}  // extern "C"
