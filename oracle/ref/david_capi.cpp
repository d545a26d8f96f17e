// Test infrastructure (oracle): a C entry point to the reference's own CPU DiagoDavid
// (module_hsolver/diago_david.cpp, compiled from the reference sources by oracle/build_ref.py), for the
// parity tests and the benchmark's CPU reference arm.  The product never loads it.
//
// H|psi> comes from a caller callback with the reference's HPsiFunc contract (diago_david.h:57): X is the
// block base, HX the output of vector id_start.  S = I (spsi copies), as HamiltPW::sPsi for norm-conserving
// pseudopotentials.
#include <complex>
#include <cstring>
#include <exception>
#include <string>

#include "module_hsolver/diago_david.h"

namespace {
std::string g_err;
}

extern "C" {

typedef void (*ref_hpsi_cb)(void* user, const void* x, void* hx, int nvec, int dim, int id_start, int id_end);

const char* ref_last_error() { return g_err.c_str(); }

// psi (in/out): nband vectors of dim complex entries at psi + m*ldpsi; eig: nband doubles; returns 0 on
// success and the total iteration count in *iters.
int ref_david(int nband, int dim, int david_ndim, int ldpsi, const double* precond, ref_hpsi_cb cb, void* user,
              void* psi, double* eig, double thr, int maxiter, int ntry_max, int notconv_max, int* iters) {
    using T = std::complex<double>;
    try {
        hsolver::diag_comm_info comm(0, 1);
        hsolver::DiagoDavid<T, base_device::DEVICE_CPU> dav(precond, nband, dim, david_ndim, false, comm);
        auto hpsi = [cb, user](T* x, T* hx, const int nvec, const int d, const int i0, const int i1) {
            cb(user, x, hx, nvec, d, i0, i1);
        };
        auto spsi = [](T* in, T* out, const int nrow, const int npw, const int nbands) {
            for (int b = 0; b < nbands; ++b) std::memcpy(out + size_t(b) * nrow, in + size_t(b) * nrow, sizeof(T) * npw);
        };
        const int it = dav.diag(hpsi, spsi, ldpsi, static_cast<T*>(psi), eig, thr, maxiter, ntry_max, notconv_max);
        if (iters) *iters = it;
        g_err.clear();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

}  // extern "C"
