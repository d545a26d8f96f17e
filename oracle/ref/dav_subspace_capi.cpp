// Test infrastructure (oracle): a C entry point to the reference's own CPU Diago_DavSubspace
// (module_hsolver/diago_dav_subspace.cpp, compiled from the reference sources by oracle/build_ref.py), for the
// parity tests.  The product never loads it.
//
// H|psi> comes from a caller callback with the reference's HPsiFunc contract (diago_dav_subspace.h:31):
// X is the block base, HX the output of vector id_start.
#include <complex>
#include <exception>
#include <string>
#include <vector>

#include "module_hsolver/diago_dav_subspace.h"

namespace {
std::string g_err_ds;
}

extern "C" {

typedef void (*ref_hpsi_cb_ds)(void* user, const void* x, void* hx, int nvec, int dim, int id_start, int id_end);

const char* ref_dav_subspace_last_error() { return g_err_ds.c_str(); }

// psi (in/out): nband vectors of dim complex entries at psi + m*ldpsi; eig: nband doubles (in: the previous
// eigenvalues, out); precond: dim doubles (HSolverPW passes g2kin for this method, hsolver_pw.cpp:550-593);
// occupied: nband flags, or NULL for all bands occupied (as HSolverPW passes them); returns 0 on success and
// the total iteration count in *iters.
int ref_dav_subspace(int nband, int dim, int david_ndim, int ldpsi, const double* precond, ref_hpsi_cb_ds cb,
                     void* user, void* psi, double* eig, double thr, int maxiter, int need_subspace, int scf,
                     const int* occupied, int* iters) {
    using T = std::complex<double>;
    try {
        hsolver::diag_comm_info comm(0, 1);
        std::vector<double> pc(precond, precond + dim);
        hsolver::Diago_DavSubspace<T, base_device::DEVICE_CPU> dav(pc, nband, dim, david_ndim, thr, maxiter,
                                                                   need_subspace != 0, comm);
        auto hpsi = [cb, user](T* x, T* hx, const int nvec, const int d, const int i0, const int i1) {
            cb(user, x, hx, nvec, d, i0, i1);
        };
        std::vector<bool> occ(nband, true);
        if (occupied)
            for (int m = 0; m < nband; ++m) occ[m] = occupied[m] != 0;
        const int it = dav.diag(hpsi, static_cast<T*>(psi), ldpsi, eig, occ, scf != 0);
        if (iters) *iters = it;
        g_err_ds.clear();
        return 0;
    } catch (const std::exception& e) {
        g_err_ds = e.what();
        return 1;
    }
}

}  // extern "C"
