// Test infrastructure (oracle): a C entry point to the reference's own CPU DiagoBPCG
// (module_hsolver/diago_bpcg.cpp, compiled from the reference sources by oracle/build_ref.py), for the parity
// tests.  The product never loads it.
//
// DiagoBPCG::diag takes a Hamilt whose operator chain applies H to a psi::Psi (diago_bpcg.cpp:184-195
// calls hamilt_in->ops->hPsi with the all-band range); here the chain is one operator whose hPsi hands the
// bands of the range to a caller callback with the HPsiFunc contract (X the first band of the range, HX its
// output, vectors of nbasis entries).
#include <complex>
#include <exception>
#include <string>
#include <tuple>

#include "module_hamilt_general/hamilt.h"
#include "module_hamilt_general/operator.h"
#include "module_hsolver/diago_bpcg.h"
#include "module_hsolver/diago_iter_assist.h"
#include "module_psi/psi.h"

namespace {
std::string g_err_bp;
using T = std::complex<double>;
using Cpu = base_device::DEVICE_CPU;
typedef void (*ref_hpsi_cb_bp)(void* user, const void* x, void* hx, int nvec, int dim, int id_start, int id_end);

class CallbackOp : public hamilt::Operator<T, Cpu> {
  public:
    ref_hpsi_cb_bp cb = nullptr;
    void* user = nullptr;
    hpsi_info hPsi(hpsi_info& input) const override {
        const psi::Psi<T, Cpu>* p = std::get<0>(input);
        const std::tuple<const T*, int> r = p->to_range(std::get<1>(input));
        const int nb = std::get<1>(r);
        cb(user, std::get<0>(r), std::get<2>(input), nb, static_cast<int>(p->get_nbasis()), 0, nb - 1);
        return input;
    }
};

class CallbackHamilt : public hamilt::Hamilt<T, Cpu> {
  public:
    explicit CallbackHamilt(CallbackOp* op) { this->ops = op; }
};
}  // namespace

extern "C" {

const char* ref_bpcg_last_error() { return g_err_bp.c_str(); }

// psi (in/out): nband vectors of nbasis complex entries at psi + m*nbasis; eig: nband doubles (out);
// precond: nbasis doubles; scf_iter: DiagoIterAssist::SCF_ITER (1 = first SCF step: up to 6 nline
// iterations with a subspace diagonalisation every nline); ncalls: successive diag calls on the same
// psi (the reference's unit test makes three).  Returns 0 on success.
int ref_bpcg(int nband, int nbasis, const double* precond, ref_hpsi_cb_bp cb, void* user, void* psi, double* eig,
             int scf_iter, int ncalls) {
    try {
        hsolver::DiagoIterAssist<T, Cpu>::SCF_ITER = scf_iter;
        int ngk[1] = {nbasis};
        psi::Psi<T, Cpu> p(static_cast<T*>(psi), 1, nband, nbasis, ngk, true);
        p.fix_k(0);
        CallbackOp op;
        op.cb = cb;
        op.user = user;
        CallbackHamilt h(&op);
        hsolver::DiagoBPCG<T, Cpu> bpcg(precond);
        bpcg.init_iter(p);
        for (int c = 0; c < ncalls; ++c) bpcg.diag(&h, p, eig);
        h.ops = nullptr;
        g_err_bp.clear();
        return 0;
    } catch (const std::exception& e) {
        g_err_bp = e.what();
        return 1;
    }
}

}  // extern "C"
