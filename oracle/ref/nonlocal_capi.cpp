// Test infrastructure (oracle): C entry point to the reference's own Nonlocal operator
// (module_hamilt_pw/hamilt_pwdft/operator_pw/nonlocal_pw.cpp: init + act, with add_nonlocal_pp and the
// nonlocal_pw_op / gemm_op / gemv_op CPU functors), compiled from its source against the cell and projector
// stand-ins in nl_stub/.  H psi += the nonlocal part for nbands bands of one k-point, npol = 1, spin 0:
// vkb (nkb x npwx, row-major: projector j at vkb + j * npwx), D as the reference's deeq(spin, iat, ih, jh)
// (nspin x natoms x nhm x nhm), psi and hpsi with band b at b * ld.  Returns 0, or 1 with the message of a
// WARNING_QUIT in err (err_len bytes).
#include <complex>
#include <cstring>
#include <exception>
#include <vector>

#include "module_hamilt_pw/hamilt_pwdft/operator_pw/nonlocal_pw.h"

extern "C" int ref_nonlocal_act(int ntype, const int* na, const int* nh, int nkb, int npwx, const void* vkb,
                                int nspin, int natoms, int nhm, const double* deeq, int nbands, int npw, int ld,
                                const void* psi, void* hpsi, char* err, int err_len) {
    try {
        std::vector<Atom> atoms(ntype);
        for (int it = 0; it < ntype; ++it) {
            atoms[it].na = na[it];
            atoms[it].ncpp.nh = nh[it];
        }
        UnitCell cell;
        cell.ntype = ntype;
        cell.atoms = atoms.data();
        pseudopot_cell_vnl pp;
        pp.nkb = nkb;
        pp.vkb.nr = nkb;
        pp.vkb.nc = npwx;
        pp.vkb_data = static_cast<std::complex<double>*>(const_cast<void*>(vkb));
        pp.deeq.b1 = nspin;
        pp.deeq.b2 = natoms;
        pp.deeq.b3 = nhm;
        pp.deeq.b4 = nhm;
        pp.deeq_data = const_cast<double*>(deeq);
        const int isk[1] = {0};
        hamilt::Nonlocal<hamilt::OperatorPW<std::complex<double>, base_device::DEVICE_CPU>> op(isk, &pp, &cell, nullptr);
        op.init(0);
        op.act(nbands, ld, 1, static_cast<const std::complex<double>*>(psi), static_cast<std::complex<double>*>(hpsi),
               npw);
        return 0;
    } catch (const std::exception& e) {
        if (err && err_len > 0) {
            std::strncpy(err, e.what(), size_t(err_len) - 1);
            err[err_len - 1] = 0;
        }
        return 1;
    }
}
