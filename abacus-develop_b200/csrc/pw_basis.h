// Host-side plane-wave basis for one pool (one process, one GPU).
//
// Mirrors ModulePW::PW_Basis_K of ABACUS: FFT grid sizing (pw_init.cpp:24-140),
// the G sphere split into z-sticks ordered by ixy = x*ny + y
// (pw_distributeg.cpp:44-200, serial order of pw_distributeg_method1.cpp:84-97),
// the per-k sphere |k+G|^2 <= ecutwfc (pw_basis_k.cpp:118-168), gk2
// (pw_basis_k.cpp:189-265) and the box map ig2ixyz_k (pw_basis_k.cpp:319-344).
#pragma once
#include <cstdint>
#include <vector>

namespace b200 {

struct PWBasisK {
    // inputs
    double lat0 = 0.0;
    double latvec[9] = {0};   // rows are lattice vectors in units of lat0
    double ecutwfc = 0.0;
    double ecutrho = 0.0;
    int nks = 0;
    std::vector<double> kvec_d;  // nks*3
    // grid
    int nx = 0, ny = 0, nz = 0;
    double tpiba = 0.0, tpiba2 = 0.0, omega = 0.0;
    double G[9] = {0}, GGT[9] = {0};
    double gridecut_lat = 0.0, gk_ecut = 0.0, ggecut = 0.0;
    std::vector<double> kvec_c;  // nks*3 (units of tpiba)
    // sticks of the ggecut sphere
    int nst = 0;
    int npw = 0;                     // G vectors in the ggecut sphere
    std::vector<int> is2fftixy;      // nst: ixy = x*ny + y
    std::vector<int> ig2isz;         // npw: s*nz + z
    // per k
    std::vector<int> npwk;           // nks
    int npwk_max = 0;
    std::vector<int> igl2isz_k;      // nks*npwk_max
    std::vector<int> ig2ixyz_k;      // nks*npwk_max
    std::vector<double> gk2;         // nks*npwk_max (units of tpiba2)
    std::vector<double> gcar;        // nks*npwk_max*3 (units of tpiba)

    // Builds everything; nx_in <= 0 selects the reference's 2,3,5-smooth rule.
    // Returns 0 on success, nonzero on invalid input.
    int setup(double lat0_in, const double* latvec_in, double ecutwfc_in, double ecutrho_in,
              int nx_in, int ny_in, int nz_in, int nks_in, const double* kvec_d_in);
};

}  // namespace b200
