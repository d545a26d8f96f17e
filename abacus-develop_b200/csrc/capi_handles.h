// Definitions of the opaque C-ABI handles (shared by the C-ABI translation units).
#pragma once
#include <memory>
#include <vector>

#include "bpcg.h"
#include "dav_subspace.h"
#include "david.h"
#include "david_batch.h"
#include "hamilt.h"
#include "pw_grid.h"

struct b200_pw_basis {
    b200::PWGrid grid;
    b200::DeviceArray<double2> aux64;
    b200::DeviceArray<float2> aux32;
    b200::DeviceArray<double2> rho_box64;  // psi(r) of one band (psi -> rho, generic grids)
    b200::DeviceArray<float2> rho_box32;
    b200::DeviceArray<double2> rho_sb64;   // psi -> rho on the register transforms: stick buffer of a chunk,
    b200::DeviceArray<float2> rho_sb32;    // partial rho planes, band weights
    b200::DeviceArray<double> rho_ws64, rho_w;
    b200::DeviceArray<float> rho_ws32;
};
// copy streams and events of b200_hamilt_hpsi_host, made at its first use and kept with the handle
struct HostPipe {
    cudaStream_t up = nullptr, down = nullptr;
    std::vector<cudaEvent_t> ev;
    ~HostPipe() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        if (up) cudaStreamDestroy(up);
        if (down) cudaStreamDestroy(down);
    }
};
// the lock-step k-point solver of b200_solve_kpoints_batched, kept with the handle between calls of the same
// shape (k-point capacity, bands, subspace, plane-wave capacity, precision, stream) so repeated solves allocate
// nothing
struct KBatchSolverCache {
    std::unique_ptr<b200::DavidBatchSolver, void (*)(b200::DavidBatchSolver*)> solver{nullptr, nullptr};
    int cap = 0, nband = 0, ndim = 0, dim_cap = 0, precision = -1;
    cudaStream_t stream = nullptr;
};
struct b200_hamilt {
    std::unique_ptr<b200::Hamilt> h;
    std::unique_ptr<HostPipe> pipe;
    KBatchSolverCache kbatch;
};
struct b200_david {
    std::unique_ptr<b200::DavidBase> d;
    b200::HpsiWork work;  // H|psi> scratch used when the solver applies a Hamiltonian handle
};
struct b200_dav_subspace {
    std::unique_ptr<b200::DavSubspaceBase> d;
    b200::HpsiWork work;  // H|psi> scratch used when the solver applies a Hamiltonian handle
};
struct b200_bpcg {
    std::unique_ptr<b200::BpcgBase> d;
    b200::HpsiWork work;  // H|psi> scratch used when the solver applies a Hamiltonian handle
};
