// Test infrastructure (oracle): stand-ins for the process-level services the reference's DiagoDavid
// links against, for a single-process CPU build.  Only the tests and the benchmark's CPU reference arm
// load the library built from this file; the product never does.
//
// * ModuleBase::WARNING_QUIT (module_base/tool_quit.h:49,57): the reference writes a log and exits; here
//   it throws, so a failure surfaces as an error status of the C entry point instead of ending the host.
// * ModuleBase::TITLE (module_base/tool_title.h:16-30): trace printing, off.
// * base_device::get_device_type<DEVICE_CPU> (module_base/module_device/device.h:25): the CPU tag.
// * Parallel_Reduce::reduce_pool (module_base/parallel_reduce.h:21-23): a sum over the processes of a pool;
//   with one process it leaves the data unchanged.
// * ModuleBase::Memory::record (module_base/memory.h): bookkeeping of allocated bytes, not kept here.
// * GlobalV::NPROC_IN_POOL (module_base/global_variable.h): processes in a pool, 1; GlobalV::NBANDS, the
//   band count the occupation code reads; GlobalV::ofs_warning, an unopened stream (warnings dropped).
// * ModuleBase::WARNING (module_base/tool_quit.h): a log line, dropped; CHECK_WARNING_QUIT throws when its
//   condition holds, as WARNING_QUIT.
// * DiagoIterAssist<T, CPU>::diagH_LAPACK (module_hsolver/diago_iter_assist.cpp): its body is the
//   reference's dngvd_op (generalised eigenproblem, all pairs, compiled from dngvd_op.cpp) and a copy of the
//   first nbands eigenvalues; restated here so that the rest of diago_iter_assist.cpp (the psi / Hamiltonian
//   layers) is not needed.
#include <complex>
#include <fstream>
#include <stdexcept>
#include <string>

#include "module_base/memory.h"
#include "module_base/module_device/device.h"
#include "module_base/parallel_reduce.h"
#include "module_base/tool_quit.h"
#include "module_base/tool_title.h"
#include "module_hsolver/diago_iter_assist.h"
#include "module_hsolver/kernels/dngvd_op.h"

#include <vector>

namespace ModuleBase {
void WARNING_QUIT(const std::string& file, const std::string& description) {
    throw std::runtime_error(file + ": " + description);
}
void WARNING_QUIT(const std::string& file, const std::string& description, int) {
    throw std::runtime_error(file + ": " + description);
}
void TITLE(const std::string&, const std::string&, const bool) {}
void WARNING(const std::string&, const std::string&) {}
void CHECK_WARNING_QUIT(const bool error_in, const std::string& file, const std::string& calculation,
                        const std::string& description) {
    if (error_in) throw std::runtime_error(file + " (" + calculation + "): " + description);
}
void Memory::record(const std::string&, const size_t&, const bool) {}
}  // namespace ModuleBase

namespace base_device {
template <> AbacusDevice_t get_device_type<DEVICE_CPU>(const DEVICE_CPU*) { return CpuDevice; }
}  // namespace base_device

namespace Parallel_Reduce {
template <> void reduce_pool<std::complex<double>>(std::complex<double>*, const int) {}
template <> void reduce_pool<std::complex<float>>(std::complex<float>*, const int) {}
template <> void reduce_pool<double>(double&) {}
template <> void reduce_pool<float>(float&) {}
}  // namespace Parallel_Reduce

namespace GlobalV {
int NPROC_IN_POOL = 1;
int NBANDS = 0;                 // set by the occupation entry point before each call
std::ofstream ofs_warning;      // never opened: warnings are dropped
}  // namespace GlobalV

namespace hsolver {
template <typename T, typename Device>
void DiagoIterAssist<T, Device>::diagH_LAPACK(const int nstart, const int nbands, const T* hcc, const T* scc,
                                              const int ldh, Real* e, T* vcc) {
    std::vector<Real> w(nstart, Real(0));
    dngvd_op<T, Device>()(nullptr, nstart, ldh, hcc, scc, w.data(), vcc);
    for (int i = 0; i < nbands; ++i) e[i] = w[i];
}
template void DiagoIterAssist<std::complex<double>, base_device::DEVICE_CPU>::diagH_LAPACK(
    int, int, const std::complex<double>*, const std::complex<double>*, int, double*, std::complex<double>*);
template void DiagoIterAssist<std::complex<float>, base_device::DEVICE_CPU>::diagH_LAPACK(
    int, int, const std::complex<float>*, const std::complex<float>*, int, float*, std::complex<float>*);
}  // namespace hsolver
