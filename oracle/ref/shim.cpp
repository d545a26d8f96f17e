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
#include <complex>
#include <stdexcept>
#include <string>

#include "module_base/memory.h"
#include "module_base/module_device/device.h"
#include "module_base/parallel_reduce.h"
#include "module_base/tool_quit.h"
#include "module_base/tool_title.h"

namespace ModuleBase {
void WARNING_QUIT(const std::string& file, const std::string& description) {
    throw std::runtime_error(file + ": " + description);
}
void WARNING_QUIT(const std::string& file, const std::string& description, int) {
    throw std::runtime_error(file + ": " + description);
}
void TITLE(const std::string&, const std::string&, const bool) {}
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
