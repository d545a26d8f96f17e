// Allocation-free variant of the local part of H|psi> (kinetic term + V_eff through
// the stick/plane FFT), for callers that cannot allocate device memory at the
// point of the call.
//
// Who cannot allocate: code running inside a region captured into a CUDA graph
// (cudaMalloc is not a capturable operation and fails the capture), code whose
// device memory is handed out by a host framework's own pool or arena (a serving
// runtime, a solver that budgets HBM up front) and which may not grow it behind
// the framework's back, and code on paths that must not synchronise the device
// (cudaFree synchronises).  The regular entry point b200_hamilt_hpsi_part grows
// a per-handle stick buffer with cudaMalloc on first use; this one instead uses
// the fixed scratch array below.
//
// The scratch is a file-scope __device__ array of kNoAllocScratchBytes (32 MiB).
// Every GPU that loads this library holds it until the process exits.  Host code
// cannot use the array's name as a device address: on the host it names a
// host-side stand-in, so the device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, and cached.  The first call on
// each device performs that lookup; make that first call before any stream
// capture begins.
//
// All calls share the one array and it keeps the contents of the last call.
// Nothing in it needs to start at zero: the inverse z pass writes every stick
// element of a chunk before the plane pass and the forward z pass read it.
// Calls that overlap on the GPU (different streams or threads at the same time,
// on the same device) race on the array and give wrong results: serialise them.
//
// Bands are processed in chunks that fit the array; a grid whose single-band
// stick buffer (nst * nz complex values) exceeds the array is rejected with
// B200_STATUS_CAPACITY_ERROR.
#include <algorithm>
#include <mutex>

#include "../../include/abacus_b200.h"
#include "capi_handles.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double2)];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
void* noalloc_scratch_on_current_device() {
    int dev = -1;
    B200_CUDA(cudaGetDevice(&dev));
    B200_CHECK(dev >= 0 && dev < kMaxDevices, b200::kInvalidArgument, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_addr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            throw b200::Error(b200::kCudaError,
                              std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") + cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    return g_noalloc_addr[dev];
}

template <typename T, typename R>
void hpsi_local_noalloc(b200::Hamilt& H, int ik, int nb, int ld, const T* psi, T* hpsi, cudaStream_t s) {
    const b200::PWGrid& g = *H.grid;
    B200_CHECK(ik >= 0 && ik < int(g.kmaps.size()), b200::kInvalidArgument, "k-point index out of range");
    B200_CHECK(nb >= 0 && ld >= g.kmaps[ik].npw, b200::kInvalidArgument, "ld smaller than npwk or negative band count");
    B200_CHECK(H.has_veff, b200::kInvalidArgument, "V_eff not set");
    B200_CHECK(psi != nullptr && hpsi != nullptr, b200::kInvalidArgument, "NULL psi or hpsi");
    const size_t per_band = size_t(g.nst) * g.nz * sizeof(T);
    B200_CHECK(per_band <= kNoAllocScratchBytes, b200::kCapacityError,
               "one band's stick buffer (" + std::to_string(per_band) + " bytes) exceeds the " +
                   std::to_string(kNoAllocScratchBytes) + "-byte no-alloc scratch");
    if (nb == 0) return;
    T* sb = static_cast<T*>(noalloc_scratch_on_current_device());
    // bands per launch: what the scratch holds, and at most 65535 (the launches put bands on gridDim.y)
    const int chunk = int(std::min<size_t>(kNoAllocScratchBytes / per_band, 65535));
    const R* veff = H.veff_of<R>();
    const R* veffp = H.veff_perm_of<R>();
    for (int b0 = 0; b0 < nb; b0 += chunk) {
        const int nbc = nb - b0 < chunk ? nb - b0 : chunk;
        b200::launch_hpsi_local<T, R>(g, ik, veff, veffp, nbc, ld, psi + size_t(b0) * ld, hpsi + size_t(b0) * ld, sb,
                                      g.basis.tpiba2, 0, s);
    }
}

}  // namespace

extern "C" int b200_hamilt_hpsi_local_noalloc(b200_hamilt* h, int ik, int nbands, int ld, const void* psi_d,
                                              void* hpsi_d, void* stream) {
    try {
        B200_CHECK(h != nullptr && h->h, b200::kInvalidArgument, "NULL Hamiltonian handle");
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        if (h->h->precision == B200_PREC_FP64)
            hpsi_local_noalloc<double2, double>(*h->h, ik, nbands, ld, (const double2*)psi_d, (double2*)hpsi_d, s);
        else
            hpsi_local_noalloc<float2, float>(*h->h, ik, nbands, ld, (const float2*)psi_d, (float2*)hpsi_d, s);
        b200::set_last_error("");
        return B200_STATUS_OK;
    } catch (const b200::Error& e) {
        b200::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        b200::set_last_error(e.what());
        return B200_STATUS_INVALID_ARGUMENT;
    }
}
