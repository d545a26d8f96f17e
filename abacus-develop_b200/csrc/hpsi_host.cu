// H|psi> between host buffers: the bands go in pieces through three streams, so that the upload of
// piece p+1, the H|psi> of piece p and the download of piece p-1 overlap (PCIe is full duplex; with
// pinned host buffers each direction runs at link speed while the GPU computes).  No counterpart in the
// reference: its Operator::hPsi (module_hamilt_general/operator.cpp:39-88) works on device memory and the
// host <-> device copies are the caller's (psi is kept on the device).  This is the entry point a host
// program uses when psi lives in host memory.
#include <algorithm>
#include <vector>

#include "capi_guard.h"
#include "../../include/abacus_b200.h"
#include "capi_handles.h"

namespace {
using b200::guarded;
}  // namespace

extern "C" int b200_hamilt_hpsi_host(b200_hamilt* h, int ik, int spin, int nbands, int ld, const void* psi_host,
                                     void* hpsi_host, void* psi_dev, void* hpsi_dev, int npieces, void* stream) {
    return guarded([&] {
        B200_CHECK(h && psi_host && hpsi_host && psi_dev && hpsi_dev, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(nbands >= 1 && ld >= 1 && npieces >= 1, b200::kInvalidArgument, "need nbands, ld, npieces >= 1");
        b200::Hamilt* H = h->h.get();
        const int P = std::min(npieces, nbands);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (!h->pipe) h->pipe = std::make_unique<HostPipe>();
        HostPipe& pp = *h->pipe;
        if (!pp.up) B200_CUDA(cudaStreamCreateWithFlags(&pp.up, cudaStreamNonBlocking));
        if (!pp.down) B200_CUDA(cudaStreamCreateWithFlags(&pp.down, cudaStreamNonBlocking));
        while (int(pp.ev.size()) < 2 * P + 2) {
            cudaEvent_t e;
            B200_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            pp.ev.push_back(e);
        }
        const bool f64 = H->precision == B200_PREC_FP64;
        const size_t row = size_t(ld) * (f64 ? sizeof(double2) : sizeof(float2));  // bytes of one band
        // piece boundaries: the first and the last piece are half as large as the others (the first upload
        // and the last download are the two copies nothing overlaps), so the P pieces weigh 1, 2, ..., 2, 1
        // (two pieces: 1, 1).  Larger middle pieces lengthen the pipeline: the upload of piece 1 and the
        // download of piece P-2 are on its critical path beside them (B200: 16, 64, 64, 16 bands took 5.1 ms
        // where 16, 32, 32, 32, 32, 16 took 4.3).  Every piece keeps at least one band (P <= nbands).
        std::vector<int> bnd(P + 1, 0);
        const long total = 2L * (P - 1);  // sum of the weights
        for (int p = 1; p < P; ++p) bnd[p] = int(long(nbands) * (2L * p - 1) / total);
        bnd[P] = nbands;
        for (int p = 1; p < P; ++p) bnd[p] = std::max(bnd[p], bnd[p - 1] + 1);
        for (int p = P - 1; p >= 1; --p) bnd[p] = std::min(bnd[p], bnd[p + 1] - 1);
        auto piece = [&](int p, int& b0, int& b1) {
            b0 = bnd[p];
            b1 = bnd[p + 1];
        };
        // the copies start after the work already queued on the caller's stream (which may still use the
        // device buffers)
        cudaEvent_t ev_start = pp.ev[2 * P], ev_done = pp.ev[2 * P + 1];
        B200_CUDA(cudaEventRecord(ev_start, s));
        B200_CUDA(cudaStreamWaitEvent(pp.up, ev_start, 0));
        B200_CUDA(cudaStreamWaitEvent(pp.down, ev_start, 0));
        for (int p = 0; p < P; ++p) {
            int b0, b1;
            piece(p, b0, b1);
            B200_CUDA(cudaMemcpyAsync(static_cast<char*>(psi_dev) + b0 * row, static_cast<const char*>(psi_host) + b0 * row,
                                      (b1 - b0) * row, cudaMemcpyHostToDevice, pp.up));
            B200_CUDA(cudaEventRecord(pp.ev[p], pp.up));
        }
        for (int p = 0; p < P; ++p) {
            int b0, b1;
            piece(p, b0, b1);
            B200_CUDA(cudaStreamWaitEvent(s, pp.ev[p], 0));
            if (f64)
                H->hpsi<double2>(ik, spin, b1 - b0, ld, static_cast<const double2*>(psi_dev) + size_t(b0) * ld,
                                 static_cast<double2*>(hpsi_dev) + size_t(b0) * ld, 0, s);
            else
                H->hpsi<float2>(ik, spin, b1 - b0, ld, static_cast<const float2*>(psi_dev) + size_t(b0) * ld,
                                static_cast<float2*>(hpsi_dev) + size_t(b0) * ld, 0, s);
            B200_CUDA(cudaEventRecord(pp.ev[P + p], s));
            B200_CUDA(cudaStreamWaitEvent(pp.down, pp.ev[P + p], 0));
            B200_CUDA(cudaMemcpyAsync(static_cast<char*>(hpsi_host) + b0 * row, static_cast<const char*>(hpsi_dev) + b0 * row,
                                      (b1 - b0) * row, cudaMemcpyDeviceToHost, pp.down));
        }
        // the caller's stream completes after the last download
        B200_CUDA(cudaEventRecord(ev_done, pp.down));
        B200_CUDA(cudaStreamWaitEvent(s, ev_done, 0));
    });
}
