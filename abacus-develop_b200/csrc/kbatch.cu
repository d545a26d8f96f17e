// k-point batches: batched H|psi>, its capture into a CUDA graph, the band-chunk autotuner, and concurrent
// Davidson solves of many k-points (one stream and one H|psi> scratch per worker).
//
// ABACUS solves its k-points one after another inside a pool (HSolverPW::solve, hsolver_pw.cpp:240-270) and
// parallelises over k only across processes.  On one B200 the k-points of a pool are independent work that
// can share the device: their local H|psi> passes are launched together (one launch per pass for all k),
// and their Davidson solves run concurrently on separate streams.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <exception>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "capi_guard.h"
#include "../../include/abacus_b200.h"
#include "capi_handles.h"

struct b200_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~b200_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

namespace {

using b200::guarded;

void kbatch_call(b200_hamilt* h, int nk, const int* iks, int spin, int nb, int ld, void* const* psi, void* const* hpsi,
                 cudaStream_t s) {
    B200_CHECK(h && iks && psi && hpsi, b200::kInvalidArgument, "NULL argument");
    if (h->h->precision == B200_PREC_FP64)
        h->h->hpsi_kbatch<double2>(nk, iks, spin, nb, ld, reinterpret_cast<const double2* const*>(psi),
                                   reinterpret_cast<double2* const*>(hpsi), s);
    else
        h->h->hpsi_kbatch<float2>(nk, iks, spin, nb, ld, reinterpret_cast<const float2* const*>(psi),
                                  reinterpret_cast<float2* const*>(hpsi), s);
}

}  // namespace

extern "C" {

int b200_hamilt_hpsi_kbatch(b200_hamilt* h, int nk, const int* iks, int spin, int nbands, int ld, void* const* psi_d,
                            void* const* hpsi_d, void* stream) {
    return guarded([&] { kbatch_call(h, nk, iks, spin, nbands, ld, psi_d, hpsi_d, reinterpret_cast<cudaStream_t>(stream)); });
}

int b200_graph_capture_hpsi_kbatch(b200_hamilt* h, int nk, const int* iks, int spin, int nbands, int ld,
                                   void* const* psi_d, void* const* hpsi_d, void* stream, b200_graph** out) {
    return guarded([&] {
        B200_CHECK(out != nullptr, b200::kInvalidArgument, "NULL argument");
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        B200_CHECK(s != nullptr, b200::kInvalidArgument, "capture needs a non-default stream");
        // one eager call first: every workspace is allocated and every kernel attribute set before capture
        kbatch_call(h, nk, iks, spin, nbands, ld, psi_d, hpsi_d, s);
        B200_CUDA(cudaStreamSynchronize(s));
        auto g = std::make_unique<b200_graph>();
        B200_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            kbatch_call(h, nk, iks, spin, nbands, ld, psi_d, hpsi_d, s);
        } catch (...) {
            cudaGraph_t dead = nullptr;
            cudaStreamEndCapture(s, &dead);
            if (dead) cudaGraphDestroy(dead);
            throw;
        }
        B200_CUDA(cudaStreamEndCapture(s, &g->graph));
        B200_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
        *out = g.release();
    });
}

int b200_graph_launch(b200_graph* g, void* stream) {
    return guarded([&] {
        B200_CHECK(g && g->exec, b200::kInvalidArgument, "NULL graph");
        B200_CUDA(cudaGraphLaunch(g->exec, reinterpret_cast<cudaStream_t>(stream)));
    });
}

int b200_graph_destroy(b200_graph* g) {
    return guarded([&] { delete g; });
}

int b200_hamilt_autotune(b200_hamilt* h, int ik, int nbands, int ld, const void* psi_d, void* hpsi_d, void* stream,
                         int* best_chunk, int* best_variant) {
    return guarded([&] {
        B200_CHECK(h && psi_d && hpsi_d, b200::kInvalidArgument, "NULL argument");
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        b200::Hamilt& H = *h->h;
        b200::PWGrid& G = *H.grid;
        const bool f64 = H.precision == B200_PREC_FP64;
        int& variant = f64 ? G.plane_variant64 : G.plane_variant32;
        std::vector<int> cand = {1, 2, 4, 8, 16, 32, 64, 128};
        cand.push_back(nbands);
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        // plane-pass variants: only grids with the register transforms have a choice
        std::vector<int> vars = {variant};
        if (b200::plane_perm_supported(G)) {
            vars.clear();
            for (int v = 1; v <= b200::kPlaneVariants; ++v) vars.push_back(v);
        }
        cudaEvent_t e0, e1;
        B200_CUDA(cudaEventCreate(&e0));
        B200_CUDA(cudaEventCreate(&e1));
        float best = 1e30f;
        int best_c = 0, best_v = variant;
        const int saved_c = H.chunk_override, saved_v = variant;
        try {
            for (int v : vars) {
                variant = v;
                for (int c : cand) {
                    if (c > nbands) continue;
                    H.chunk_override = c;
                    auto run = [&] {
                        if (f64)
                            H.hpsi<double2>(ik, 0, nbands, ld, (const double2*)psi_d, (double2*)hpsi_d, 1, s);
                        else
                            H.hpsi<float2>(ik, 0, nbands, ld, (const float2*)psi_d, (float2*)hpsi_d, 1, s);
                    };
                    run();  // warm-up (allocates the stick buffer for this chunk size)
                    B200_CUDA(cudaEventRecord(e0, s));
                    for (int r = 0; r < 3; ++r) run();
                    B200_CUDA(cudaEventRecord(e1, s));
                    B200_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    B200_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    if (ms < best) {
                        best = ms;
                        best_c = c;
                        best_v = v;
                    }
                }
            }
        } catch (...) {
            H.chunk_override = saved_c;
            variant = saved_v;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        H.chunk_override = best_c > 0 ? best_c : saved_c;
        variant = best_v;
        if (best_chunk) *best_chunk = H.chunk_override;
        if (best_variant) *best_variant = variant;
    });
}

int b200_hamilt_set_band_chunk(b200_hamilt* h, int chunk) {
    return guarded([&] {
        B200_CHECK(h != nullptr, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(chunk >= 0, b200::kInvalidArgument, "band chunk must be >= 0");
        h->h->chunk_override = chunk;
    });
}

int b200_hamilt_set_plane_variant(b200_hamilt* h, int variant) {
    return guarded([&] {
        B200_CHECK(h != nullptr, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(variant >= 0 && variant <= b200::kPlaneVariants, b200::kInvalidArgument, "plane variant out of range");
        b200::PWGrid& G = *h->h->grid;
        (h->h->precision == B200_PREC_FP64 ? G.plane_variant64 : G.plane_variant32) = variant;
    });
}

int b200_hamilt_set_fp64_gemm(b200_hamilt* h, int mode, int nmods) {
    return guarded([&] {
        B200_CHECK(h != nullptr, b200::kInvalidArgument, "NULL argument");
        h->h->set_fp64_gemm(mode, nmods);
    });
}

int b200_solve_kpoints(b200_hamilt* h, int nk, const int* iks, int spin, int nband, int david_ndim, int precision,
                       const double* const* precond_d, void* const* psi_d, int ldpsi, double* eigenvalues,
                       double thr, int maxiter, int ntry_max, int notconv_max, int nworkers, int* iters) {
    return guarded([&] {
        B200_CHECK(h && iks && precond_d && psi_d && eigenvalues, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(nk >= 1 && nworkers >= 1, b200::kInvalidArgument, "need nk >= 1 and nworkers >= 1");
        b200::Hamilt* H = h->h.get();
        int dev = 0;
        B200_CUDA(cudaGetDevice(&dev));
        // one solver per worker, sized for the largest k-point and re-targeted to each k-point in turn: a solver
        // made and destroyed per k-point would allocate inside the loop, and its cudaFree would synchronise the
        // device under the other workers' solves
        int q_max = 0;
        for (int q = 0; q < nk; ++q) {
            B200_CHECK(iks[q] >= 0 && iks[q] < int(H->grid->kmaps.size()), b200::kInvalidArgument,
                       "k-point index out of range");
            if (H->grid->kmaps[iks[q]].npw > H->grid->kmaps[iks[q_max]].npw) q_max = q;
        }
        const int dim_max = H->grid->kmaps[iks[q_max]].npw;
        std::atomic<int> next{0};
        std::mutex err_mu;
        std::exception_ptr first_err;
        auto worker = [&]() {
            try {
                B200_CUDA(cudaSetDevice(dev));
                cudaStream_t s = nullptr;
                B200_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
                auto work = std::make_unique<b200::HpsiWork>();
                auto d = b200::make_david(nband, dim_max, david_ndim, precision, precond_d[q_max]);
                d->set_stream(s);
                for (int q = next.fetch_add(1); q < nk; q = next.fetch_add(1)) {
                    {
                        std::lock_guard<std::mutex> lk(err_mu);
                        if (first_err) break;
                    }
                    const int ik = iks[q];
                    const int dim = H->grid->kmaps[ik].npw;
                    d->retarget(dim, precond_d[q]);
                    b200::HpsiWork* W = work.get();
                    b200::HPsiDevice f64 = [H, W, ik, spin](const void* x, void* hx, int, int ld, int i0, int i1,
                                                            cudaStream_t st) {
                        H->hpsi<double2>(ik, spin, i1 - i0 + 1, ld, (const double2*)x + size_t(i0) * ld, (double2*)hx, 0,
                                         st, W);
                    };
                    b200::HPsiDevice f32 = [H, W, ik, spin](const void* x, void* hx, int, int ld, int i0, int i1,
                                                            cudaStream_t st) {
                        H->hpsi<float2>(ik, spin, i1 - i0 + 1, ld, (const float2*)x + size_t(i0) * ld, (float2*)hx, 0,
                                        st, W);
                    };
                    const int it = d->diag_hamilt(f64, f32, precision, ldpsi, psi_d[q], eigenvalues + size_t(q) * nband,
                                                  thr, maxiter, ntry_max, notconv_max);
                    if (iters) iters[q] = it;
                }
                B200_CUDA(cudaStreamSynchronize(s));
                d.reset();
                work.reset();
                cudaStreamDestroy(s);
            } catch (...) {
                std::lock_guard<std::mutex> lk(err_mu);
                if (!first_err) first_err = std::current_exception();
            }
        };
        const int nw = std::min(nworkers, nk);
        std::vector<std::thread> pool;
        for (int w = 0; w < nw; ++w) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
        if (first_err) std::rethrow_exception(first_err);
    });
}

}  // extern "C"
