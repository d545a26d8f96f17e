// Serving loop for non-self-consistent band solves (a resident cell's V_eff, D and projectors, one of its
// k-points, nbands), with continuous admission under an HBM budget.
//
// The reference solves the k-points of an NSCF run one after another (ESolver_KS_PW::nscf ->
// HSolverPW::solve, hsolver_pw.cpp:212-299); here independent requests arrive at any time and run
// concurrently on one GPU:
//  * cells stay resident: their Hamiltonian handles hold V_eff, D and the projectors of every k-point
//    of the cell (built once, on the device, by getvnl);
//  * each request needs a solver slot: a Davidson solver (mixed or FP64) sized for the cell's largest
//    k-point and the request's band count, the start / result vectors and an H|psi> scratch.  Slots are
//    pooled and re-targeted to the request's k-point, so the steady state allocates nothing (cudaFree
//    would synchronise the device and stall every other request in flight);
//  * admission is first come, first served within a cell: a worker that falls idle takes the oldest queued
//    request whose cell is below its in-flight cap and whose slot is pooled or fits in the HBM budget (idle
//    slots of other shapes are released to make room).  The per-cell caps keep small requests from waiting
//    behind large ones and bound how many large solves share the device at once;
//  * every slot owns a non-blocking stream, so admitted requests overlap on the device; its priority
//    follows the cell's size (smallest cell highest), so short solves are not queued behind the blocks of a
//    large cell's kernels.  A slot keeps its stream for life, whichever worker runs it.
// A request's result depends only on (cell, k-point, nbands, thr, precision, seed): the start vectors come
// from a counter-based generator keyed by the seed, each solve starts from a zeroed subspace, and no
// kernel's result depends on what else runs.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "capi_guard.h"
#include "../../include/abacus_b200.h"
#include "capi_handles.h"

namespace b200 {
namespace {

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// psi[b*ld + g] = (complex normal)(seed, b, g) / (1 + |k+G|^2) for g < npw, 0 for npw <= g < ld
__global__ void k_init_guess(int nb, int npw, int ld, const double* __restrict__ gk2, double tpiba2,
                             unsigned long long seed, double2* __restrict__ psi) {
    const long n = long(nb) * ld;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int b = int(i / ld), g = int(i - long(b) * ld);
        if (g >= npw) {
            psi[i] = make_double2(0.0, 0.0);
            continue;
        }
        const unsigned long long key = splitmix64(seed) ^ ((unsigned long long)b << 32 | (unsigned)g);
        const unsigned long long r1 = splitmix64(key), r2 = splitmix64(key ^ 0xD1B54A32D192ED03ull);
        const double u1 = (double(r1 >> 11) + 0.5) * 0x1.0p-53, u2 = double(r2 >> 11) * 0x1.0p-53;
        const double rad = sqrt(-2.0 * log(u1));
        double sp, cp;
        sincospi(2.0 * u2, &sp, &cp);
        const double w = 1.0 / (1.0 + gk2[g] * tpiba2);
        psi[i] = make_double2(rad * cp * w, rad * sp * w);
    }
}

double now_s(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

struct ServeCell {
    b200_hamilt* h;
    int dim_max, npwx, nks, nkb, kmax;
    int max_inflight, inflight;
};

// a solver slot's own stream, destroyed after everything else in the slot (declared first)
struct SlotStream {
    cudaStream_t s = nullptr;
    ~SlotStream() {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
};

struct Slot {
    SlotStream stream;  // every request on this slot runs on it: start vectors, solve, H|psi>
    int cell = 0, nbands = 0, precision = 0, priority = 0;
    std::unique_ptr<DavidBase> dav;
    DeviceArray<double2> psi;
    std::unique_ptr<HpsiWork> work;
    size_t bytes = 0;
    unsigned long long last_used = 0;
};

struct Request {
    long long id = 0;
    int cell = 0, ik = 0, nbands = 0, precision = 0, maxiter = 0;
    double thr = 0;
    unsigned long long seed = 0;
    double* eig_out = nullptr;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int iters = 0, status = 0, iters_low = 0;
    std::string err;
};

using SlotKey = std::tuple<int, int, int>;  // cell, nbands, precision

}  // namespace

class Server {
  public:
    Server(size_t budget, int nworkers, int david_ndim) : budget_(budget), ndim_(david_ndim) {
        B200_CHECK(nworkers >= 1 && nworkers <= 64, kInvalidArgument, "1..64 workers");
        B200_CHECK(david_ndim >= 2, kInvalidArgument, "david_ndim must be at least 2");
        B200_CUDA(cudaGetDevice(&dev_));
        t0_ = std::chrono::steady_clock::now();
        for (int w = 0; w < nworkers; ++w) workers_.emplace_back([this, w] { worker(w); });
    }
    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_work_.notify_all();
        for (auto& t : workers_) t.join();
        free_.clear();
    }

    int add_cell(b200_hamilt* h, int max_inflight) {
        B200_CHECK(h != nullptr, kInvalidArgument, "NULL Hamiltonian");
        const PWGrid& g = *h->h->grid;
        B200_CHECK(h->h->has_veff, kInvalidArgument, "cell without V_eff");
        B200_CHECK(max_inflight >= 1, kInvalidArgument, "max_inflight must be at least 1");
        ServeCell c{h, 0, g.basis.npwk_max, g.basis.nks, 0, 0, max_inflight, 0};
        for (int ik = 0; ik < c.nks; ++ik) {
            if (g.kmaps[ik].npw > c.dim_max) {
                c.dim_max = g.kmaps[ik].npw;
                c.kmax = ik;
            }
            c.nkb = std::max(c.nkb, h->h->nl[ik].nkb);
        }
        std::lock_guard<std::mutex> lk(mu_);
        cells_.push_back(c);
        svc_mean_.push_back(0.0);
        return int(cells_.size()) - 1;
    }

    long long submit(int cell, int ik, int nbands, int precision, double thr, int maxiter, unsigned long long seed,
                     double* eig_out) {
        auto r = std::make_unique<Request>();
        std::lock_guard<std::mutex> lk(mu_);
        B200_CHECK(cell >= 0 && cell < int(cells_.size()), kInvalidArgument, "unknown cell");
        const ServeCell& c = cells_[cell];
        B200_CHECK(ik >= 0 && ik < c.nks, kInvalidArgument, "k-point index out of range");
        B200_CHECK(nbands >= 1 && ndim_ * nbands < c.h->h->grid->kmaps[ik].npw, kInvalidArgument,
                   "need 1 <= nbands and david_ndim*nbands < npwk");
        B200_CHECK(precision == B200_PREC_FP64 || precision == B200_PREC_MIXED, kInvalidArgument, "bad precision");
        B200_CHECK(eig_out != nullptr, kInvalidArgument, "NULL eigenvalue buffer");
        B200_CHECK(maxiter >= 1, kInvalidArgument, "maxiter must be positive");
        r->id = next_id_++;
        r->cell = cell;
        r->ik = ik;
        r->nbands = nbands;
        r->precision = precision;
        r->thr = thr;
        r->maxiter = maxiter;
        r->seed = seed;
        r->eig_out = eig_out;
        r->t_submit = now_s(t0_);
        Request* p = r.get();
        reqs_[p->id] = std::move(r);
        if (slot_bytes(cell, nbands, precision) > budget_) {
            p->status = kCapacityError;
            p->err = "request needs more device memory than the whole budget";
            p->t_admit = p->t_done = p->t_submit;
            done_.push_back(p);
            cv_done_.notify_all();
        } else {
            queue_.push_back(p);
            // every worker re-checks: an express worker may not take this request while another could
            cv_work_.notify_all();
        }
        return p->id;
    }

    // Completed requests not yet reported; with wait != 0 blocks until one is available or none is
    // outstanding.
    int poll(int max_out, int wait, long long* ids, int* status, double* t_submit, double* t_admit, double* t_done,
             int* iters, int* iters_low) {
        std::unique_lock<std::mutex> lk(mu_);
        if (wait) cv_done_.wait(lk, [&] { return !done_.empty() || outstanding() == 0; });
        int n = 0;
        while (n < max_out && !done_.empty()) {
            Request* r = done_.front();
            done_.pop_front();
            ids[n] = r->id;
            status[n] = r->status;
            t_submit[n] = r->t_submit;
            t_admit[n] = r->t_admit;
            t_done[n] = r->t_done;
            iters[n] = r->iters;
            iters_low[n] = r->iters_low;
            if (r->status != 0) set_last_error(r->err);
            reqs_.erase(r->id);
            ++n;
        }
        return n;
    }

    void drain() {
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] { return queue_.empty() && inflight_ == 0; });
    }

    void set_policy(int policy, double shed_factor) {
        B200_CHECK(policy == 0 || policy == 1, kInvalidArgument, "policy must be 0 (oldest first) or 1 (response ratio)");
        B200_CHECK(shed_factor >= 0, kInvalidArgument, "shed_factor must be >= 0");
        std::lock_guard<std::mutex> lk(mu_);
        policy_ = policy;
        shed_factor_ = shed_factor;
    }
    long long shed_count() {
        std::lock_guard<std::mutex> lk(mu_);
        return shed_count_;
    }
    // workers 0 .. n-1 take only requests of cells whose mean service time is at most max_service_s (cells
    // not yet timed included), so that short solves never wait behind a full set of long ones
    void set_express(int n, double max_service_s) {
        B200_CHECK(n >= 0 && n < int(workers_.size()), kInvalidArgument, "express workers: 0 .. nworkers-1");
        B200_CHECK(max_service_s >= 0, kInvalidArgument, "express service bound must be >= 0");
        {
            std::lock_guard<std::mutex> lk(mu_);
            n_express_ = n;
            express_s_ = max_service_s;
        }
        cv_work_.notify_all();
    }

    void stats(double* out) {
        std::lock_guard<std::mutex> lk(mu_);
        out[0] = double(pool_bytes_);
        out[1] = double(peak_bytes_);
        out[2] = double(peak_inflight_);
        out[3] = double(slots_created_);
        out[4] = double(slots_evicted_);
        out[5] = now_s(t0_);
    }

  private:
    size_t outstanding() const { return queue_.size() + size_t(inflight_); }

    // device bytes of one solver slot: Davidson buffers (FP64 engine, plus the FP32 engine when mixed),
    // start vectors, and the H|psi> scratch (stick-buffer chunk of at most ~48 MB, becp / ps)
    size_t slot_bytes(int cell, int nb, int precision) const {
        const ServeCell& c = cells_[cell];
        const size_t nbx = size_t(ndim_) * nb, d = size_t(c.dim_max), d32 = d + (d & 1);
        auto engine = [&](size_t elem, size_t ld) {
            return (2 * nbx * ld + size_t(nb) * ld + 2 * nbx * nbx + 3 * (nbx + 1) * nb + size_t(nb + 1) * (nb + 1)) *
                       elem +
                   (2 * nbx * nbx + 3 * size_t(nb + 1) * (nb + 1)) * 16 + (size_t(8) << 20);
        };
        size_t b = engine(16, d) + size_t(nb) * c.npwx * 16;
        // the FP32 engine also reserves its tensor-core GEMM workspaces (split-K tiles, pre-split B)
        if (precision == B200_PREC_MIXED)
            b += engine(8, d32) + size_t(nb) * c.npwx * 8 + size_t(16) * 2 * nb * nbx * 4 + 2 * (nbx + 1) * nb * 8;
        const PWGrid& g = *c.h->h->grid;
        const size_t per_band = size_t(g.nst) * g.nz * 16;
        b += std::max(per_band, std::min(per_band * nb, size_t(48) << 20)) + per_band;
        b += size_t(c.nkb + 1) * nb * 16 * 4 + (size_t(16) << 20);
        // FP64 projector products on the int8 tensor cores: psi residues (2 real rows per band, one byte per
        // modulus and real entry) and the per-modulus product residues of H psi
        if (c.h->h->fp64_gemm != 0) b += size_t(c.h->h->oz_mods) * nb * (size_t(4) * c.npwx + 2 * size_t(c.npwx + 16));
        return b;
    }

    // The next request to run.  For each cell only its oldest queued request is considered (first come, first
    // served within a cell); among those whose cell is below its cap and whose slot can be had: policy 0 the
    // oldest, policy 1 the highest response ratio (wait + S_c) / S_c (S_c: running mean service time of the
    // cell; a cell not yet timed counts as the shortest).  With shedding on, requests that waited past
    // shed_factor * S_c are completed as shed first.
    std::deque<Request*>::iterator next_admissible_locked(bool express) {
        const double now = now_s(t0_);
        if (shed_factor_ > 0) {
            bool shed = false;
            for (auto it = queue_.begin(); it != queue_.end();) {
                Request* r = *it;
                const double sc = svc_mean_[r->cell];
                if (sc > 0 && now - r->t_submit > shed_factor_ * sc) {
                    r->status = kShed;
                    r->err = "waited past the cell's admission bound";
                    r->t_admit = r->t_done = now;
                    done_.push_back(r);
                    ++shed_count_;
                    it = queue_.erase(it);
                    shed = true;
                } else {
                    ++it;
                }
            }
            if (shed) cv_done_.notify_all();
        }
        std::vector<char> seen(cells_.size(), 0);
        auto best = queue_.end();
        double best_key = -1e300;
        for (auto it = queue_.begin(); it != queue_.end(); ++it) {
            const int c = (*it)->cell;
            if (seen[c]) continue;
            seen[c] = 1;
            if (express && svc_mean_[c] > express_s_) continue;
            if (!(cells_[c].inflight < cells_[c].max_inflight && can_admit_locked(**it))) continue;
            if (policy_ == 0) return it;  // the queue is in arrival order: the first admissible one is the oldest
            const double sc = svc_mean_[c];
            const double key = sc > 0 ? (now - (*it)->t_submit + sc) / sc : 1e300;
            if (key > best_key) {
                best_key = key;
                best = it;
            }
        }
        return best;
    }

    bool can_admit_locked(const Request& r) const {
        const SlotKey key{r.cell, r.nbands, r.precision};
        if (free_.count(key)) return true;
        const size_t need = slot_bytes(r.cell, r.nbands, r.precision);
        if (pool_bytes_ + need <= budget_) return true;
        size_t idle = 0;
        for (auto& kv : free_) idle += kv.second->bytes;
        return pool_bytes_ - idle + need <= budget_;
    }

    // under the lock: a pooled slot, or the room for a new one (reserved in pool_bytes_); idle slots
    // evicted to make room are moved to `victims` and released outside the lock
    std::unique_ptr<Slot> take_slot_locked(const Request& r, size_t& reserve,
                                           std::vector<std::unique_ptr<Slot>>& victims) {
        const SlotKey key{r.cell, r.nbands, r.precision};
        auto it = free_.find(key);
        if (it != free_.end()) {
            std::unique_ptr<Slot> s = std::move(it->second);
            free_.erase(it);
            reserve = 0;
            return s;
        }
        const size_t need = slot_bytes(r.cell, r.nbands, r.precision);
        while (pool_bytes_ + need > budget_ && !free_.empty()) {
            auto lru = free_.begin();
            for (auto i = free_.begin(); i != free_.end(); ++i)
                if (i->second->last_used < lru->second->last_used) lru = i;
            pool_bytes_ -= lru->second->bytes;
            victims.push_back(std::move(lru->second));
            free_.erase(lru);
            ++slots_evicted_;
        }
        pool_bytes_ += need;
        peak_bytes_ = std::max(peak_bytes_, pool_bytes_);
        reserve = need;
        return nullptr;
    }

    // stream priority of a cell: smaller cells (fewer plane waves) run at higher priority, so the block
    // scheduler dispatches their short kernels as soon as blocks of a larger cell's kernels retire instead of
    // after them; levels spread over the device's range by the cell's rank among the resident cells
    int priority_locked(int cell) const {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) return 0;
        int rank = 0, n = 0;
        std::vector<int> sizes;
        for (const ServeCell& c : cells_) sizes.push_back(c.dim_max);
        std::sort(sizes.begin(), sizes.end());
        sizes.erase(std::unique(sizes.begin(), sizes.end()), sizes.end());
        n = int(sizes.size());
        rank = int(std::lower_bound(sizes.begin(), sizes.end(), cells_[cell].dim_max) - sizes.begin());
        if (n <= 1) return least;
        return greatest + (least - greatest) * rank / (n - 1);
    }

    std::unique_ptr<Slot> make_slot(const Request& r, const ServeCell& c, int priority) {
        auto slot = std::make_unique<Slot>();
        B200_CUDA(cudaStreamCreateWithPriority(&slot->stream.s, cudaStreamNonBlocking, priority));
        slot->priority = priority;
        slot->cell = r.cell;
        slot->nbands = r.nbands;
        slot->precision = r.precision;
        slot->dav = make_david(r.nbands, c.dim_max, ndim_, r.precision, c.h->h->grid->kmaps[c.kmax].precond.ptr);
        slot->dav->set_stream(slot->stream.s);
        slot->psi.resize(size_t(r.nbands) * c.npwx);
        slot->work = std::make_unique<HpsiWork>();
        slot->bytes = slot_bytes(r.cell, r.nbands, r.precision);
        return slot;
    }

    void run(Request& r, const ServeCell& c, Slot& slot) {
        cudaStream_t s = slot.stream.s;
        Hamilt* H = c.h->h.get();
        const KMap& km = H->grid->kmaps[r.ik];
        slot.dav->retarget(km.npw, km.precond.ptr);
        const long n = long(r.nbands) * c.npwx;
        k_init_guess<<<int(std::min<long>((n + 255) / 256, 148 * 16)), 256, 0, s>>>(r.nbands, km.npw, c.npwx, km.gk2.ptr,
                                                                                H->grid->basis.tpiba2, r.seed,
                                                                                slot.psi.ptr);
        note_launch();
        B200_CUDA(cudaGetLastError());
        HpsiWork* W = slot.work.get();
        const int ik = r.ik;
        HPsiDevice f64 = [H, W, ik](const void* x, void* hx, int, int ld, int i0, int i1, cudaStream_t st) {
            H->hpsi<double2>(ik, 0, i1 - i0 + 1, ld, (const double2*)x + size_t(i0) * ld, (double2*)hx, 0, st, W);
        };
        HPsiDevice f32 = [H, W, ik](const void* x, void* hx, int, int ld, int i0, int i1, cudaStream_t st) {
            H->hpsi<float2>(ik, 0, i1 - i0 + 1, ld, (const float2*)x + size_t(i0) * ld, (float2*)hx, 0, st, W);
        };
        r.iters = slot.dav->diag_hamilt(f64, f32, r.precision, c.npwx, slot.psi.ptr, r.eig_out, r.thr, r.maxiter, 5, 0);
        r.iters_low = slot.dav->stats().iters_low;
        if (W->tcw.err.ptr) {
            const int e = W->tcw.read_error(s);
            B200_CHECK(e == 0, kCudaError, "tensor-core GEMM wait ran out in H|psi> (error word " + std::to_string(e) + ")");
        }
        B200_CUDA(cudaStreamSynchronize(s));
    }

    void worker(int id) {
        cudaSetDevice(dev_);
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            std::deque<Request*>::iterator pick;
            cv_work_.wait(lk, [&] {
                if (stop_) return true;
                pick = next_admissible_locked(id < n_express_);
                return pick != queue_.end();
            });
            if (stop_) break;
            Request* r = *pick;
            queue_.erase(pick);
            ++cells_[r->cell].inflight;
            size_t reserve = 0;
            std::vector<std::unique_ptr<Slot>> victims;
            std::unique_ptr<Slot> slot = take_slot_locked(*r, reserve, victims);
            const ServeCell cell = cells_[r->cell];  // a copy: add_cell may grow cells_ while this request runs
            const int priority = slot ? slot->priority : priority_locked(r->cell);
            ++inflight_;
            peak_inflight_ = std::max(peak_inflight_, inflight_);
            r->t_admit = now_s(t0_);
            lk.unlock();
            victims.clear();  // frees idle slots of other shapes (outside the lock)
            try {
                if (!slot) {
                    slot = make_slot(*r, cell, priority);
                    std::lock_guard<std::mutex> g(mu_);
                    ++slots_created_;
                }
                run(*r, cell, *slot);
                r->status = 0;
            } catch (const Error& e) {
                r->status = e.code;
                r->err = e.what();
                if (slot && slot->stream.s) cudaStreamSynchronize(slot->stream.s);
            } catch (const std::exception& e) {
                r->status = kInvalidArgument;
                r->err = e.what();
                if (slot && slot->stream.s) cudaStreamSynchronize(slot->stream.s);
            }
            r->t_done = now_s(t0_);
            lk.lock();
            if (r->status == 0) {  // running mean of the cell's service time (the last 16 requests' weight)
                double& m = svc_mean_[r->cell];
                const double svc = r->t_done - r->t_admit;
                m = m > 0 ? m + (svc - m) / 16.0 : svc;
            }
            if (slot) {
                slot->last_used = ++use_clock_;
                free_.emplace(SlotKey{slot->cell, slot->nbands, slot->precision}, std::move(slot));
            } else if (reserve) {
                pool_bytes_ -= reserve;  // the slot could not be made
            }
            --inflight_;
            --cells_[r->cell].inflight;
            done_.push_back(r);
            cv_done_.notify_all();
            cv_work_.notify_all();
        }
        lk.unlock();
    }

    size_t budget_;
    int ndim_;
    int policy_ = 0;
    double shed_factor_ = 0;
    int n_express_ = 0;
    double express_s_ = 0;
    long long shed_count_ = 0;
    std::vector<double> svc_mean_;  // per cell
    int dev_ = 0;
    std::chrono::steady_clock::time_point t0_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::vector<ServeCell> cells_;
    std::deque<Request*> queue_;
    std::deque<Request*> done_;
    std::unordered_map<long long, std::unique_ptr<Request>> reqs_;
    std::multimap<SlotKey, std::unique_ptr<Slot>> free_;
    size_t pool_bytes_ = 0, peak_bytes_ = 0;
    int inflight_ = 0, peak_inflight_ = 0;
    long long next_id_ = 1, slots_created_ = 0, slots_evicted_ = 0;
    unsigned long long use_clock_ = 0;
    bool stop_ = false;
    std::vector<std::thread> workers_;
};

}  // namespace b200

struct b200_server {
    std::unique_ptr<b200::Server> s;
};

namespace {
using b200::guarded;
}  // namespace

extern "C" {

int b200_server_create(unsigned long long hbm_budget_bytes, int nworkers, int david_ndim, b200_server** out) {
    return guarded([&] {
        B200_CHECK(out != nullptr, b200::kInvalidArgument, "NULL argument");
        auto p = std::make_unique<b200_server>();
        p->s = std::make_unique<b200::Server>(size_t(hbm_budget_bytes), nworkers, david_ndim);
        *out = p.release();
    });
}

int b200_server_destroy(b200_server* s) {
    return guarded([&] { delete s; });
}

int b200_server_add_cell(b200_server* s, b200_hamilt* h, int max_inflight, int* cell_id) {
    return guarded([&] {
        B200_CHECK(s && h && cell_id, b200::kInvalidArgument, "NULL argument");
        *cell_id = s->s->add_cell(h, max_inflight);
    });
}

int b200_server_submit(b200_server* s, int cell, int ik, int nbands, int precision, double thr, int maxiter,
                       unsigned long long seed, double* eig_out, long long* req_id) {
    return guarded([&] {
        B200_CHECK(s && req_id, b200::kInvalidArgument, "NULL argument");
        *req_id = s->s->submit(cell, ik, nbands, precision, thr, maxiter, seed, eig_out);
    });
}

int b200_server_poll(b200_server* s, int max_out, int wait, long long* ids, int* status, double* t_submit,
                     double* t_admit, double* t_done, int* iters, int* iters_low, int* n_out) {
    try {
        B200_CHECK(s && ids && status && t_submit && t_admit && t_done && iters && iters_low && n_out,
                   b200::kInvalidArgument, "NULL argument");
        b200::set_last_error("");
        *n_out = s->s->poll(max_out, wait, ids, status, t_submit, t_admit, t_done, iters, iters_low);
        return B200_STATUS_OK;
    } catch (const b200::Error& e) {
        b200::set_last_error(e.what());
        return e.code;
    }
}

int b200_server_drain(b200_server* s) {
    return guarded([&] {
        B200_CHECK(s != nullptr, b200::kInvalidArgument, "NULL argument");
        s->s->drain();
    });
}

int b200_server_set_policy(b200_server* s, int policy, double shed_factor) {
    return guarded([&] {
        B200_CHECK(s != nullptr, b200::kInvalidArgument, "NULL argument");
        s->s->set_policy(policy, shed_factor);
    });
}

int b200_server_set_express(b200_server* s, int nworkers, double max_service_s) {
    return guarded([&] {
        B200_CHECK(s != nullptr, b200::kInvalidArgument, "NULL argument");
        s->s->set_express(nworkers, max_service_s);
    });
}

int b200_server_stats(b200_server* s, double* out6) {
    return guarded([&] {
        B200_CHECK(s && out6, b200::kInvalidArgument, "NULL argument");
        s->s->stats(out6);
    });
}

}  // extern "C"
