#include <algorithm>
// C-ABI entry points (include/abacus_b200.h).  Every call catches library
// errors and returns a status; the message is kept per thread.
#include <cstring>
#include <memory>
#include <string>

#include "capi_guard.h"
#include "../../include/abacus_b200.h"
#include "david.h"
#include "functors.h"
#include "hamilt.h"
#include "pw_grid.h"

#include "capi_handles.h"
#include "gemm_oz.h"
#include "gemm_tc.h"

#include <atomic>

namespace b200 {
namespace {
thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launches{0};
}  // namespace
void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }
void note_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
unsigned long long launches() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace b200

namespace {
using b200::guarded;
inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// A user H|psi> callback as the solvers' HPsiDevice.  The solver's stream is drained first, so the callback
// may read X from any stream or the host; afterwards the solver's stream waits for the legacy default stream,
// where a callback that does not synchronise leaves its writes (torch's default stream is that stream).  A
// nonzero return abandons the solve with B200_STATUS_CALLBACK_ERROR instead of reading an unwritten HX.
b200::HPsiDevice host_callback(b200_hpsi_cb hpsi, void* user) {
    return [hpsi, user](const void* x, void* hx, int nvec, int dim, int i0, int i1, cudaStream_t s) {
        B200_CUDA(cudaStreamSynchronize(s));
        const int rc = hpsi(user, x, hx, nvec, dim, i0, i1);
        B200_CHECK(rc == 0, b200::kCallbackError, "H|psi> callback returned status " + std::to_string(rc));
        if (s != nullptr && s != cudaStreamLegacy) {
            cudaEvent_t ev;
            B200_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            cudaError_t e = cudaEventRecord(ev, cudaStreamLegacy);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev, 0);
            cudaEventDestroy(ev);
            B200_CUDA(e);
        }
    };
}
}  // namespace

namespace {
template <typename T> T* aux_of(b200_pw_basis* b);
// device maps are uploaded on first device use, so basis set-up works without a GPU
template <> double2* aux_of<double2>(b200_pw_basis* b) {
    b->aux64.resize(size_t(b->grid.nxyz()));
    return b->aux64.ptr;
}
template <> float2* aux_of<float2>(b200_pw_basis* b) {
    b->aux32.resize(size_t(b->grid.nxyz()));
    return b->aux32.ptr;
}
template <typename T> int r2r_impl(b200_pw_basis* b, const void* in, void* out, int ik, int add, double f, void* st) {
    return guarded([&] {
        B200_CHECK(b && in && out, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(ik >= 0 && ik < int(b->grid.kmaps.size()), b200::kInvalidArgument, "k-point index out of range");
        b->grid.ensure_device();
        b200::launch_recip_to_real<T>(b->grid, ik, (const T*)in, (T*)out, aux_of<T>(b), add, f, S(st));
    });
}
template <typename T> int r2g_impl(b200_pw_basis* b, const void* in, void* out, int ik, int add, double f, void* st) {
    return guarded([&] {
        B200_CHECK(b && in && out, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(ik >= 0 && ik < int(b->grid.kmaps.size()), b200::kInvalidArgument, "k-point index out of range");
        b->grid.ensure_device();
        b200::launch_real_to_recip<T>(b->grid, ik, (const T*)in, (T*)out, aux_of<T>(b), add, f, S(st));
    });
}
}  // namespace

extern "C" {

const char* b200_last_error(void) { return b200::last_error(); }
const char* b200_version(void) { return "abacus_b200 0.1 (sm_100a)"; }
unsigned long long b200_kernel_launches(void) { return b200::launches(); }

// ------------------------------------------------------------------ functors
int b200_ekinetic_pw_op_f64(int nband, int npw, int max_npw, double tpiba2, const double* gk2, void* hpsi,
                            const void* psi, void* stream) {
    return guarded([&] {
        B200_CHECK(max_npw >= npw, b200::kInvalidArgument, "max_npw < npw");
        b200::ekinetic_pw<double2, double>(nband, npw, max_npw, tpiba2, gk2, (double2*)hpsi, (const double2*)psi, S(stream));
    });
}
int b200_ekinetic_pw_op_f32(int nband, int npw, int max_npw, float tpiba2, const float* gk2, void* hpsi, const void* psi,
                            void* stream) {
    return guarded([&] {
        B200_CHECK(max_npw >= npw, b200::kInvalidArgument, "max_npw < npw");
        b200::ekinetic_pw<float2, float>(nband, npw, max_npw, tpiba2, gk2, (float2*)hpsi, (const float2*)psi, S(stream));
    });
}
int b200_veff_pw_op_f64(int size, void* out, const double* in, void* stream) {
    return guarded([&] { b200::veff_pw<double2, double>(size, (double2*)out, in, S(stream)); });
}
int b200_veff_pw_op_f32(int size, void* out, const float* in, void* stream) {
    return guarded([&] { b200::veff_pw<float2, float>(size, (float2*)out, in, S(stream)); });
}
int b200_veff_pw_op_npol2_f64(int size, void* out, void* out1, const double* in0, const double* in1, const double* in2,
                              const double* in3, void* stream) {
    return guarded([&] {
        const double* in[4] = {in0, in1, in2, in3};
        b200::veff_pw_npol2<double2, double>(size, (double2*)out, (double2*)out1, in, S(stream));
    });
}
int b200_veff_pw_op_npol2_f32(int size, void* out, void* out1, const float* in0, const float* in1, const float* in2,
                              const float* in3, void* stream) {
    return guarded([&] {
        const float* in[4] = {in0, in1, in2, in3};
        b200::veff_pw_npol2<float2, float>(size, (float2*)out, (float2*)out1, in, S(stream));
    });
}
int b200_nonlocal_pw_op_f64(int l1, int l2, int l3, int* sum, int* iat, int spin, int nkb, int dx, int dy, int dz,
                            const double* deeq, void* ps, const void* becp, void* stream) {
    return guarded([&] {
        B200_CHECK(sum && iat, b200::kInvalidArgument, "sum/iat must not be NULL");
        b200::nonlocal_pw<double2, double>(l1, l2, l3, *sum, *iat, spin, nkb, dx, dy, dz, deeq, (double2*)ps,
                                           (const double2*)becp, S(stream));
    });
}
int b200_nonlocal_pw_op_f32(int l1, int l2, int l3, int* sum, int* iat, int spin, int nkb, int dx, int dy, int dz,
                            const float* deeq, void* ps, const void* becp, void* stream) {
    return guarded([&] {
        B200_CHECK(sum && iat, b200::kInvalidArgument, "sum/iat must not be NULL");
        b200::nonlocal_pw<float2, float>(l1, l2, l3, *sum, *iat, spin, nkb, dx, dy, dz, deeq, (float2*)ps,
                                         (const float2*)becp, S(stream));
    });
}
int b200_nonlocal_pw_op_nc_f64(int l1, int l2, int l3, int* sum, int* iat, int nkb, int dx, int dy, int dz,
                               const void* deeq_nc, void* ps, const void* becp, void* stream) {
    return guarded([&] {
        B200_CHECK(sum && iat, b200::kInvalidArgument, "sum/iat must not be NULL");
        b200::nonlocal_pw_nc<double2>(l1, l2, l3, *sum, *iat, nkb, dx, dy, dz, (const double2*)deeq_nc, (double2*)ps,
                                      (const double2*)becp, S(stream));
    });
}
int b200_nonlocal_pw_op_nc_f32(int l1, int l2, int l3, int* sum, int* iat, int nkb, int dx, int dy, int dz,
                               const void* deeq_nc, void* ps, const void* becp, void* stream) {
    return guarded([&] {
        B200_CHECK(sum && iat, b200::kInvalidArgument, "sum/iat must not be NULL");
        b200::nonlocal_pw_nc<float2>(l1, l2, l3, *sum, *iat, nkb, dx, dy, dz, (const float2*)deeq_nc, (float2*)ps,
                                     (const float2*)becp, S(stream));
    });
}
int b200_set_3d_fft_box_op_f64(int npwk, const int* idx, const void* in, void* out, void* stream) {
    return guarded([&] { b200::set_3d_fft_box<double2>(npwk, idx, (const double2*)in, (double2*)out, S(stream)); });
}
int b200_set_3d_fft_box_op_f32(int npwk, const int* idx, const void* in, void* out, void* stream) {
    return guarded([&] { b200::set_3d_fft_box<float2>(npwk, idx, (const float2*)in, (float2*)out, S(stream)); });
}
int b200_set_recip_to_real_output_op_f64(int nrxx, int add, double factor, const void* in, void* out, void* stream) {
    return guarded([&] {
        b200::set_recip_to_real_output<double2, double>(nrxx, add, factor, (const double2*)in, (double2*)out, S(stream));
    });
}
int b200_set_recip_to_real_output_op_f32(int nrxx, int add, float factor, const void* in, void* out, void* stream) {
    return guarded([&] {
        b200::set_recip_to_real_output<float2, float>(nrxx, add, factor, (const float2*)in, (float2*)out, S(stream));
    });
}
int b200_set_real_to_recip_output_op_f64(int npw_k, int nxyz, int add, double factor, const int* idx, const void* in,
                                         void* out, void* stream) {
    return guarded([&] {
        b200::set_real_to_recip_output<double2, double>(npw_k, nxyz, add, factor, idx, (const double2*)in, (double2*)out,
                                                        S(stream));
    });
}
int b200_set_real_to_recip_output_op_f32(int npw_k, int nxyz, int add, float factor, const int* idx, const void* in,
                                         void* out, void* stream) {
    return guarded([&] {
        b200::set_real_to_recip_output<float2, float>(npw_k, nxyz, add, factor, idx, (const float2*)in, (float2*)out,
                                                      S(stream));
    });
}

// ------------------------------------------------------------------ basis
int b200_pw_basis_create(double lat0, const double* latvec, double ecutwfc, double ecutrho, int nx, int ny, int nz,
                         int nks, const double* kvec_d, b200_pw_basis** out) {
    return guarded([&] {
        B200_CHECK(out != nullptr, b200::kInvalidArgument, "out must not be NULL");
        b200::PWBasisK b;
        const int rc = b.setup(lat0, latvec, ecutwfc, ecutrho, nx, ny, nz, nks, kvec_d);
        B200_CHECK(rc == 0, b200::kInvalidArgument,
                   rc == 2 ? "a k-point has no plane waves" : "invalid lattice, cut-off or k-points");
        auto p = std::make_unique<b200_pw_basis>();
        p->grid.build(b);
        *out = p.release();
    });
}
int b200_pw_basis_destroy(b200_pw_basis* b) {
    return guarded([&] { delete b; });
}
int b200_pw_basis_dims(const b200_pw_basis* b, int* dims) {
    return guarded([&] {
        B200_CHECK(b && dims, b200::kInvalidArgument, "NULL argument");
        const auto& g = b->grid;
        dims[0] = g.nx;
        dims[1] = g.ny;
        dims[2] = g.nz;
        dims[3] = g.nst;
        dims[4] = g.basis.npw;
        dims[5] = g.basis.npwk_max;
        dims[6] = g.basis.nks;
        dims[7] = g.nxc;
    });
}
int b200_pw_basis_scalars(const b200_pw_basis* b, double* scal) {
    return guarded([&] {
        B200_CHECK(b && scal, b200::kInvalidArgument, "NULL argument");
        scal[0] = b->grid.basis.tpiba2;
        scal[1] = b->grid.basis.omega;
        scal[2] = b->grid.basis.gk_ecut;
    });
}
int b200_pw_basis_kpoint(const b200_pw_basis* b, int ik, int* npwk, int* ig2ixyz, double* gk2, double* gcar) {
    return guarded([&] {
        B200_CHECK(b != nullptr, b200::kInvalidArgument, "NULL basis");
        const auto& B = b->grid.basis;
        B200_CHECK(ik >= 0 && ik < B.nks, b200::kInvalidArgument, "k-point index out of range");
        const int n = B.npwk[ik];
        const size_t off = size_t(ik) * B.npwk_max;
        if (npwk) *npwk = n;
        if (ig2ixyz) std::memcpy(ig2ixyz, &B.ig2ixyz_k[off], n * sizeof(int));
        if (gk2) std::memcpy(gk2, &B.gk2[off], n * sizeof(double));
        if (gcar) std::memcpy(gcar, &B.gcar[off * 3], n * 3 * sizeof(double));
    });
}
int b200_pw_basis_kvec_c(const b200_pw_basis* b, int ik, double* kvec_c) {
    return guarded([&] {
        B200_CHECK(b && kvec_c, b200::kInvalidArgument, "NULL argument");
        const auto& B = b->grid.basis;
        B200_CHECK(ik >= 0 && ik < B.nks, b200::kInvalidArgument, "k-point index out of range");
        for (int j = 0; j < 3; ++j) kvec_c[j] = B.kvec_c[3 * ik + j];
    });
}
int b200_pw_basis_device_maps(const b200_pw_basis* b, int ik, const double** gk2_d, const float** gk2f_d,
                              const int** ig2ixyz_d) {
    return guarded([&] {
        B200_CHECK(b != nullptr, b200::kInvalidArgument, "NULL basis");
        B200_CHECK(ik >= 0 && ik < int(b->grid.kmaps.size()), b200::kInvalidArgument, "k-point index out of range");
        const_cast<b200::PWGrid&>(b->grid).ensure_device();
        const auto& k = b->grid.kmaps[ik];
        if (gk2_d) *gk2_d = k.gk2.ptr;
        if (gk2f_d) *gk2f_d = k.gk2f.ptr;
        if (ig2ixyz_d) *ig2ixyz_d = k.ig2ixyz.ptr;
    });
}

int b200_recip_to_real_f64(b200_pw_basis* b, const void* in, void* out, int ik, int add, double factor, void* stream) {
    return r2r_impl<double2>(b, in, out, ik, add, factor, stream);
}
int b200_recip_to_real_f32(b200_pw_basis* b, const void* in, void* out, int ik, int add, float factor, void* stream) {
    return r2r_impl<float2>(b, in, out, ik, add, factor, stream);
}
int b200_real_to_recip_f64(b200_pw_basis* b, const void* in, void* out, int ik, int add, double factor, void* stream) {
    return r2g_impl<double2>(b, in, out, ik, add, factor, stream);
}
int b200_real_to_recip_f32(b200_pw_basis* b, const void* in, void* out, int ik, int add, float factor, void* stream) {
    return r2g_impl<float2>(b, in, out, ik, add, factor, stream);
}

// ------------------------------------------------------------------ Hamiltonian
int b200_hamilt_create(b200_pw_basis* b, int precision, b200_hamilt** out) {
    return guarded([&] {
        B200_CHECK(b && out, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(precision == B200_PREC_FP64 || precision == B200_PREC_MIXED, b200::kInvalidArgument, "bad precision");
        b->grid.ensure_device();
        auto p = std::make_unique<b200_hamilt>();
        p->h = std::make_unique<b200::Hamilt>(&b->grid, precision);
        *out = p.release();
    });
}
int b200_hamilt_destroy(b200_hamilt* h) {
    return guarded([&] { delete h; });
}
int b200_hamilt_set_veff(b200_hamilt* h, const double* veff) {
    return guarded([&] {
        B200_CHECK(h && veff, b200::kInvalidArgument, "NULL argument");
        h->h->set_veff(veff);
    });
}
int b200_hamilt_set_vkb(b200_hamilt* h, int ik, int nkb, int npwx, const void* vkb) {
    return guarded([&] {
        B200_CHECK(h != nullptr && (nkb == 0 || vkb != nullptr), b200::kInvalidArgument, "NULL argument");
        h->h->set_vkb(ik, nkb, npwx, (const double2*)vkb);
    });
}
int b200_hamilt_set_deeq(b200_hamilt* h, int ntype, const int* na, const int* nh, int nspin, int dx, int dy, int dz,
                         const double* deeq) {
    return guarded([&] {
        B200_CHECK(h && na && nh && deeq, b200::kInvalidArgument, "NULL argument");
        h->h->set_deeq(ntype, na, nh, nspin, dx, dy, dz, deeq);
    });
}
int b200_hamilt_set_veff_nc(b200_hamilt* h, const double* veff4) {
    return guarded([&] {
        B200_CHECK(h && veff4, b200::kInvalidArgument, "NULL argument");
        h->h->set_veff_nc(veff4);
    });
}
int b200_hamilt_set_deeq_nc(b200_hamilt* h, int ntype, const int* na, const int* nh, int dx, int dy, int dz,
                            const void* deeq_nc) {
    return guarded([&] {
        B200_CHECK(h && na && nh && deeq_nc, b200::kInvalidArgument, "NULL argument");
        h->h->set_deeq_nc(ntype, na, nh, dx, dy, dz, (const double2*)deeq_nc);
    });
}
int b200_hamilt_hpsi_nc(b200_hamilt* h, int ik, int nbands, int ld, const void* psi, void* hpsi, void* stream) {
    return guarded([&] {
        B200_CHECK(h && psi && hpsi, b200::kInvalidArgument, "NULL argument");
        if (h->h->precision == B200_PREC_FP64)
            h->h->hpsi_nc<double2>(ik, nbands, ld, (const double2*)psi, (double2*)hpsi, S(stream));
        else
            h->h->hpsi_nc<float2>(ik, nbands, ld, (const float2*)psi, (float2*)hpsi, S(stream));
    });
}
static int hpsi_impl(b200_hamilt* h, int ik, int spin, int nb, int ld, const void* psi, void* hpsi, int mode, void* st) {
    return guarded([&] {
        B200_CHECK(h && psi && hpsi, b200::kInvalidArgument, "NULL argument");
        if (h->h->precision == B200_PREC_FP64)
            h->h->hpsi<double2>(ik, spin, nb, ld, (const double2*)psi, (double2*)hpsi, mode, S(st));
        else
            h->h->hpsi<float2>(ik, spin, nb, ld, (const float2*)psi, (float2*)hpsi, mode, S(st));
    });
}
int b200_hamilt_hpsi(b200_hamilt* h, int ik, int spin, int nbands, int ld, const void* psi, void* hpsi, void* stream) {
    return hpsi_impl(h, ik, spin, nbands, ld, psi, hpsi, 0, stream);
}
int b200_hamilt_hpsi_part(b200_hamilt* h, int ik, int spin, int nbands, int ld, const void* psi, void* hpsi, int mode,
                          void* stream) {
    if (mode != 1 && mode != 2) {
        b200::set_last_error("mode must be 1 (local) or 2 (nonlocal)");
        return B200_STATUS_INVALID_ARGUMENT;
    }
    return hpsi_impl(h, ik, spin, nbands, ld, psi, hpsi, mode, stream);
}

// ------------------------------------------------------------------ Davidson
int b200_david_create(int nband, int dim, int david_ndim, int precision, const double* precond, b200_david** out) {
    return guarded([&] {
        B200_CHECK(out && precond, b200::kInvalidArgument, "NULL argument");
        auto d = b200::make_david(nband, dim, david_ndim, precision, precond);  // arguments checked first
        auto p = std::make_unique<b200_david>();
        p->d = std::move(d);
        *out = p.release();
    });
}
int b200_david_destroy(b200_david* d) {
    return guarded([&] { delete d; });
}
int b200_david_diag(b200_david* d, b200_hpsi_cb hpsi, void* user, int ldpsi, void* psi, double* eig, double thr,
                    int maxiter, int ntry_max, int notconv_max, int* iters) {
    return guarded([&] {
        B200_CHECK(d && hpsi && psi && eig, b200::kInvalidArgument, "NULL argument");
        b200::HPsiDevice f = host_callback(hpsi, user);
        const int it = d->d->diag(f, ldpsi, psi, eig, thr, maxiter, ntry_max, notconv_max);
        if (iters) *iters = it;
    });
}
static thread_local b200::TcGemmWorkspace g_tc_ws;
int b200_tc_cgemm(char transa, char transb, int m, int n, int k, float alpha_re, float alpha_im, const void* a, int lda,
                  const void* b, int ldb, float beta_re, float beta_im, void* c, int ldc, void* stream) {
    b200::TcGemmWorkspace& ws = g_tc_ws;
    return guarded([&] {
        B200_CHECK(transb == 'N' || transb == 'n', b200::kInvalidArgument, "transb must be 'N'");
        const char opa = (transa == 'n' || transa == 'N') ? 'N' : ((transa == 'c' || transa == 'C') ? 'C' : '?');
        B200_CHECK(opa != '?', b200::kInvalidArgument, "transa must be 'N' or 'C'");
        b200::tc_cgemm(opa, m, n, k, make_float2(alpha_re, alpha_im), (const float2*)a, lda, (const float2*)b, ldb,
                       make_float2(beta_re, beta_im), (float2*)c, ldc, ws, S(stream));
    });
}
int b200_tc_cgemm_error(int* code) {
    return guarded([&] {
        B200_CHECK(code != nullptr, b200::kInvalidArgument, "NULL argument");
        *code = g_tc_ws.read_error();
    });
}
int b200_tc_set_wait_limit_ns(unsigned long long ns) {
    return guarded([&] { b200::set_tc_wait_limit_ns(ns); });
}
static thread_local b200::OzWorkspace g_oz_ws;
int b200_zgemm_i8(char transa, char transb, int m, int n, int k, const double* alpha, const void* a, int lda,
                  const void* b, int ldb, const double* beta, void* c, int ldc, int nmods, void* stream) {
    b200::OzWorkspace& ws = g_oz_ws;
    return guarded([&] {
        B200_CHECK(transb == 'N' || transb == 'n', b200::kInvalidArgument, "transb must be 'N'");
        const char opa = (transa == 'n' || transa == 'N') ? 'N' : ((transa == 'c' || transa == 'C') ? 'C' : '?');
        B200_CHECK(opa != '?', b200::kInvalidArgument, "transa must be 'N' or 'C'");
        B200_CHECK(alpha && beta, b200::kInvalidArgument, "NULL alpha or beta");
        B200_CHECK(m >= 0 && n >= 0 && k >= 0, b200::kInvalidArgument, "negative dimension");
        if (m == 0 || n == 0) return;
        B200_CHECK(a && b && c, b200::kInvalidArgument, "NULL matrix");
        const double2 al = make_double2(alpha[0], alpha[1]), be = make_double2(beta[0], beta[1]);
        if (k == 0) {  // C = beta C
            b200::scale_matrix_z(m, n, be, static_cast<double2*>(c), ldc, S(stream));
            return;
        }
        b200::oz_prepare_a(opa, m, k, static_cast<const double2*>(a), lda, nmods, ws.a, ws, S(stream));
        b200::oz_zgemm(opa, m, n, k, al, ws.a, static_cast<const double2*>(b), ldb, be, static_cast<double2*>(c), ldc,
                       ws, nullptr, S(stream));
    });
}
int b200_zgemm_i8_error(int* code) {
    return guarded([&] {
        B200_CHECK(code != nullptr, b200::kInvalidArgument, "NULL argument");
        *code = g_oz_ws.read_error(0);
    });
}
int b200_zgemm_i8_constants(int nmods, long long kr, int* mods, double* wa, double* wb, double* mprod, int* q) {
    return guarded([&] {
        B200_CHECK(mods && wa && wb && mprod && q, b200::kInvalidArgument, "NULL argument");
        B200_CHECK(kr >= 1, b200::kInvalidArgument, "kr < 1");
        b200::oz_constants(nmods, long(kr), mods, wa, wb, mprod, q);
    });
}
int b200_david_set_stream(b200_david* d, void* stream) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        d->d->set_stream(S(stream));
    });
}
int b200_david_set_verbosity(b200_david* d, int level) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        d->d->set_verbosity(level);
    });
}
int b200_david_set_mixed_threshold(b200_david* d, double thr) {
    return guarded([&] {
        B200_CHECK(d != nullptr && thr > 0.0, b200::kInvalidArgument, "bad argument");
        d->d->set_mixed_thr(thr);
    });
}
int b200_david_set_fp64_gemm(b200_david* d, int mode) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        d->d->set_fp64_gemm(mode);
    });
}
int b200_david_set_low_ndim(b200_david* d, int ndim) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        d->d->set_low_ndim(ndim);
    });
}
int b200_david_set_trace(b200_david* d, int on) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        d->d->trace().on = on != 0;
    });
}
int b200_david_trace(b200_david* d, int max_iters, int nband, double* t, int* stage, double* eig, int* n_out) {
    return guarded([&] {
        B200_CHECK(d && n_out, b200::kInvalidArgument, "NULL argument");
        const b200::DavidTrace& tr = d->d->trace();
        const int n = int(tr.t.size());
        B200_CHECK(n == 0 || int(tr.eig.size()) == n * nband, b200::kInvalidArgument, "nband differs from the solver's");
        const int m = n < max_iters ? n : max_iters;
        for (int i = 0; i < m; ++i) {
            if (t) t[i] = tr.t[i];
            if (stage) stage[i] = tr.stage[i];
            if (eig) std::copy(tr.eig.begin() + size_t(i) * nband, tr.eig.begin() + size_t(i + 1) * nband, eig + size_t(i) * nband);
        }
        *n_out = n;
    });
}
int b200_david_stats(const b200_david* d, int* iters_low, int* iters_fp64, int* hpsi_bands) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        const auto& st = d->d->stats();
        if (iters_low) *iters_low = st.iters_low;
        if (iters_fp64) *iters_fp64 = st.iters_fp64;
        if (hpsi_bands) *hpsi_bands = st.hpsi_bands;
    });
}
int b200_david_diag_hamilt(b200_david* d, b200_hamilt* h, int ik, int spin, int ldpsi, void* psi, double* eig,
                           double thr, int maxiter, int ntry_max, int notconv_max, int* iters) {
    return guarded([&] {
        B200_CHECK(d && h && psi && eig, b200::kInvalidArgument, "NULL argument");
        b200::Hamilt* H = h->h.get();
        b200::HpsiWork* W = &d->work;
        b200::HPsiDevice f64 = [H, W, ik, spin](const void* x, void* hx, int, int dim, int i0, int i1, cudaStream_t s) {
            const double2* X = (const double2*)x + size_t(i0) * dim;
            H->hpsi<double2>(ik, spin, i1 - i0 + 1, dim, X, (double2*)hx, 0, s, W);
        };
        b200::HPsiDevice f32 = [H, W, ik, spin](const void* x, void* hx, int, int dim, int i0, int i1, cudaStream_t s) {
            const float2* X = (const float2*)x + size_t(i0) * dim;
            H->hpsi<float2>(ik, spin, i1 - i0 + 1, dim, X, (float2*)hx, 0, s, W);
        };
        const int it = d->d->diag_hamilt(f64, f32, d->d->precision(), ldpsi, psi, eig, thr, maxiter, ntry_max, notconv_max);
        if (iters) *iters = it;
    });
}

// ------------------------------------------------------------------ Davidson with subspace rotation
int b200_dav_subspace_create(int nband, int dim, int david_ndim, double diag_thr, int diag_nmax, int need_subspace,
                             const double* precond, b200_dav_subspace** out) {
    return guarded([&] {
        B200_CHECK(out && precond, b200::kInvalidArgument, "NULL argument");
        // the solver (which checks its arguments before any device call) before the handle's H|psi> scratch
        auto d = b200::make_dav_subspace(nband, dim, david_ndim, diag_thr, diag_nmax, need_subspace != 0, precond);
        auto p = std::make_unique<b200_dav_subspace>();
        p->d = std::move(d);
        *out = p.release();
    });
}
int b200_dav_subspace_destroy(b200_dav_subspace* d) {
    return guarded([&] { delete d; });
}
int b200_dav_subspace_diag(b200_dav_subspace* d, b200_hpsi_cb hpsi, void* user, void* psi, int psi_in_dmax, double* eig,
                           const int* is_occupied, int scf_type, int* iters) {
    return guarded([&] {
        B200_CHECK(d && hpsi && psi && eig, b200::kInvalidArgument, "NULL argument");
        b200::HPsiDevice f = host_callback(hpsi, user);
        const int it = d->d->diag(f, psi, psi_in_dmax, eig, is_occupied, scf_type != 0);
        if (iters) *iters = it;
    });
}
int b200_dav_subspace_diag_hamilt(b200_dav_subspace* d, b200_hamilt* h, int ik, int spin, void* psi, int psi_in_dmax,
                                  double* eig, const int* is_occupied, int scf_type, int* iters) {
    return guarded([&] {
        B200_CHECK(d && h && psi && eig, b200::kInvalidArgument, "NULL argument");
        b200::Hamilt* H = h->h.get();
        b200::HpsiWork* W = &d->work;
        b200::HPsiDevice f = [H, W, ik, spin](const void* x, void* hx, int, int dim, int i0, int i1, cudaStream_t s) {
            const double2* X = (const double2*)x + size_t(i0) * dim;
            H->hpsi<double2>(ik, spin, i1 - i0 + 1, dim, X, (double2*)hx, 0, s, W);
        };
        const int it = d->d->diag(f, psi, psi_in_dmax, eig, is_occupied, scf_type != 0);
        if (iters) *iters = it;
    });
}
int b200_dav_subspace_set_stream(b200_dav_subspace* d, void* stream) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        d->d->set_stream(S(stream));
    });
}
int b200_dav_subspace_set_verbosity(b200_dav_subspace* d, int level) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        d->d->set_verbosity(level);
    });
}
int b200_dav_subspace_stats(const b200_dav_subspace* d, int* notconv, int* hpsi_bands) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        if (notconv) *notconv = d->d->notconv();
        if (hpsi_bands) *hpsi_bands = d->d->hpsi_bands();
    });
}

// ------------------------------------------------------------------ band-parallel CG
int b200_bpcg_create(const double* precond, int nband, int nbasis, b200_bpcg** out) {
    return guarded([&] {
        B200_CHECK(out && precond, b200::kInvalidArgument, "NULL argument");
        auto d = b200::make_bpcg(nband, nbasis, precond);  // arguments checked before any device call
        auto p = std::make_unique<b200_bpcg>();
        p->d = std::move(d);
        *out = p.release();
    });
}
int b200_bpcg_destroy(b200_bpcg* d) {
    return guarded([&] { delete d; });
}
int b200_bpcg_diag(b200_bpcg* d, b200_hpsi_cb hpsi, void* user, void* psi, double* eig, int scf_iter, int* iters) {
    return guarded([&] {
        B200_CHECK(d && hpsi && psi && eig, b200::kInvalidArgument, "NULL argument");
        b200::HPsiDevice f = host_callback(hpsi, user);
        const int it = d->d->diag(f, psi, eig, scf_iter);
        if (iters) *iters = it;
    });
}
int b200_bpcg_diag_hamilt(b200_bpcg* d, b200_hamilt* h, int ik, int spin, void* psi, double* eig, int scf_iter,
                          int* iters) {
    return guarded([&] {
        B200_CHECK(d && h && psi && eig, b200::kInvalidArgument, "NULL argument");
        b200::Hamilt* H = h->h.get();
        B200_CHECK(ik >= 0 && ik < int(H->grid->kmaps.size()), b200::kInvalidArgument, "k-point index out of range");
        const int npw = H->grid->kmaps[ik].npw;
        b200::HpsiWork* W = &d->work;
        b200::HPsiDevice f = [H, W, ik, spin, npw](const void* x, void* hx, int, int dim, int i0, int i1,
                                                   cudaStream_t s) {
            const int nb = i1 - i0 + 1;
            const double2* X = (const double2*)x + size_t(i0) * dim;
            H->hpsi<double2>(ik, spin, nb, dim, X, (double2*)hx, 0, s, W);
            if (dim > npw)
                B200_CUDA(cudaMemset2DAsync((double2*)hx + npw, size_t(dim) * sizeof(double2), 0,
                                            size_t(dim - npw) * sizeof(double2), nb, s));
        };
        const int it = d->d->diag(f, psi, eig, scf_iter);
        if (iters) *iters = it;
    });
}
int b200_bpcg_set_stream(b200_bpcg* d, void* stream) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        d->d->set_stream(S(stream));
    });
}
int b200_bpcg_stats(const b200_bpcg* d, double* max_err, int* hpsi_bands) {
    return guarded([&] {
        B200_CHECK(d != nullptr, b200::kInvalidArgument, "NULL argument");
        if (max_err) *max_err = d->d->max_err();
        if (hpsi_bands) *hpsi_bands = d->d->hpsi_bands();
    });
}

}  // extern "C"
