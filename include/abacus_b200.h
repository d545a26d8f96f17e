/*
 * abacus_b200.h -- C-ABI of the B200-native plane-wave H|psi> / Davidson path.
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream (as void*,
 * NULL = legacy default stream, which is what ABACUS uses implicitly) and
 * returns an int status (0 = success, see B200_STATUS_*).  On failure
 * b200_last_error() returns a message for the calling thread.  No entry point
 * calls exit(); the reference's cudaErrcheck / WARNING_QUIT become statuses.
 *
 * Device pointers (suffix _d in the comments) are CUDA device memory owned by
 * the caller, exactly as in the reference where buffers come from
 * resize_memory_op<T, DEVICE_GPU> (module_base/module_device/memory_op.h:16-93).
 * Complex numbers are interleaved (re, im) pairs, layout-compatible with
 * std::complex<double> / std::complex<float>.
 *
 * Reference = abacus-develop v3.8.0; paths are relative to its source/ tree.
 */
#ifndef ABACUS_B200_H
#define ABACUS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define B200_STATUS_OK 0
#define B200_STATUS_INVALID_ARGUMENT 1
#define B200_STATUS_CUDA_ERROR 2
#define B200_STATUS_CUBLAS_ERROR 3
#define B200_STATUS_CUSOLVER_ERROR 4
#define B200_STATUS_NUMERICAL_ERROR 5
#define B200_STATUS_CAPACITY_ERROR 6
#define B200_STATUS_NOT_CONVERGED 7
#define B200_STATUS_CALLBACK_ERROR 8 /* a user H|psi> callback returned nonzero; the solve was abandoned */
#define B200_STATUS_SHED 9           /* a served request waited past its cell's admission bound and was not run */

/* precision of a handle: plain FP64, or mixed (FP32 FFTs / split-precision GEMMs) */
#define B200_PREC_FP64 0
#define B200_PREC_MIXED 1

typedef struct b200_pw_basis b200_pw_basis; /* host + device plane-wave basis of one pool */
typedef struct b200_hamilt b200_hamilt;     /* V_eff, projectors, D and workspaces */
typedef struct b200_david b200_david;       /* Davidson workspaces */
typedef struct b200_dav_subspace b200_dav_subspace; /* Davidson-with-subspace-rotation workspaces */
typedef struct b200_bpcg b200_bpcg;         /* band-parallel CG workspaces */
typedef struct b200_graph b200_graph;       /* an instantiated CUDA graph of a captured call */

/* Message of the last failed call on this thread ("" if none). */
const char* b200_last_error(void);
/* Library version string. */
const char* b200_version(void);
/* Number of kernels this library has launched so far in this process (its own
 * kernels only; cuBLAS / cuSOLVER launches are not counted). */
unsigned long long b200_kernel_launches(void);

/* ------------------------------------------------------------------ op functors
 * Each replaces the body of a DEVICE_GPU partial specialisation; arguments keep
 * the reference's meaning and order. */

/* ekinetic_pw_op<FP, DEVICE_GPU>::operator()
 *   module_hamilt_pw/hamilt_pwdft/kernels/ekinetic_op.h:38-48
 *   tmhpsi_d[ib*max_npw+ig] += gk2_ik_d[ig]*tpiba2*tmpsi_in_d[ib*max_npw+ig], ig < npw */
int b200_ekinetic_pw_op_f64(int nband, int npw, int max_npw, double tpiba2, const double* gk2_ik_d, void* tmhpsi_d,
                            const void* tmpsi_in_d, void* stream);
int b200_ekinetic_pw_op_f32(int nband, int npw, int max_npw, float tpiba2, const float* gk2_ik_d, void* tmhpsi_d,
                            const void* tmpsi_in_d, void* stream);

/* veff_pw_op<FP, DEVICE_GPU>::operator()(dev, size, out, in)
 *   module_hamilt_pw/hamilt_pwdft/kernels/veff_op.h:57-66 -- out_d[ir] *= in_d[ir] */
int b200_veff_pw_op_f64(int size, void* out_d, const double* in_d, void* stream);
int b200_veff_pw_op_f32(int size, void* out_d, const float* in_d, void* stream);
/* npol = 2 form (dev, size, out, out1, const FP** in): in0..in3 are the four spin components */
int b200_veff_pw_op_npol2_f64(int size, void* out_d, void* out1_d, const double* in0_d, const double* in1_d,
                              const double* in2_d, const double* in3_d, void* stream);
int b200_veff_pw_op_npol2_f32(int size, void* out_d, void* out1_d, const float* in0_d, const float* in1_d,
                              const float* in2_d, const float* in3_d, void* stream);

/* nonlocal_pw_op<FP, DEVICE_GPU>::operator()
 *   module_hamilt_pw/hamilt_pwdft/kernels/nonlocal_op.h:82-113
 *   l1 = na, l2 = nbands, l3 = nh; *sum += l1*l3 and *iat += l1 on return, as the reference does. */
int b200_nonlocal_pw_op_f64(int l1, int l2, int l3, int* sum, int* iat, int spin, int nkb, int deeq_x, int deeq_y,
                            int deeq_z, const double* deeq_d, void* ps_d, const void* becp_d, void* stream);
int b200_nonlocal_pw_op_f32(int l1, int l2, int l3, int* sum, int* iat, int spin, int nkb, int deeq_x, int deeq_y,
                            int deeq_z, const float* deeq_d, void* ps_d, const void* becp_d, void* stream);
/* non-collinear form with complex deeq_nc (same header, second overload) */
int b200_nonlocal_pw_op_nc_f64(int l1, int l2, int l3, int* sum, int* iat, int nkb, int deeq_x, int deeq_y,
                               int deeq_z, const void* deeq_nc_d, void* ps_d, const void* becp_d, void* stream);
int b200_nonlocal_pw_op_nc_f32(int l1, int l2, int l3, int* sum, int* iat, int nkb, int deeq_x, int deeq_y,
                               int deeq_z, const void* deeq_nc_d, void* ps_d, const void* becp_d, void* stream);

/* set_3d_fft_box_op / set_recip_to_real_output_op / set_real_to_recip_output_op <FP, DEVICE_GPU>
 *   module_basis/module_pw/kernels/pw_op.h (CPU bodies pw_op.cpp:6-68) */
int b200_set_3d_fft_box_op_f64(int npwk, const int* box_index_d, const void* in_d, void* out_d, void* stream);
int b200_set_3d_fft_box_op_f32(int npwk, const int* box_index_d, const void* in_d, void* out_d, void* stream);
int b200_set_recip_to_real_output_op_f64(int nrxx, int add, double factor, const void* in_d, void* out_d, void* stream);
int b200_set_recip_to_real_output_op_f32(int nrxx, int add, float factor, const void* in_d, void* out_d, void* stream);
int b200_set_real_to_recip_output_op_f64(int npw_k, int nxyz, int add, double factor, const int* box_index_d,
                                         const void* in_d, void* out_d, void* stream);
int b200_set_real_to_recip_output_op_f32(int npw_k, int nxyz, int add, float factor, const int* box_index_d,
                                         const void* in_d, void* out_d, void* stream);

/* ------------------------------------------------------------------ plane-wave basis
 * Replaces PW_Basis_K set-up for one pool: initgrids (module_basis/module_pw/pw_init.cpp:24-170),
 * initparameters (pw_basis_k.cpp:53-116), setuptransform + setupIndGk (pw_basis_k.cpp:118-187),
 * collect_local_pw (:189-265) and get_ig2ixyz_k (:319-344).  Builds the host maps and
 * uploads the device stick maps.  nx = ny = nz = 0 selects the reference's 2,3,5-smooth
 * grid rule; ecutrho == 0 means 4*ecutwfc; ecutrho < 0 with an explicit grid means the cutoff that
 * grid holds (initgrids(lat0, latvec, nx, ny, nz), pw_init.cpp:157-207).  latvec is row-major (rows = a1, a2, a3 in
 * units of lat0), kvec_d is nks x 3 direct coordinates. */
int b200_pw_basis_create(double lat0, const double* latvec, double ecutwfc, double ecutrho, int nx, int ny, int nz,
                         int nks, const double* kvec_d, b200_pw_basis** out);
int b200_pw_basis_destroy(b200_pw_basis* b);
/* dims[0..7] = nx, ny, nz, nst, npw (ggecut sphere), npwk_max, nks, nxc (occupied x columns) */
int b200_pw_basis_dims(const b200_pw_basis* b, int* dims);
/* scal[0..2] = tpiba2, omega, gk_ecut */
int b200_pw_basis_scalars(const b200_pw_basis* b, double* scal);
/* host copies for k-point ik: npwk, ig2ixyz (npwk ints), gk2 (npwk), gcar (npwk x 3, units of tpiba);
 * any output pointer may be NULL */
int b200_pw_basis_kpoint(const b200_pw_basis* b, int ik, int* npwk, int* ig2ixyz, double* gk2, double* gcar);
/* kvec_c (3 doubles, units of tpiba) of k-point ik */
int b200_pw_basis_kvec_c(const b200_pw_basis* b, int ik, double* kvec_c);
/* device pointers of gk2 (FP64 and FP32 copies, npwk) and ig2ixyz for k-point ik -- the
 * arrays ABACUS keeps as d_gk2 / s_gk2 / ig2ixyz_k (pw_basis_k.h). */
int b200_pw_basis_device_maps(const b200_pw_basis* b, int ik, const double** gk2_d, const float** gk2f_d,
                              const int** ig2ixyz_d);

/* PW_Basis_K::recip_to_real<FP, DEVICE_GPU>(ctx, in, out, ik, add, factor)
 *   module_basis/module_pw/pw_basis_k.h:140-153, GPU bodies pw_transform_k.cpp:404-476.
 *   in_d: npwk coefficients of k-point ik; out_d: nx*ny*nz box in r = (ix*ny+iy)*nz+iz order.
 *   out = r (add = 0) or out += factor*r (add = 1); r is the un-normalised exp(+iGr) sum. */
int b200_recip_to_real_f64(b200_pw_basis* b, const void* in_d, void* out_d, int ik, int add, double factor,
                           void* stream);
int b200_recip_to_real_f32(b200_pw_basis* b, const void* in_d, void* out_d, int ik, int add, float factor,
                           void* stream);
/* PW_Basis_K::real_to_recip<FP, DEVICE_GPU>(ctx, in, out, ik, add, factor)
 *   GPU bodies pw_transform_k.cpp:336-401: out = box/nxyz (add = 0) or out += factor/nxyz*box. */
int b200_real_to_recip_f64(b200_pw_basis* b, const void* in_d, void* out_d, int ik, int add, double factor,
                           void* stream);
int b200_real_to_recip_f32(b200_pw_basis* b, const void* in_d, void* out_d, int ik, int add, float factor,
                           void* stream);

/* ------------------------------------------------------------------ Hamiltonian
 * One handle holds what the operator chain Ekinetic -> Veff -> Nonlocal of
 * HamiltPW (module_hamilt_pw/hamilt_pwdft/hamilt_pw.cpp:21-114) holds on the
 * device: V_eff, the projectors vkb per k (Nonlocal::init, nonlocal_pw.cpp:42-58)
 * and deeq.  npol = 1, one spin channel per call. */
int b200_hamilt_create(b200_pw_basis* b, int precision, b200_hamilt** out);
int b200_hamilt_destroy(b200_hamilt* h);
/* veff_d: nx*ny*nz FP64 in ABACUS's r order (the row this->veff + spin*veff_col of Veff::act) */
int b200_hamilt_set_veff(b200_hamilt* h, const double* veff_d);
/* vkb_d: nkb x npwx row-major complex128 (ABACUS's ppcell->vkb for k-point ik, VNL_in_pw.h:106);
 * pass nkb = 0 for no projectors */
int b200_hamilt_set_vkb(b200_hamilt* h, int ik, int nkb, int npwx, const void* vkb_d);
/* deeq_d: (nspin, deeq_x = nat, deeq_y = nhm, deeq_z = nhm) FP64; na/nh per atom type (host arrays) */
int b200_hamilt_set_deeq(b200_hamilt* h, int ntype, const int* na, const int* nh, int nspin, int deeq_x, int deeq_y,
                         int deeq_z, const double* deeq_d);
/* Operator::hPsi for bands [0, nbands) of k-point ik (module_hamilt_general/operator.cpp:39-88):
 * hpsi = (T + V_loc + V_NL) psi, entries npwk..ld-1 of each band zeroed.
 * psi_d / hpsi_d: complex128 (FP64 handle) or complex64 (mixed handle), band b at b*ld.
 * spin selects the deeq spin channel (isk[ik]). */
int b200_hamilt_hpsi(b200_hamilt* h, int ik, int spin, int nbands, int ld, const void* psi_d, void* hpsi_d,
                     void* stream);
/* ---- npol = 2 (non-collinear) ----
 * Veff's four components for the spinor branch of Veff::act (veff_pw.cpp:73-104, veff_pw_op's npol = 2
 * form veff_op.cpp:20-37): veff4_d = 4 x nrxx doubles (V, then the three magnetic components), each in
 * b200_hamilt_set_veff's order. */
int b200_hamilt_set_veff_nc(b200_hamilt* h, const double* veff4_d);
/* D's four complex spin blocks deeq_nc(4, dx, dy, dz) (nonlocal_pw_op's npol = 2 overload,
 * nonlocal_op.h:82-113, CPU body nonlocal_op.cpp:43-74), folded into the projectors of every k-point:
 * W_s = vkb D_s per atom block, so that H psi_up += W0 becp_up + W1 becp_dn, H psi_dn += W2 becp_up +
 * W3 becp_dn. */
int b200_hamilt_set_deeq_nc(b200_hamilt* h, int ntype, const int* na, const int* nh, int deeq_x, int deeq_y,
                            int deeq_z, const void* deeq_nc_d);
/* Operator::hPsi with npol = 2 (operator.cpp:39-88): band b's two spinor components at psi_d + (2b + c) ld
 * (the reference's nbasis = 2 ld layout), hpsi_d overwritten (padding zeroed): the kinetic diagonal on
 * both components, the 2x2 V_eff in real space, the projectors with deeq_nc.  The local part runs the stick
 * passes on the 2 nbands spinor columns and splits the plane pass at the real-space product (a scratch of
 * two real-space boxes per band, in chunks of 512 MB). */
int b200_hamilt_hpsi_nc(b200_hamilt* h, int ik, int nbands, int ld, const void* psi_d, void* hpsi_d, void* stream);
/* H|psi> between host buffers (psi_h in, hpsi_h out, band b at b*ld, the handle's element type), through
 * the caller's device buffers psi_d / hpsi_d (nbands*ld each): the bands go in npieces pieces through
 * three streams so that the upload of piece p+1, H|psi> of piece p and the download of piece p-1 overlap
 * (the first and last piece are half as large as the others: their copies are not overlapped).
 * Asynchronous: hpsi_h is complete when `stream` is.  Pinned (page-locked) host buffers give the overlap;
 * pageable ones work with synchronous copies.  The handle's copy streams are shared: one call at a time
 * per handle.  No counterpart in the reference (its Operator::hPsi works on device memory,
 * module_hamilt_general/operator.cpp:39-88; the host <-> device copies are the caller's). */
int b200_hamilt_hpsi_host(b200_hamilt* h, int ik, int spin, int nbands, int ld, const void* psi_h, void* hpsi_h,
                          void* psi_d, void* hpsi_d, int npieces, void* stream);
/* Parts of H|psi>, for checking and for callers that compose their own chain:
 * mode 1 = kinetic + local only, mode 2 = nonlocal only (accumulated into hpsi_d). */
int b200_hamilt_hpsi_part(b200_hamilt* h, int ik, int spin, int nbands, int ld, const void* psi_d, void* hpsi_d,
                          int mode, void* stream);

/* Allocation-free form of b200_hamilt_hpsi_part(mode = 1): kinetic + local part of
 * H|psi> for bands [0, nbands) of k-point ik, written to hpsi_d (padding zeroed).
 * No counterpart in the reference: it exists for callers that cannot allocate device
 * memory during the call (inside a CUDA-graph capture, under a host framework that owns
 * the device memory pool, or on paths that must not synchronise).  It calls no
 * cudaMalloc/cudaFree; its scratch is a fixed 32 MiB device array inside the library,
 * held by every GPU that loads the library until exit.  The first call on each device
 * looks up that array's address (cudaGetSymbolAddress), so make it before any stream
 * capture.  A grid whose one-band stick buffer (nst*nz complex values) exceeds 32 MiB is
 * rejected with B200_STATUS_CAPACITY_ERROR.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller. */
int b200_hamilt_hpsi_local_noalloc(b200_hamilt* h, int ik, int nbands, int ld, const void* psi_d, void* hpsi_d,
                                   void* stream);

/* H|psi> for nbands bands of each of nk k-points (1 <= nk <= 128) in one call: the same result as
 * b200_hamilt_hpsi once per k-point (HamiltPW::updateHk + Operator::hPsi per k, hsolver_pw.cpp:240-270),
 * with the kinetic + local part of all k-points done in one launch per FFT pass.
 * iks: host array of nk k-point indices; psi_d / hpsi_d: host arrays of nk device pointers. */
int b200_hamilt_hpsi_kbatch(b200_hamilt* h, int nk, const int* iks, int spin, int nbands, int ld, void* const* psi_d,
                            void* const* hpsi_d, void* stream);
/* Captures b200_hamilt_hpsi_kbatch with these arguments into a CUDA graph (after one eager call that
 * allocates every workspace; the eager call's output is the same as a replay's).  stream must not be
 * the legacy default stream.  Replays read psi_d and write hpsi_d at the captured addresses.
 * No counterpart in the reference. */
int b200_graph_capture_hpsi_kbatch(b200_hamilt* h, int nk, const int* iks, int spin, int nbands, int ld,
                                   void* const* psi_d, void* const* hpsi_d, void* stream, b200_graph** out);
int b200_graph_launch(b200_graph* g, void* stream);
int b200_graph_destroy(b200_graph* g);
/* Times the kinetic + local pass of k-point ik over candidate band-chunk sizes (1, 2, 4 ... 128 and
 * nbands) and, on grids with square planes of 64, 96 or 128 points, over the plane-pass variants
 * (three timed repetitions each after one warm-up), and keeps the fastest pair: the chunk for this
 * handle, the plane variant for every handle of this basis in the handle's precision.  Overwrites
 * hpsi_d.  best_chunk / best_variant may be NULL.  No counterpart in the reference. */
int b200_hamilt_autotune(b200_hamilt* h, int ik, int nbands, int ld, const void* psi_d, void* hpsi_d, void* stream,
                         int* best_chunk, int* best_variant);
/* Plane pass of the local H|psi> on grids with square planes of 64, 96 or 128 points, for every
 * handle of this basis in this handle's precision: 1 = one warp per line, five warp-shuffle lane
 * stages; 2-5 = two-pass register transforms through shared memory (four launch shapes); 0 = the
 * default.  All variants give the same results within rounding.  No counterpart in the reference. */
int b200_hamilt_set_plane_variant(b200_hamilt* h, int variant);
/* The FP64 projector products of Nonlocal::act (nonlocal_pw.cpp:255-276, becp = vkb^H psi and
 * H psi += vkb (D becp), here with D folded into the projectors) for this handle: on the int8 tensor
 * cores (exact modular emulation of the FP64 product with nmods (12..16, default 16) moduli, as
 * b200_zgemm_i8) for H|psi> calls of at least 48 bands (mode 1, the default) or for every call (mode 2),
 * else cuBLAS ZGEMM (mode 0, and narrower calls in mode 1: the int8 path reads the projectors' whole
 * residue form per call).  Modes 1 and 2 keep the projectors also in residue form (2 x nmods bytes per
 * projector entry and spin) and each H|psi> caller about 6 x nmods bytes per psi entry of scratch.
 * Rebuilds the projector forms of every k-point (synchronous). */
int b200_hamilt_set_fp64_gemm(b200_hamilt* h, int mode, int nmods);
/* Bands per stick-buffer chunk of this handle's local pass (0 = the default: the largest chunk whose
 * stick buffer stays within 48 MB).  What b200_hamilt_autotune sets.  No counterpart in the reference. */
int b200_hamilt_set_band_chunk(b200_hamilt* h, int chunk);

/* ---- psi -> rho (ElecStatePW::psiToRho, module_elecstate/elecstate_pw.cpp:78-216) ---- */
/* elecstate::elecstate_pw_op<FP, DEVICE_GPU> (module_elecstate/kernels/elecstate_op.h):
 * rho[spin][ir] += w1 * |wfcr[ir]|^2.  rho is a host array of device pointers, as the reference's FPTYPE**. */
int b200_elecstate_pw_op_f64(int spin, int nrxx, double w1, double* const* rho, const void* wfcr_d, void* stream);
int b200_elecstate_pw_op_f32(int spin, int nrxx, float w1, float* const* rho, const void* wfcr_d, void* stream);
/* the nspin = 4 overload (DOMAG, DOMAG_Z, four rho components) */
int b200_elecstate_pw_op_nc_f64(int domag, int domag_z, int nrxx, double w1, double* const* rho, const void* wfcr_d,
                                const void* wfcr_another_spin_d, void* stream);
int b200_elecstate_pw_op_nc_f32(int domag, int domag_z, int nrxx, float w1, float* const* rho, const void* wfcr_d,
                                const void* wfcr_another_spin_d, void* stream);
/* The band loop of psiToRho for k-point ik (collinear): for every band with w1[ib] != 0,
 * rho_d[r] += w1[ib] * |psi_ib(r)|^2, psi(r) = recip_to_real of band ib (psi_d + ib*ld).
 * w1: host array of nbands weights (wg(ik, ib) / omega in the reference); rho_d: nx*ny*nz in ABACUS's
 * r order, accumulated into. */
int b200_pw_basis_psi_to_rho_f64(b200_pw_basis* b, int ik, int nbands, int ld, const void* psi_d, const double* w1,
                                 double* rho_d, void* stream);
int b200_pw_basis_psi_to_rho_f32(b200_pw_basis* b, int ik, int nbands, int ld, const void* psi_d, const double* w1,
                                 float* rho_d, void* stream);

/* ---- projector generation (pseudopot_cell_vnl::getvnl, VNL_in_pw.cpp:412-540) ---- */
/* ModuleBase::cal_ylm_real_op<FP, DEVICE_GPU> (module_base/kernels/math_op.h): real Y_lm of ng vectors
 * g (ng x 3) into ylm ((lmax+1)^2 x ng), lmax <= 4.  The reference's scratch p is internal here. */
int b200_cal_ylm_real_op_f64(int ng, int lmax, const double* g_d, double* ylm_d, void* stream);
int b200_cal_ylm_real_op_f32(int ng, int lmax, const float* g_d, float* ylm_d, void* stream);
/* hamilt::cal_sk_op<FP, DEVICE_GPU> (kernels/wf_op.h): structure factor sk (nat x npw complex).
 * atom_na is a host array of ntype counts; every other pointer is device memory, as the reference's. */
int b200_cal_sk_op_f64(int ik, int ntype, int nx, int ny, int nz, int rho_nx, int rho_ny, int rho_nz, int npw, int npwx,
                       int fftny, int eigts1_nc, int eigts2_nc, int eigts3_nc, const int* atom_na,
                       const int* igl2isz_d, const int* is2fftixy_d, double two_pi, const double* kvec_c_d,
                       const double* atom_tau_d, const void* eigts1_d, const void* eigts2_d, const void* eigts3_d,
                       void* sk_d, void* stream);
int b200_cal_sk_op_f32(int ik, int ntype, int nx, int ny, int nz, int rho_nx, int rho_ny, int rho_nz, int npw, int npwx,
                       int fftny, int eigts1_nc, int eigts2_nc, int eigts3_nc, const int* atom_na,
                       const int* igl2isz_d, const int* is2fftixy_d, float two_pi, const float* kvec_c_d,
                       const float* atom_tau_d, const void* eigts1_d, const void* eigts2_d, const void* eigts3_d,
                       void* sk_d, void* stream);
/* hamilt::cal_vnl_op<FP, DEVICE_GPU> (kernels/vnl_op.h:58-100): vkb (nkb x npwx complex, entries < npw
 * written) from gk, ylm, the radial table and sk.  atom_na / atom_nb / atom_nh are host arrays (ntype <= 8;
 * the reference copies them to the device first, VNL_in_pw.cpp:467-473); vkb1_d is accepted and unused
 * (the product kernel keeps that intermediate in registers). */
int b200_cal_vnl_op_f64(int ntype, int npw, int npwx, int nhm, int tab_2, int tab_3, const int* atom_na,
                        const int* atom_nb, const int* atom_nh, double dq, double tpiba, const double* gk_d,
                        const double* ylm_d, const double* indv_d, const double* nhtol_d, const double* nhtolm_d,
                        const double* tab_d, double* vkb1_d, const void* sk_d, void* vkb_d, void* stream);
int b200_cal_vnl_op_f32(int ntype, int npw, int npwx, int nhm, int tab_2, int tab_3, const int* atom_na,
                        const int* atom_nb, const int* atom_nh, float dq, float tpiba, const float* gk_d,
                        const float* ylm_d, const float* indv_d, const float* nhtol_d, const float* nhtolm_d,
                        const float* tab_d, float* vkb1_d, const void* sk_d, void* vkb_d, void* stream);
/* Projector tables of the handle's cell (the state pseudopot_cell_vnl::init_vnl prepares): per type na,
 * nbeta, nh; per (type, ih) indv / nhtol / nhtolm (host, ntype x nhm); the radial table tab
 * (host, ntype x tab_2 x tab_3, step dq in bohr^-1, the 4-pi/sqrt(omega) factor included); atom positions
 * tau (host, nat x 3, units of lat0, grouped by type).  The table must reach past the cut-off. */
int b200_hamilt_set_projectors(b200_hamilt* h, int ntype, const int* na, const int* nbeta, const int* nh, int nhm,
                               int lmax, const int* indv, const int* nhtol, const int* nhtolm, int tab_2, int tab_3,
                               double dq, const double* tab, const double* tau);
/* getvnl for k-point ik into the handle's projectors (FP64 and the FP32 copy), one fused launch;
 * replaces any b200_hamilt_set_vkb of that k-point. */
int b200_hamilt_build_vkb(b200_hamilt* h, int ik, void* stream);
/* Copies the handle's FP64 projectors of k-point ik (nkb x npwk_max complex128) to vkb_d. */
int b200_hamilt_copy_vkb(const b200_hamilt* h, int ik, void* vkb_d, void* stream);

/* gemm_op<std::complex<float>, DEVICE_GPU> (module_hsolver/kernels/math_kernel_op.h:240-265) on the
 * tensor cores: C = alpha * op(A) * B + beta * C, complex64 column-major, transa 'N' or 'C', transb 'N'.
 * Split precision (3xTF32: hi*hi + hi*lo + lo*hi, FP32 accumulate), about FP32 accuracy.
 * lda and ldb must be even and A, B 16-byte aligned (TMA row pitch); other shapes return
 * B200_STATUS_INVALID_ARGUMENT. */
int b200_tc_cgemm(char transa, char transb, int m, int n, int k, float alpha_re, float alpha_im, const void* a_d,
                  int lda, const void* b_d, int ldb, float beta_re, float beta_im, void* c_d, int ldc, void* stream);
/* Error word of the calling thread's tensor-core GEMMs (synchronous read, cleared by the read):
 * nonzero if a bounded wait inside a kernel ran out (the kernel then drained its own copies and
 * MMAs in flight, freed its tensor memory and returned without finishing its tile). */
int b200_tc_cgemm_error(int* code);
/* Time limit of each pipeline wait inside the tensor-core GEMMs launched after this call, in
 * nanoseconds (process-wide; 0 restores the default, 2 s).  No counterpart in the reference, whose
 * cuBLAS calls have no bounded waits: a test sets a limit that cannot be met and checks that
 * b200_tc_cgemm_error reports it and that the next GEMM with the default limit is correct. */
int b200_tc_set_wait_limit_ns(unsigned long long ns);

/* gemm_op<std::complex<double>, DEVICE_GPU> (math_kernel_op.h:240-265, cuda/math_kernel_op.cu:815-874) on
 * the int8 tensor cores: C = alpha op(A) B + beta C, complex128 column-major, transa 'N' or 'C', transb
 * 'N'; alpha, beta: host complex (2 doubles each).  Exact modular emulation of the FP64 product: every
 * row of op(A) and column of B is scaled by a power of two to integers, reduced modulo nmods (12..16)
 * coprime moduli <= 256, one int8 tcgen05 GEMM per modulus, and the product recombined by the Chinese
 * remainder theorem.  With nmods = 16 the largest entry of each row and column keeps all 53 bits and the
 * result is as accurate as an FP64 GEMM; NaN or infinite entries make the entries of C they reach NaN.
 * Stream-ordered; its scratch (about 16 bytes per entry of A and B) is kept per calling thread. */
int b200_zgemm_i8(char transa, char transb, int m, int n, int k, const double* alpha, const void* a_d, int lda,
                  const void* b_d, int ldb, const double* beta, void* c_d, int ldc, int nmods, void* stream);
/* Error word of the calling thread's int8 GEMMs (synchronous read of the legacy stream, cleared by the
 * read): nonzero if a bounded wait inside the GEMM kernel ran out (its output is then not valid). */
int b200_zgemm_i8_error(int* code);
/* Host copies of the recombination constants of b200_zgemm_i8 for nmods moduli: the moduli, the weights
 * w_l / M as wa + wb, M as a double, and the scale exponent q for real rows of length kr (every row is
 * scaled so that its largest magnitude is below 2^q).  No GPU needed; for tests of the scheme. */
int b200_zgemm_i8_constants(int nmods, long long kr, int* mods, double* wa, double* wb, double* mprod, int* q);

/* Measured arithmetic peaks of the current device in TFLOP/s (CUDA events on the legacy default
 * stream; one warm-up launch each): FP64 and FP32 fused multiply-add chains on the CUDA cores, and
 * FP64 tensor-core MMAs (mma.sync m8n8k4 f64).  The compute denominators of the rooflines.  No
 * counterpart in the reference. */
int b200_measure_peaks(double* fp64_tflops, double* fp32_tflops, double* dmma_tflops);

/* ---- FP64 BLAS functors of the Davidson / nonlocal path (module_hsolver/kernels/math_kernel_op.h) ----
 * gemm_op<std::complex<double>, DEVICE_GPU> (math_kernel_op.h:240-265, cuda/math_kernel_op.cu:815-874):
 * C = alpha op(A) op(B) + beta C, column-major, trans 'N' / 'T' / 'C'; alpha, beta: host complex
 * (2 doubles each).  cuBLAS ZGEMM, as the reference. */
int b200_gemm_op_f64(char transa, char transb, int m, int n, int k, const double* alpha, const void* a_d, int lda,
                     const void* b_d, int ldb, const double* beta, void* c_d, int ldc, void* stream);
/* gemv_op<std::complex<double>, DEVICE_GPU> (math_kernel_op.h:214-237, cuda/math_kernel_op.cu:741-792):
 * y = alpha op(A) x + beta y.  The reference passes incx as y's increment; incy is used here (the same
 * for the reference's callers, which pass incx == incy). */
int b200_gemv_op_f64(char trans, int m, int n, const double* alpha, const void* a_d, int lda, const void* x_d,
                     int incx, const double* beta, void* y_d, int incy, void* stream);
/* dot_real_op<std::complex<T>, DEVICE_GPU> (math_kernel_op.h:86-104, cuda/math_kernel_op.cu:468-506):
 * Re sum conj(L) R over dim complex entries, returned on the host (the call synchronises the stream);
 * reduce (the pool reduction) is the identity with one process per pool.  Deterministic two-pass sum. */
int b200_dot_real_op_f64(int dim, const void* psi_l_d, const void* psi_r_d, int reduce, double* result, void* stream);
int b200_dot_real_op_f32(int dim, const void* psi_l_d, const void* psi_r_d, int reduce, float* result, void* stream);

/* ------------------------------------------------------------------ Davidson
 * hsolver::DiagoDavid<T, DEVICE_GPU> (module_hsolver/diago_david.h:19-84):
 * constructor (precondition, nband, dim, david_ndim, use_paw = false) and
 * diag(hpsi_func, spsi_func, ldPsi, psi_in, eigenvalue_in, thr, maxiter, ntry_max, notconv_max)
 * (diago_david.cpp:1173-1200).  S = I (norm-conserving).  precondition_d is a device array of dim. */
int b200_david_create(int nband, int dim, int david_ndim, int precision, const double* precondition_d,
                      b200_david** out);
int b200_david_destroy(b200_david* d);
/* HPsiFunc (diago_david.h:57): hpsi(X, HX, nvec, dim, id_start, id_end) with X the base pointer of
 * the block (vectors of length dim at X + m*dim) and HX already offset to vector id_start.
 * Returns 0 on success; any other value abandons the solve, which then returns
 * B200_STATUS_CALLBACK_ERROR (the reference's HPsiFunc returns void and has no failure path).
 * Ordering: the solver's stream is synchronised before the call, so X may be read on any stream or
 * from the host.  The callback's writes to HX must be complete when it returns, or queued on the
 * legacy default stream (the solver's stream waits for that stream before it reads HX); work left on
 * another stream is not waited for. */
typedef int (*b200_hpsi_cb)(void* user, const void* x_d, void* hx_d, int nvec, int dim, int id_start, int id_end);
/* psi_d: nband vectors at psi_d + m*ldpsi (complex128 for FP64, complex128 for mixed: the solver
 * demotes internally); eigenvalue: host array of nband doubles; returns iterations in *iters. */
int b200_david_diag(b200_david* d, b200_hpsi_cb hpsi, void* user, int ldpsi, void* psi_d, double* eigenvalue,
                    double thr, int maxiter, int ntry_max, int notconv_max, int* iters);
/* Same, with H|psi> taken from a Hamiltonian handle at k-point ik (no host callback per block). */
int b200_david_diag_hamilt(b200_david* d, b200_hamilt* h, int ik, int spin, int ldpsi, void* psi_d,
                           double* eigenvalue, double thr, int maxiter, int ntry_max, int notconv_max, int* iters);

/* Stream on which the solver runs all its work (default NULL = legacy default stream, as the
 * reference).  Solvers on different streams run concurrently; each solver handle owns its own
 * H|psi> scratch, so several solvers may share one Hamiltonian handle. */
int b200_david_set_stream(b200_david* d, void* stream);
/* Verbosity of the solver (the role of DiagoDavid's test_david, diago_david.cpp:53-58):
 * 0 = quiet, 1 = one line per iteration on stderr. */
int b200_david_set_verbosity(b200_david* d, int level);
/* Mixed precision only: eigenvalue-change threshold at which the FP32 stage hands over to the
 * FP64 refinement (default 1e-7 Ry; never below the requested thr). */
int b200_david_set_mixed_threshold(b200_david* d, double thr);
/* FP64 subspace products of the solver (GEMMs of cal_grad, cal_elem, the orthogonalisation and refresh,
 * the reference's gemm_op<complex<double>> calls in diago_david.cpp): 0 = cuBLAS ZGEMM (the default);
 * 1 = the int8 tensor-core emulation of b200_zgemm_i8 in the FP64 refinement sweep of a mixed solve;
 * 2 = the int8 emulation in every FP64 iteration; 1 and 2 take it for the products on which it is
 * faster (m n / (m + n) >= 256 and k >= 128 for an m x n result over k terms), cuBLAS for the others;
 * 3 = the int8 emulation for every product of every FP64 iteration.  The emulation's operand residues
 * and products are device workspaces grown at their first use.  No counterpart in the reference. */
int b200_david_set_fp64_gemm(b200_david* d, int mode);
/* Statistics of the last solve: Davidson iterations in the FP32 stage (mixed only), in FP64,
 * and the number of single-band H applications (all stages). */
int b200_david_stats(const b200_david* d, int* iters_low, int* iters_fp64, int* hpsi_bands);
/* Mixed precision only: subspace size factor of the FP32 stage (nbase_x = ndim * nband, ndim >= 2;
 * default: the solver's david_ndim).  No counterpart in the reference. */
int b200_david_set_low_ndim(b200_david* d, int ndim);
/* Eigenvalue trace (no counterpart in the reference): with on != 0 the next solves record, per
 * iteration, the seconds since the solve began (taken when that iteration's eigenvalues reach the host
 * for the convergence test), the stage (0 = FP64, 1 = FP32) and the nband Ritz values.
 * b200_david_trace copies up to max_iters records (t, stage: max_iters entries; eig: max_iters x nband,
 * any may be NULL) of the last solve and sets *n_out to the number recorded. */
int b200_david_set_trace(b200_david* d, int on);
int b200_david_trace(b200_david* d, int max_iters, int nband, double* t, int* stage, double* eig, int* n_out);

/* ------------------------------------------------------------------ Davidson with subspace rotation
 * hsolver::Diago_DavSubspace<T, DEVICE_GPU> (module_hsolver/diago_dav_subspace.h:20-40), FP64:
 * constructor (precondition, nband, nbasis, david_ndim, diag_thr, diag_nmax, need_subspace, comm) with a
 * single-rank comm; precondition_d is a device array of dim (HSolverPW passes |k+G|^2 tpiba2 for this
 * method, hsolver_pw.cpp:573-580).  The subspace problem is the generalised (hcc, scc) one of the
 * reference's CPU branch (diago_dav_subspace.cpp:628-652). */
int b200_dav_subspace_create(int nband, int dim, int david_ndim, double diag_thr, int diag_nmax, int need_subspace,
                             const double* precondition_d, b200_dav_subspace** out);
int b200_dav_subspace_destroy(b200_dav_subspace* d);
/* diag(hpsi_func, psi_in, psi_in_dmax, eigenvalue_in, is_occupied, scf_type) (diago_dav_subspace.cpp:804-838):
 * psi_d: nband complex128 vectors at psi_d + m*psi_in_dmax (psi_in_dmax >= dim), replaced by the Ritz
 * vectors; eigenvalue: host, nband; is_occupied: host, nband flags, or NULL for all occupied (an empty
 * band converges at max(5 diag_thr, 1e-5)); scf_type: 1 = SCF (stop once at most 5 bands are unconverged),
 * 0 = NSCF (retry until all converge, up to 6 tries).  hpsi has the b200_hpsi_cb contract, called with the
 * solver's own block (vectors at stride dim).  Returns the total iterations in *iters. */
int b200_dav_subspace_diag(b200_dav_subspace* d, b200_hpsi_cb hpsi, void* user, void* psi_d, int psi_in_dmax,
                           double* eigenvalue, const int* is_occupied, int scf_type, int* iters);
/* Same, with H|psi> taken from a Hamiltonian handle at k-point ik. */
int b200_dav_subspace_diag_hamilt(b200_dav_subspace* d, b200_hamilt* h, int ik, int spin, void* psi_d,
                                  int psi_in_dmax, double* eigenvalue, const int* is_occupied, int scf_type,
                                  int* iters);
/* Stream of all the solver's work (default NULL = legacy default stream); verbosity 1 = one line per
 * iteration on stderr. */
int b200_dav_subspace_set_stream(b200_dav_subspace* d, void* stream);
int b200_dav_subspace_set_verbosity(b200_dav_subspace* d, int level);
/* Last solve: unconverged bands (the reference's notconv) and single-band H applications. */
int b200_dav_subspace_stats(const b200_dav_subspace* d, int* notconv, int* hpsi_bands);

/* ------------------------------------------------------------------ band-parallel CG
 * hsolver::DiagoBPCG<T, DEVICE_GPU> (module_hsolver/diago_bpcg.h:18-337), FP64: the constructor
 * DiagoBPCG(precondition) and init_iter(psi) (nband, nbasis) in one call; precondition_d: device array
 * of nbasis (HSolverPW: 1 + g2 + sqrt(1 + (g2 - 1)^2) on the plane waves, 1 on the padding). */
int b200_bpcg_create(const double* precondition_d, int nband, int nbasis, b200_bpcg** out);
int b200_bpcg_destroy(b200_bpcg* d);
/* diag(hamilt, psi, eigenvalue) (diago_bpcg.cpp:254-306) with DiagoIterAssist::SCF_ITER = scf_iter
 * (1 = the first SCF step: up to 24 iterations with a Rayleigh-Ritz every 4; otherwise up to 4):
 * psi_d: nband complex128 vectors of nbasis entries, contiguous, replaced; eigenvalue: host, nband;
 * hpsi: the b200_hpsi_cb contract, always called for all nband vectors (id_start 0, id_end nband-1,
 * dim = nbasis).  *iters (or NULL): iterations of the CG loop. */
int b200_bpcg_diag(b200_bpcg* d, b200_hpsi_cb hpsi, void* user, void* psi_d, double* eigenvalue, int scf_iter,
                   int* iters);
/* Same, with H|psi> taken from a Hamiltonian handle at k-point ik (entries npwk..nbasis-1 of every H|psi>
 * zeroed, as the reference's operator chain leaves them). */
int b200_bpcg_diag_hamilt(b200_bpcg* d, b200_hamilt* h, int ik, int spin, void* psi_d, double* eigenvalue,
                          int scf_iter, int* iters);
int b200_bpcg_set_stream(b200_bpcg* d, void* stream);
/* Last diag: largest residual norm of its last iteration and the single-band H applications. */
int b200_bpcg_stats(const b200_bpcg* d, double* max_err, int* hpsi_bands);

/* Davidson solves of nk k-points of one Hamiltonian handle, nworkers at a time on separate streams
 * (the k loop of HSolverPW::solve, hsolver_pw.cpp:240-270, with the k-points running concurrently).
 * precision: B200_PREC_FP64 or B200_PREC_MIXED; precond_d / psi_d: host arrays of nk device pointers
 * (psi_d[q]: complex128, nband vectors at ldpsi); eigenvalues: host, nk x nband; iters: host, nk
 * (or NULL).  Each k-point's result is the same as a b200_david_diag_hamilt solve of it alone. */
int b200_solve_kpoints(b200_hamilt* h, int nk, const int* iks, int spin, int nband, int david_ndim, int precision,
                       const double* const* precond_d, void* const* psi_d, int ldpsi, double* eigenvalues, double thr,
                       int maxiter, int ntry_max, int notconv_max, int nworkers, int* iters);
/* The same Davidson for nk k-points of one pool advanced in lock-step (HSolverPW::solve's k loop,
 * hsolver_pw.cpp:240-270, around DiagoDavid, diago_david.cpp:151-341): every phase of an iteration
 * is one batched call for all k (H|psi> of every k's new vectors through one local pass per FFT
 * pass, strided-batched subspace products, batched FP64 Cholesky-QR, one batched FP64 subspace
 * eigensolver call) and the convergence test runs on the device (one small read per iteration).
 * precision: B200_PREC_FP64, or B200_PREC_MIXED (an FP32 stage to 1e-7, then the FP64 iteration
 * from its vectors).
 * k-points with fewer unconverged bands pad their new block with zero columns kept out of the
 * subspace problem; all k-points restart together when the common basis would exceed
 * david_ndim*nband.  precond_d / psi_d: host arrays of nk device pointers; psi_d[q] holds nband
 * vectors at m*ldpsi (ldpsi >= the largest npwk of the batch) and receives the eigenvectors;
 * eigenvalues: host nk x nband; iters: host nk, the iteration after which each k-point had
 * converged (may be NULL).  1 <= nk <= 128.  Runs on stream (NULL = legacy default). */
int b200_solve_kpoints_batched(b200_hamilt* h, int nk, const int* iks, int spin, int nband, int david_ndim,
                               int precision, const double* const* precond_d, void* const* psi_d, int ldpsi,
                               double* eigenvalues, double thr, int maxiter, int* iters, void* stream);

/* ---- serving: non-self-consistent band solves with continuous admission (no counterpart in the
 * reference, whose NSCF driver solves its k-points one after another, hsolver_pw.cpp:212-299) ----
 * A server owns nworkers threads, each with its own non-blocking stream.  Cells are Hamiltonian handles
 * with V_eff, D and the projectors of all their k-points set; they stay resident.  A request (cell,
 * k-point, nbands, precision, thr, seed) is queued; a worker that falls idle takes the oldest queued
 * request whose cell has fewer than max_inflight requests running and whose solver slot is pooled or fits
 * in the HBM budget (idle slots of other shapes are released to make room); requests of one cell are
 * served first come, first served.  Start vectors are generated on the device from the seed, so a result does
 * not depend on the other requests in flight.  Times are seconds since the server was created. */
typedef struct b200_server b200_server;
int b200_server_create(unsigned long long hbm_budget_bytes, int nworkers, int david_ndim, b200_server** out);
int b200_server_destroy(b200_server* s);
int b200_server_add_cell(b200_server* s, b200_hamilt* h, int max_inflight, int* cell_id);
/* eig_out (host, nbands doubles) must stay valid until the request is reported by b200_server_poll. */
int b200_server_submit(b200_server* s, int cell, int ik, int nbands, int precision, double thr, int maxiter,
                       unsigned long long seed, double* eig_out, long long* req_id);
/* Reports up to max_out completed requests (wait != 0: blocks until one is done or none is outstanding):
 * id, status (B200_STATUS_*), submit / admit / completion times, Davidson iterations (all stages and
 * the low-precision stage).  The message of the last failed request reported is b200_last_error(). */
int b200_server_poll(b200_server* s, int max_out, int wait, long long* ids, int* status, double* t_submit,
                     double* t_admit, double* t_done, int* iters, int* iters_low, int* n_out);
/* Blocks until every submitted request has completed. */
int b200_server_drain(b200_server* s);
/* Admission policy of the server (no counterpart in the reference, which has no serving mode).
 * policy 0: the oldest admissible request first (first come, first served); 1: highest response ratio
 * first, (waiting time + S_c) / S_c over the oldest request of each cell c, with S_c a running mean of
 * the cell's service time (short cells go first, a long wait raises any request).  shed_factor > 0:
 * a queued request that has waited longer than shed_factor * S_c is completed with B200_STATUS_SHED
 * instead of being run (bounded latency under overload); 0 never sheds.  Default: 0 and 0. */
int b200_server_set_policy(b200_server* s, int policy, double shed_factor);
/* Express workers (no counterpart in the reference): workers 0 .. nworkers-1 take only requests of cells
 * whose running mean service time is at most max_service_s (cells not yet timed included), so that short
 * solves never wait behind a full set of long ones; the other workers serve every cell under the
 * admission policy.  nworkers in 0 .. (workers of the server) - 1; 0 (the default) turns it off. */
int b200_server_set_express(b200_server* s, int nworkers, double max_service_s);
/* out6: pooled slot bytes, peak pooled bytes, peak requests in flight, slots created, slots evicted,
 * seconds since creation. */
int b200_server_stats(b200_server* s, double* out6);

#ifdef __cplusplus
}
#endif
#endif /* ABACUS_B200_H */
