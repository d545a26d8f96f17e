/* Test infrastructure (oracle build only): compile-time stand-in for FFTW's API, as far as the reference's
 * sources in this oracle's builds name it (FFTW is absent here): DiagoBPCG's header reaches
 * module_basis/module_pw/fft.h, and the reference's PW_Basis_K set-up and transforms (pw_basis*.cpp, fft.cpp,
 * pw_transform_k.cpp) are compiled to compare their maps and transforms with this repository's.
 * oracle/ref/fftw_stub.cpp defines these routines: plans record a batch of one-dimensional complex lines,
 * executing one runs a mixed-radix (2, 3, 5) FFT on each line. */
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fftw_plan_s* fftw_plan;
typedef struct fftwf_plan_s* fftwf_plan;
typedef double fftw_complex[2];
typedef float fftwf_complex[2];

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed, int ostride, int odist, int sign,
                             unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int* inembed, int istride,
                                 int idist, fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed,
                                 int istride, int idist, double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_destroy_plan(fftw_plan p);

fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany, fftwf_complex* in, const int* inembed,
                               int istride, int idist, fftwf_complex* out, const int* onembed, int ostride, int odist,
                               int sign, unsigned flags);
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany, float* in, const int* inembed, int istride,
                                   int idist, fftwf_complex* out, const int* onembed, int ostride, int odist,
                                   unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany, fftwf_complex* in, const int* inembed,
                                   int istride, int idist, float* out, const int* onembed, int ostride, int odist,
                                   unsigned flags);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out);
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif
