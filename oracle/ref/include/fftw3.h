/* Test infrastructure (oracle build only): compile-time stand-in for FFTW's header.  The reference's
 * DiagoBPCG header reaches module_basis/module_pw/fft.h through structure_factor.h; that header names FFTW's
 * plan and complex types in class members but the solver calls no FFTW routine, so the types alone let the
 * solver compile without FFTW (absent here).  Nothing is linked against FFTW. */
#pragma once
typedef struct fftw_plan_s* fftw_plan;
typedef struct fftwf_plan_s* fftwf_plan;
typedef double fftw_complex[2];
typedef float fftwf_complex[2];
