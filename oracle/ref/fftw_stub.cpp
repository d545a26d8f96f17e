// Test infrastructure (oracle build only): link-time stand-ins for the FFTW routines the reference's fft.cpp
// names (declared in oracle/ref/include/fftw3.h).  Only the PW_Basis_K set-up of the reference is run through
// them, to compare its index maps with this library's: buffers are allocated, plans are placeholders, and a
// plan that is executed throws, so no transform is ever computed here.
#include <cstdlib>
#include <stdexcept>

#include "fftw3.h"

namespace {
struct Placeholder {
    int unused;
} g_plan;
fftw_plan dplan() { return reinterpret_cast<fftw_plan>(&g_plan); }
fftwf_plan fplan() { return reinterpret_cast<fftwf_plan>(&g_plan); }
[[noreturn]] void no_transform() {
    throw std::runtime_error("FFT executed through the oracle's FFTW stand-in: no transform is available here");
}
}  // namespace

extern "C" {
void* fftw_malloc(size_t n) { return std::malloc(n > 0 ? n : 1); }
void fftw_free(void* p) { std::free(p); }
fftw_plan fftw_plan_many_dft(int, const int*, int, fftw_complex*, const int*, int, int, fftw_complex*, const int*, int,
                             int, int, unsigned) { return dplan(); }
fftw_plan fftw_plan_many_dft_r2c(int, const int*, int, double*, const int*, int, int, fftw_complex*, const int*, int,
                                 int, unsigned) { return dplan(); }
fftw_plan fftw_plan_many_dft_c2r(int, const int*, int, fftw_complex*, const int*, int, int, double*, const int*, int,
                                 int, unsigned) { return dplan(); }
fftw_plan fftw_plan_dft_3d(int, int, int, fftw_complex*, fftw_complex*, int, unsigned) { return dplan(); }
void fftw_execute_dft(const fftw_plan, fftw_complex*, fftw_complex*) { no_transform(); }
void fftw_execute_dft_r2c(const fftw_plan, double*, fftw_complex*) { no_transform(); }
void fftw_execute_dft_c2r(const fftw_plan, fftw_complex*, double*) { no_transform(); }
void fftw_destroy_plan(fftw_plan) {}
fftwf_plan fftwf_plan_many_dft(int, const int*, int, fftwf_complex*, const int*, int, int, fftwf_complex*, const int*,
                               int, int, int, unsigned) { return fplan(); }
fftwf_plan fftwf_plan_many_dft_r2c(int, const int*, int, float*, const int*, int, int, fftwf_complex*, const int*, int,
                                   int, unsigned) { return fplan(); }
fftwf_plan fftwf_plan_many_dft_c2r(int, const int*, int, fftwf_complex*, const int*, int, int, float*, const int*, int,
                                   int, unsigned) { return fplan(); }
void fftwf_execute_dft(const fftwf_plan, fftwf_complex*, fftwf_complex*) { no_transform(); }
void fftwf_execute_dft_r2c(const fftwf_plan, float*, fftwf_complex*) { no_transform(); }
void fftwf_execute_dft_c2r(const fftwf_plan, fftwf_complex*, float*) { no_transform(); }
void fftwf_destroy_plan(fftwf_plan) {}
}
