// Test infrastructure (oracle build only): stand-ins for the FFTW routines the reference's fft.cpp names
// (declared in oracle/ref/include/fftw3.h; FFTW itself is absent here).  Plans record the layout of a batch
// of one-dimensional complex transforms (length n, howmany lines, element stride and line distance on input
// and output, sign); executing a plan evaluates each line's discrete Fourier transform directly,
//     y_k = sum_j x_j exp(sign * 2 pi i j k / n),  un-normalised,
// with the angle reduced exactly (j k mod n) and accumulated in long double.  That is O(n^2) per line, meant
// for the small grids of the parity tests, and lets the reference's own PW_Basis_K transforms
// (pw_transform_k.cpp) run as written.  Real-to-complex and 3-D plans, which the reference's non-gamma
// plane-wave transforms do not execute, throw when executed.
#include <cmath>
#include <complex>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "fftw3.h"

namespace {

struct Plan {
    int n = 0, howmany = 0, istride = 1, idist = 0, ostride = 1, odist = 0, sign = -1;
    bool c2c = true;
};

template <typename R> void run(const Plan& p, const R* in, R* out) {
    if (!p.c2c) throw std::runtime_error("the oracle's FFTW stand-in computes complex-to-complex lines only");
    const int n = p.n;
    const long double two_pi = 6.283185307179586476925286766559L;
    std::vector<std::complex<long double>> tw(n), x(n);
    for (int m = 0; m < n; ++m) {
        const long double a = p.sign * two_pi * static_cast<long double>(m) / static_cast<long double>(n);
        tw[m] = std::complex<long double>(std::cos(a), std::sin(a));
    }
    for (int t = 0; t < p.howmany; ++t) {
        const R* xi = in + 2L * t * p.idist;
        for (int j = 0; j < n; ++j) x[j] = std::complex<long double>(xi[2L * j * p.istride], xi[2L * j * p.istride + 1]);
        R* yo = out + 2L * t * p.odist;
        std::vector<std::complex<long double>> y(n);
        for (int k = 0; k < n; ++k) {
            std::complex<long double> s = 0.0L;
            for (int j = 0; j < n; ++j) s += x[j] * tw[(static_cast<long>(j) * k) % n];
            y[k] = s;
        }
        for (int k = 0; k < n; ++k) {
            yo[2L * k * p.ostride] = static_cast<R>(y[k].real());
            yo[2L * k * p.ostride + 1] = static_cast<R>(y[k].imag());
        }
    }
}

Plan* make(int rank, const int* n, int howmany, int istride, int idist, int ostride, int odist, int sign, bool c2c) {
    if (rank != 1) throw std::runtime_error("the oracle's FFTW stand-in plans one-dimensional transforms only");
    Plan* p = new Plan;
    p->n = n[0];
    p->howmany = howmany;
    p->istride = istride;
    p->idist = idist;
    p->ostride = ostride;
    p->odist = odist;
    p->sign = sign;
    p->c2c = c2c;
    return p;
}

}  // namespace

extern "C" {
void* fftw_malloc(size_t n) { return std::malloc(n > 0 ? n : 1); }
void fftw_free(void* p) { std::free(p); }
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex*, const int*, int istride, int idist,
                             fftw_complex*, const int*, int ostride, int odist, int sign, unsigned) {
    return reinterpret_cast<fftw_plan>(make(rank, n, howmany, istride, idist, ostride, odist, sign, true));
}
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double*, const int*, int istride, int idist,
                                 fftw_complex*, const int*, int ostride, int odist, unsigned) {
    return reinterpret_cast<fftw_plan>(make(rank, n, howmany, istride, idist, ostride, odist, -1, false));
}
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex*, const int*, int istride, int idist,
                                 double*, const int*, int ostride, int odist, unsigned) {
    return reinterpret_cast<fftw_plan>(make(rank, n, howmany, istride, idist, ostride, odist, +1, false));
}
fftw_plan fftw_plan_dft_3d(int, int, int, fftw_complex*, fftw_complex*, int, unsigned) {
    Plan* p = new Plan;
    p->c2c = false;  // executed only by the reference's own FFT tests, which do not run here
    return reinterpret_cast<fftw_plan>(p);
}
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) {
    run<double>(*reinterpret_cast<const Plan*>(p), &in[0][0], &out[0][0]);
}
void fftw_execute_dft_r2c(const fftw_plan, double*, fftw_complex*) {
    throw std::runtime_error("the oracle's FFTW stand-in computes complex-to-complex lines only");
}
void fftw_execute_dft_c2r(const fftw_plan, fftw_complex*, double*) {
    throw std::runtime_error("the oracle's FFTW stand-in computes complex-to-complex lines only");
}
void fftw_destroy_plan(fftw_plan p) { delete reinterpret_cast<Plan*>(p); }

fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany, fftwf_complex*, const int*, int istride, int idist,
                               fftwf_complex*, const int*, int ostride, int odist, int sign, unsigned) {
    return reinterpret_cast<fftwf_plan>(make(rank, n, howmany, istride, idist, ostride, odist, sign, true));
}
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany, float*, const int*, int istride, int idist,
                                   fftwf_complex*, const int*, int ostride, int odist, unsigned) {
    return reinterpret_cast<fftwf_plan>(make(rank, n, howmany, istride, idist, ostride, odist, -1, false));
}
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany, fftwf_complex*, const int*, int istride,
                                   int idist, float*, const int*, int ostride, int odist, unsigned) {
    return reinterpret_cast<fftwf_plan>(make(rank, n, howmany, istride, idist, ostride, odist, +1, false));
}
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out) {
    run<float>(*reinterpret_cast<const Plan*>(p), &in[0][0], &out[0][0]);
}
void fftwf_execute_dft_r2c(const fftwf_plan, float*, fftwf_complex*) {
    throw std::runtime_error("the oracle's FFTW stand-in computes complex-to-complex lines only");
}
void fftwf_execute_dft_c2r(const fftwf_plan, fftwf_complex*, float*) {
    throw std::runtime_error("the oracle's FFTW stand-in computes complex-to-complex lines only");
}
void fftwf_destroy_plan(fftwf_plan p) { delete reinterpret_cast<Plan*>(p); }
}
