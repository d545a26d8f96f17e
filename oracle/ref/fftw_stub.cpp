// Test infrastructure (oracle build only): stand-ins for the FFTW routines the reference's fft.cpp names
// (declared in oracle/ref/include/fftw3.h; FFTW itself is absent here).  Plans record the layout of a batch
// of one-dimensional complex transforms (length n, howmany lines, element stride and line distance on input
// and output, sign); executing a plan transforms each line,
//     y_k = sum_j x_j exp(sign * 2 pi i j k / n),  un-normalised,
// by a recursive mixed-radix decimation in time for lengths whose factors are 2, 3 and 5 (the reference's
// grid rule gives only those) and directly otherwise, with twiddles from long-double angles reduced exactly
// (j k mod n).  This lets the reference's own PW_Basis_K transforms and operators (pw_transform_k.cpp,
// veff_pw.cpp) run as written, fast enough to be timed as the CPU baseline.  Real-to-complex and 3-D plans,
// which the reference's non-gamma plane-wave transforms do not execute, throw when executed.
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

using cplx = std::complex<double>;

void fft_rec(const cplx* x, long s, int n, cplx* y, const cplx* w, int N, cplx* scratch);

// one line: the recursion needs, per level, an output block and a scratch block that do not alias its input;
// level buffers are allocated once per line length
void fft_line(const cplx* x, int n, cplx* y, const cplx* w, cplx* scratch, cplx*) {
    fft_rec(x, 1, n, y, w, n, scratch);
}

// y[0..n) = DFT of x[0], x[s], ..., x[(n-1)s] with twiddles w[j] = exp(sign 2 pi i j / N) of the top-level
// length N, of which this length n divides N (step = N / n); scratch holds at least n entries
void fft_rec(const cplx* x, long s, int n, cplx* y, const cplx* w, int N, cplx* scratch) {
    if (n == 1) {
        y[0] = x[0];
        return;
    }
    int p = 0;
    for (int f : {2, 3, 5})
        if (n % f == 0) {
            p = f;
            break;
        }
    const int step = N / n;
    if (p == 0) {  // no 2, 3 or 5 factor left: the direct sum
        for (int k = 0; k < n; ++k) {
            cplx acc = 0.0;
            for (int j = 0; j < n; ++j) acc += x[j * s] * w[(static_cast<long>(j) * k % n) * step];
            y[k] = acc;
        }
        return;
    }
    const int m = n / p;
    // sub-transforms of the p decimated sequences into scratch (p blocks of m), then the radix-p butterflies
    for (int r = 0; r < p; ++r) fft_rec(x + r * s, s * p, m, scratch + r * m, w, N, y);
    for (int k = 0; k < m; ++k) {
        cplx t[5];
        for (int r = 0; r < p; ++r) t[r] = scratch[r * m + k] * w[(static_cast<long>(r) * k % n) * step];
        for (int q = 0; q < p; ++q) {
            cplx acc = 0.0;
            for (int r = 0; r < p; ++r) acc += t[r] * w[(static_cast<long>(r) * q * m % n) * step];
            y[k + q * m] = acc;
        }
    }
}

template <typename R> void run(const Plan& p, const R* in, R* out) {
    if (!p.c2c) throw std::runtime_error("the oracle's FFTW stand-in computes complex-to-complex lines only");
    const int n = p.n;
    const long double two_pi = 6.283185307179586476925286766559L;
    std::vector<cplx> w(n), x(n), y(n), scratch(n), scratch2(n);
    for (int m = 0; m < n; ++m) {
        const long double a = p.sign * two_pi * static_cast<long double>(m) / static_cast<long double>(n);
        w[m] = cplx(static_cast<double>(std::cos(a)), static_cast<double>(std::sin(a)));
    }
    for (int t = 0; t < p.howmany; ++t) {
        const R* xi = in + 2L * t * p.idist;
        for (int j = 0; j < n; ++j) x[j] = cplx(xi[2L * j * p.istride], xi[2L * j * p.istride + 1]);
        fft_line(x.data(), n, y.data(), w.data(), scratch.data(), scratch2.data());
        R* yo = out + 2L * t * p.odist;
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
