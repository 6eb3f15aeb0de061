// Oracle build shim (test infrastructure only): link-time stand-ins for the
// FFTW 3 single-precision symbols declared in shim/fftw3.h, which the
// reference's lib/fft.cpp calls (FFTW is not installed here). The batched
// 1-D real transforms the Fourier-domain FFA uses are computed from the DFT
// definition in double and rounded to float, with FFTW's conventions:
//   r2c: X[m] = sum_j x[j] exp(-2 pi i m j / n), m = 0 .. n/2 (unscaled);
//   c2r: x[j] = Re X[0] + 2 sum_{0<m<n/2} Re(X[m] exp(+2 pi i m j / n))
//               + Re X[n/2] (-1)^j for even n (unscaled; the imaginary
//               parts of X[0] and X[n/2] are not used).
// The 2-D plans (matched filter only) and FFTW's own allocators throw.
#include <cmath>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "fftw3.h"

namespace {
[[noreturn]] void unavailable(const char* what) {
    throw std::logic_error(std::string("oracle shim: ") + what +
                           " is not available (FFTW is not linked)");
}
} // namespace

struct fftwf_plan_s {
    bool r2c;
    int n, howmany, idist, odist;
    void* in;
    void* out;
    std::vector<double> c, s; // cos / sin of 2 pi t / n
};

namespace {
fftwf_plan make_plan(bool r2c, int n, int howmany, void* in, int idist, void* out, int odist) {
    auto* p = new fftwf_plan_s{r2c, n, howmany, idist, odist, in, out, {}, {}};
    p->c.resize(static_cast<std::size_t>(n));
    p->s.resize(static_cast<std::size_t>(n));
    const double two_pi = 6.283185307179586476925286766559;
    for (int t = 0; t < n; ++t) {
        p->c[t] = std::cos(two_pi * t / n);
        p->s[t] = std::sin(two_pi * t / n);
    }
    return p;
}

void run(const fftwf_plan_s* p, void* in, void* out) {
    const int n = p->n, nbf = n / 2 + 1;
    // the batch is split over the OpenMP threads, as FFTW's threaded plans do
#pragma omp parallel for schedule(static)
    for (int b = 0; b < p->howmany; ++b) {
        if (p->r2c) {
            const float* x = static_cast<const float*>(in) + static_cast<std::ptrdiff_t>(b) * p->idist;
            float* y = reinterpret_cast<float*>(static_cast<fftwf_complex*>(out) +
                                                static_cast<std::ptrdiff_t>(b) * p->odist);
            for (int m = 0; m < nbf; ++m) {
                double re = 0.0, im = 0.0;
                for (int j = 0; j < n; ++j) {
                    const int t = static_cast<int>((static_cast<long>(m) * j) % n);
                    re += x[j] * p->c[t];
                    im -= x[j] * p->s[t];
                }
                y[2 * m] = static_cast<float>(re);
                y[2 * m + 1] = static_cast<float>(im);
            }
        } else {
            const float* x = reinterpret_cast<const float*>(static_cast<fftwf_complex*>(in) +
                                                            static_cast<std::ptrdiff_t>(b) * p->idist);
            float* y = static_cast<float*>(out) + static_cast<std::ptrdiff_t>(b) * p->odist;
            for (int j = 0; j < n; ++j) {
                double acc = x[0];
                for (int m = 1; m < nbf; ++m) {
                    const int t = static_cast<int>((static_cast<long>(m) * j) % n);
                    const double re = x[2 * m] * p->c[t] - x[2 * m + 1] * p->s[t];
                    acc += (2 * m == n) ? re : 2.0 * re;
                }
                y[j] = static_cast<float>(acc);
            }
        }
    }
}

void check_layout(int rank, const int* inembed, int istride, const int* onembed, int ostride) {
    if (rank != 1 || inembed != nullptr || onembed != nullptr || istride != 1 || ostride != 1) {
        unavailable("an FFTW plan other than a contiguous batch of 1-D transforms");
    }
}
} // namespace

extern "C" {
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int) {}
void fftwf_cleanup_threads(void) {}
void fftwf_cleanup(void) {}
void fftw_cleanup(void) {}
fftwf_complex* fftwf_alloc_complex(std::size_t) { unavailable("fftwf_alloc_complex"); }
float* fftwf_alloc_real(std::size_t) { unavailable("fftwf_alloc_real"); }
void fftwf_free(void* p) { std::free(p); }
void fftwf_destroy_plan(fftwf_plan p) { delete p; }
void fftwf_execute(const fftwf_plan p) { run(p, p->in, p->out); }
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out) {
    if (!p->r2c) {
        unavailable("fftwf_execute_dft_r2c on a c2r plan");
    }
    run(p, in, out);
}
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out) {
    if (p->r2c) {
        unavailable("fftwf_execute_dft_c2r on an r2c plan");
    }
    run(p, in, out);
}
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany, float* in, const int* inembed,
                                   int istride, int idist, fftwf_complex* out, const int* onembed,
                                   int ostride, int odist, unsigned) {
    check_layout(rank, inembed, istride, onembed, ostride);
    return make_plan(true, *n, howmany, in, idist, out, odist);
}
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany, fftwf_complex* in,
                                   const int* inembed, int istride, int idist, float* out,
                                   const int* onembed, int ostride, int odist, unsigned) {
    check_layout(rank, inembed, istride, onembed, ostride);
    return make_plan(false, *n, howmany, in, idist, out, odist);
}
fftwf_plan fftwf_plan_dft_r2c_2d(int, int, float*, fftwf_complex*, unsigned) {
    unavailable("fftwf_plan_dft_r2c_2d");
}
fftwf_plan fftwf_plan_dft_c2r_2d(int, int, fftwf_complex*, float*, unsigned) {
    unavailable("fftwf_plan_dft_c2r_2d");
}
}
