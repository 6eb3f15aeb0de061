// Oracle build shim (test infrastructure only): link-time stand-ins for the
// FFTW symbols declared in shim/fftw3.h. Nothing on the time-domain FP32 path
// reaches them; a call from the Fourier path throws instead of computing.
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "fftw3.h"

namespace {
[[noreturn]] void unavailable(const char* what) {
    throw std::logic_error(std::string("oracle shim: ") + what +
                           " is not available (FFTW is not linked)");
}
} // namespace

extern "C" {
int fftwf_init_threads(void) { return 0; }
void fftwf_plan_with_nthreads(int) {}
void fftwf_cleanup_threads(void) {}
void fftwf_cleanup(void) {}
void fftw_cleanup(void) {}
fftwf_complex* fftwf_alloc_complex(std::size_t) { unavailable("fftwf_alloc_complex"); }
float* fftwf_alloc_real(std::size_t) { unavailable("fftwf_alloc_real"); }
void fftwf_free(void* p) { std::free(p); }
void fftwf_destroy_plan(fftwf_plan) {}
void fftwf_execute(const fftwf_plan) { unavailable("fftwf_execute"); }
void fftwf_execute_dft_r2c(const fftwf_plan, float*, fftwf_complex*) {
    unavailable("fftwf_execute_dft_r2c");
}
void fftwf_execute_dft_c2r(const fftwf_plan, fftwf_complex*, float*) {
    unavailable("fftwf_execute_dft_c2r");
}
fftwf_plan fftwf_plan_many_dft_r2c(int, const int*, int, float*, const int*, int, int,
                                   fftwf_complex*, const int*, int, int, unsigned) {
    unavailable("fftwf_plan_many_dft_r2c");
}
fftwf_plan fftwf_plan_many_dft_c2r(int, const int*, int, fftwf_complex*, const int*, int,
                                   int, float*, const int*, int, int, unsigned) {
    unavailable("fftwf_plan_many_dft_c2r");
}
fftwf_plan fftwf_plan_dft_r2c_2d(int, int, float*, fftwf_complex*, unsigned) {
    unavailable("fftwf_plan_dft_r2c_2d");
}
fftwf_plan fftwf_plan_dft_c2r_2d(int, int, fftwf_complex*, float*, unsigned) {
    unavailable("fftwf_plan_dft_c2r_2d");
}
}
