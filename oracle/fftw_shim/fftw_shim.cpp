// ORACLE / TEST INFRASTRUCTURE ONLY.
// Implements the FFTW-API subset declared in fftw3.h on top of the project
// FFT engine (fft_engine.hpp).  Plans record rank, dims, sign and buffers;
// execute transforms `in` and leaves the result in `out` (in place when
// in == out, which is how PowerGrid/fftCPU.cpp uses them).
#include "fftw3.h"

#include <complex>
#include <cstring>

#include "../fft_engine.hpp"

namespace {
template <typename T>
struct PlanT {
  int rank;
  std::size_t dims[3];
  int sign;
  std::complex<T>* in;
  std::complex<T>* out;
  void run() const {
    std::size_t total = 1;
    for (int d = 0; d < rank; ++d) total *= dims[d];
    if (in != out) std::memcpy(out, in, sizeof(std::complex<T>) * total);
    pgo::fft_nd<T>(out, dims, rank, sign);
  }
};
}  // namespace

struct pg_fftwf_plan_s : PlanT<float> {};
struct pg_fftw_plan_s : PlanT<double> {};

extern "C" {

static fftwf_plan mkf(int rank, int n0, int n1, int n2, fftwf_complex* in, fftwf_complex* out, int sign) {
  fftwf_plan p = new pg_fftwf_plan_s;
  p->rank = rank;
  p->dims[0] = (std::size_t)n0; p->dims[1] = (std::size_t)n1; p->dims[2] = (std::size_t)n2;
  p->sign = sign;
  p->in = reinterpret_cast<std::complex<float>*>(in);
  p->out = reinterpret_cast<std::complex<float>*>(out);
  return p;
}
static fftw_plan mkd(int rank, int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign) {
  fftw_plan p = new pg_fftw_plan_s;
  p->rank = rank;
  p->dims[0] = (std::size_t)n0; p->dims[1] = (std::size_t)n1; p->dims[2] = (std::size_t)n2;
  p->sign = sign;
  p->in = reinterpret_cast<std::complex<double>*>(in);
  p->out = reinterpret_cast<std::complex<double>*>(out);
  return p;
}

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex* in, fftwf_complex* out, int sign, unsigned) { return mkf(1, n, 1, 1, in, out, sign); }
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex* in, fftwf_complex* out, int sign, unsigned) { return mkf(2, n0, n1, 1, in, out, sign); }
fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex* in, fftwf_complex* out, int sign, unsigned) { return mkf(3, n0, n1, n2, in, out, sign); }
void fftwf_execute(const fftwf_plan p) { p->run(); }
void fftwf_destroy_plan(fftwf_plan p) { delete p; }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned) { return mkd(1, n, 1, 1, in, out, sign); }
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned) { return mkd(2, n0, n1, 1, in, out, sign); }
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign, unsigned) { return mkd(3, n0, n1, n2, in, out, sign); }
void fftw_execute(const fftw_plan p) { p->run(); }
void fftw_destroy_plan(fftw_plan p) { delete p; }

}  // extern "C"
