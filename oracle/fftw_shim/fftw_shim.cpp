// The FFTW subset of fftw3.h (this directory) for the oracle build of the
// reference's cross-correlator. TEST INFRASTRUCTURE ONLY.
//
// fftwf_execute computes the real-to-complex transform of the plan's n
// float inputs in double precision -- a mixed-radix Cooley-Tukey recursion
// (decimation in time over the smallest prime factor, a direct sum for a
// prime length) with twiddles e^{-2 pi i m / n} taken at the integer phase
// m = (q k) mod n -- and stores bins 0 .. n/2 rounded to float. Its error is
// about 1e-15 relative, far below FFTW's own single-precision error, so the
// reference's outputs through this shim are the reference's arithmetic on
// (nearly) exact spectra. Plans hold no shared state: CrossCorr.cpp executes
// one plan per station from OpenMP threads.
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <vector>

struct ccfj_fftwf_plan_s {
  int n;
  float *in;
  fftwf_complex *out;
};

namespace {

using cd = std::complex<double>;

cd root(long long m, long long n) {  // e^{-2 pi i m / n}
  const double a = -2.0 * M_PI * (double)(m % n) / (double)n;
  return cd(std::cos(a), std::sin(a));
}

long long smallest_factor(long long n) {
  for (long long p = 2; p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;
}

// y[k] = sum_j x[j * stride] e^{-2 pi i j k / n}, k < n
void dft(const cd *x, long long stride, long long n, cd *y) {
  if (n == 1) {
    y[0] = x[0];
    return;
  }
  const long long p = smallest_factor(n);
  if (p == n) {  // prime length: direct sum
    for (long long k = 0; k < n; ++k) {
      cd s = 0;
      for (long long j = 0; j < n; ++j) s += x[j * stride] * root(j * k, n);
      y[k] = s;
    }
    return;
  }
  const long long m = n / p;
  std::vector<cd> sub(n);  // p sub-transforms of length m: inputs q, q + p, ...
  for (long long q = 0; q < p; ++q) dft(x + q * stride, stride * p, m, sub.data() + q * m);
  for (long long k = 0; k < n; ++k) {
    cd s = 0;
    for (long long q = 0; q < p; ++q) s += sub[q * m + k % m] * root(q * k, n);
    y[k] = s;
  }
}

}  // namespace

extern "C" {

float *fftwf_alloc_real(size_t n) { return static_cast<float *>(std::calloc(n ? n : 1, sizeof(float))); }

fftwf_complex *fftwf_alloc_complex(size_t n) {
  return static_cast<fftwf_complex *>(std::calloc(n ? n : 1, sizeof(fftwf_complex)));
}

void fftwf_free(void *p) { std::free(p); }

fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned) {
  fftwf_plan p = new ccfj_fftwf_plan_s;
  p->n = n;
  p->in = in;
  p->out = out;
  return p;
}

void fftwf_execute(const fftwf_plan p) {
  const long long n = p->n;
  std::vector<cd> x(n), y(n);
  for (long long j = 0; j < n; ++j) x[j] = cd(p->in[j], 0.0);
  dft(x.data(), 1, n, y.data());
  for (long long k = 0; k <= n / 2; ++k) {
    p->out[k][0] = (float)y[k].real();
    p->out[k][1] = (float)y[k].imag();
  }
}

void fftwf_destroy_plan(fftwf_plan p) { delete p; }

}  // extern "C"
