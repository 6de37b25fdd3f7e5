// Arithmetic of the cross-correlation front end (xcorr.cu), written once
// for the device kernels and for host-side checks: every function here
// compiles with nvcc (host and device) and with a plain C++ compiler, where
// the tests drive it thread by thread.
//
// The reference computes, for every station pair, the average over the
// overlapping windows both stations keep of conj(X_a) X_b, where X is the
// (optionally one-bit, optionally whitened) real FFT of a window at bins
// j*fstride (src/CrossCorr.cpp:33-159). Here:
//
// * shift_range: the shifts k a station keeps form one interval [lo, hi]
//   (both tests of src/CrossCorr.cpp:88-95 are monotone in k), so a pair's
//   count is the length of the intersection of two intervals;
// * the real FFT of N = 2M samples is a complex FFT of z[m] = x[2m] +
//   i x[2m+1] (M points, self-sorting Stockham passes of radix 2, 3, 4, 5
//   or 8) followed by the split
//     X[k] = (Z[k] + conj Z[M-k]) / 2 - (i/2) e^{-i pi k/M} (Z[k] - conj Z[M-k]);
// * whiten: X / max(|X|, 1e-8) in float32, as the reference;
// * gram_step: one thread's share of a 16 x 16 station tile of
//   conj(X_a) X_b for one frequency lane.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define CC_HD __host__ __device__ __forceinline__
#else
#define CC_HD inline
#endif

namespace ccfj {
namespace xc {

struct alignas(8) Cpx {
  float re, im;
};

CC_HD Cpx cpx(float re, float im) {
  Cpx c;
  c.re = re;
  c.im = im;
  return c;
}
CC_HD Cpx cadd(Cpx a, Cpx b) { return cpx(a.re + b.re, a.im + b.im); }
CC_HD Cpx csub(Cpx a, Cpx b) { return cpx(a.re - b.re, a.im - b.im); }
CC_HD Cpx cmul(Cpx a, Cpx b) { return cpx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
CC_HD Cpx cscale(Cpx a, float s) { return cpx(a.re * s, a.im * s); }
// -i * a
CC_HD Cpx cmul_negi(Cpx a) { return cpx(a.im, -a.re); }
CC_HD Cpx cconj(Cpx a) { return cpx(a.re, -a.im); }

// ------------------------------------------------------------ small DFTs
// Forward DFT of R points in place, natural order:
// X[q] = sum_r v[r] exp(-2 pi i r q / R).
template <int R>
CC_HD void dft(Cpx* v);

template <>
CC_HD void dft<2>(Cpx* v) {
  const Cpx a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <>
CC_HD void dft<4>(Cpx* v) {
  const Cpx t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  const Cpx t2 = cadd(v[1], v[3]), t3 = cmul_negi(csub(v[1], v[3]));
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3);
  v[3] = csub(t1, t3);
}

template <>
CC_HD void dft<8>(Cpx* v) {
  // even and odd halves, then X[q] = E[q] + W8^q O[q], X[q+4] = E[q] - W8^q O[q]
  Cpx e[4] = {v[0], v[2], v[4], v[6]};
  Cpx o[4] = {v[1], v[3], v[5], v[7]};
  dft<4>(e);
  dft<4>(o);
  const float h = 0.70710678118654752f;  // 1/sqrt(2)
  const Cpx w1 = cmul(o[1], cpx(h, -h));
  const Cpx w2 = cmul_negi(o[2]);
  const Cpx w3 = cmul(o[3], cpx(-h, -h));
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], w1);
  v[5] = csub(e[1], w1);
  v[2] = cadd(e[2], w2);
  v[6] = csub(e[2], w2);
  v[3] = cadd(e[3], w3);
  v[7] = csub(e[3], w3);
}

template <>
CC_HD void dft<3>(Cpx* v) {
  // w = exp(-2 pi i / 3) = -1/2 - i sqrt(3)/2
  const float s3 = 0.86602540378443865f;
  const Cpx s = cadd(v[1], v[2]);
  const Cpx d = cscale(cmul_negi(csub(v[1], v[2])), s3);
  const Cpx m = csub(v[0], cscale(s, 0.5f));
  v[0] = cadd(v[0], s);
  v[1] = cadd(m, d);
  v[2] = csub(m, d);
}

template <>
CC_HD void dft<5>(Cpx* v) {
  // cos and sin of 2 pi / 5 and 4 pi / 5
  const float c1 = 0.30901699437494742f, s1 = 0.95105651629515357f;
  const float c2 = -0.80901699437494742f, s2 = 0.58778525229247313f;
  const Cpx s14 = cadd(v[1], v[4]), d14 = csub(v[1], v[4]);
  const Cpx s23 = cadd(v[2], v[3]), d23 = csub(v[2], v[3]);
  const Cpx x0 = v[0];
  const Cpx m1 = cadd(x0, cadd(cscale(s14, c1), cscale(s23, c2)));
  const Cpx m2 = cadd(x0, cadd(cscale(s14, c2), cscale(s23, c1)));
  const Cpx n1 = cmul_negi(cadd(cscale(d14, s1), cscale(d23, s2)));
  const Cpx n2 = cmul_negi(csub(cscale(d14, s2), cscale(d23, s1)));
  v[0] = cadd(x0, cadd(s14, s23));
  v[1] = cadd(m1, n1);
  v[4] = csub(m1, n1);
  v[2] = cadd(m2, n2);
  v[3] = csub(m2, n2);
}

// ------------------------------------------------------ Stockham passes
// One pass of radix R over M points, done by butterflies t = 0 .. M/R - 1
// after Ns points have been combined (Ns = product of the earlier radices).
// Butterfly t reads src[t + r M/R], twiddles input r by
// exp(-2 pi i (t mod Ns) r / (Ns R)) = tw[(t mod Ns) r M / (Ns R)], with
// tw[u] = exp(-2 pi i u / M), and writes dst[(t / Ns) Ns R + t mod Ns + q Ns].
// After the last pass (Ns R = M) dst holds the DFT in natural order. The
// load and the rest are separate so that a caller can run the pass in place
// (every load before any store).
template <int R>
CC_HD void bf_load(const Cpx* src, int M, int t, Cpx* v) {
  const int stride = M / R;
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = src[t + r * stride];
}

// w[r] = tw[r step] for 0 < r < R: the table entries of step, 2 step and
// (radix 8) 4 step, the other powers as products of those (one or two
// products deep). The twiddle indices of neighbouring butterflies lie far
// apart in the table, so fewer reads mean fewer cache wavefronts.
template <int R>
CC_HD void twiddle_powers(const Cpx* tw, int step, Cpx* w) {
  w[1] = tw[step];
  if (R >= 3) w[2 % R] = tw[2 * step];
  if (R >= 4) w[3 % R] = cmul(w[1], w[2 % R]);
  if (R == 5) w[4 % R] = cmul(w[2 % R], w[2 % R]);
  if (R == 8) {
    w[4 % R] = tw[4 * step];
    w[5 % R] = cmul(w[4 % R], w[1]);
    w[6 % R] = cmul(w[4 % R], w[2 % R]);
    w[7 % R] = cmul(w[4 % R], w[3 % R]);
  }
}

template <int R>
CC_HD void bf_finish(Cpx* dst, int M, int Ns, const Cpx* tw, int t, Cpx* v) {
  const int jn = t % Ns;
  if (jn != 0) {
    const int step = (M / (Ns * R)) * jn;
    Cpx w[R];
    twiddle_powers<R>(tw, step, w);
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
  }
  dft<R>(v);
  const int base = (t / Ns) * Ns * R + jn;
#pragma unroll
  for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
}

// Radices of a self-sorting plan for M points: 8s, then a 4 or 2, then 3s
// and 5s. Returns the number of passes, or 0 when M has another prime
// factor (or needs more than kMaxPasses passes).
constexpr int kMaxPasses = 24;
CC_HD int fft_plan(int M, int* radix) {
  if (M < 2) return 0;
  int n = 0;
  while (M % 8 == 0 && n < kMaxPasses) {
    radix[n++] = 8;
    M /= 8;
  }
  if (M % 4 == 0 && n < kMaxPasses) {
    radix[n++] = 4;
    M /= 4;
  }
  if (M % 2 == 0 && n < kMaxPasses) {
    radix[n++] = 2;
    M /= 2;
  }
  while (M % 3 == 0 && n < kMaxPasses) {
    radix[n++] = 3;
    M /= 3;
  }
  while (M % 5 == 0 && n < kMaxPasses) {
    radix[n++] = 5;
    M /= 5;
  }
  return M == 1 ? n : 0;
}

// Bin k (0 <= k <= M) of the real FFT of 2M samples from the complex FFT Z
// of z[m] = x[2m] + i x[2m+1]; wk = exp(-i pi k / M).
CC_HD Cpx real_bin(const Cpx* Z, int M, int k, Cpx wk) {
  const Cpx a = Z[k == M ? 0 : k];
  const Cpx b = cconj(Z[k == 0 ? 0 : M - k]);
  const Cpx s = cscale(cadd(a, b), 0.5f);
  const Cpx d = cscale(csub(a, b), 0.5f);
  return cadd(s, cmul_negi(cmul(wk, d)));
}

// X / max(|X|, 1e-8) with float32 sqrt and division (src/CrossCorr.cpp:104-110);
// std::max(a, b) is (a < b) ? b : a, so a NaN magnitude stays NaN
CC_HD Cpx whiten(Cpx x) {
  float a = sqrtf(x.re * x.re + x.im * x.im);
  a = a < 1e-8f ? 1e-8f : a;
  return cpx(x.re / a, x.im / a);
}

CC_HD float onebit(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

// ------------------------------------------------------- window geometry
// floor(a / b) and ceil(a / b) for b > 0
CC_HD long long floor_div(long long a, long long b) {
  return a >= 0 ? a / b : -((-a + b - 1) / b);
}
CC_HD long long ceil_div(long long a, long long b) { return -floor_div(-a, b); }

// The shifts k in [0, nshifts) with k*steplen >= start and
// k*steplen + fftlen < end (src/CrossCorr.cpp:88-95), as [*lo, *hi];
// empty when *lo > *hi. steplen > 0 unless nshifts == 1.
CC_HD void shift_range(long long nshifts, long long steplen, long long fftlen, long long start,
                       long long end, long long* lo, long long* hi) {
  if (nshifts <= 1) {
    const bool keep = nshifts == 1 && 0 >= start && fftlen < end;
    *lo = 0;
    *hi = keep ? 0 : -1;
    return;
  }
  long long a = start <= 0 ? 0 : ceil_div(start, steplen);
  long long b = floor_div(end - fftlen - 1, steplen);
  if (b > nshifts - 1) b = nshifts - 1;
  *lo = a;
  *hi = b;
}

// Windows both stations keep
CC_HD int pair_count(int lo_a, int hi_a, int lo_b, int hi_b) {
  const int lo = lo_a > lo_b ? lo_a : lo_b;
  const int hi = hi_a < hi_b ? hi_a : hi_b;
  return hi >= lo ? hi - lo + 1 : 0;
}

// --------------------------------------------------------- pair products
// Station tiles of kTile x kTile and kLanes frequencies; a CTA of
// kGramThreads threads: warp w owns tile rows 2w and 2w+1, lane j frequency
// j of the tile, and every column b.
constexpr int kTile = 16;
constexpr int kLanes = 32;
constexpr int kGramThreads = 256;
constexpr int kRowsPerWarp = kTile / (kGramThreads / 32);  // 2

// One shift: xa = the tile's a rows [kTile][kLanes], xb its b rows.
CC_HD void gram_step(const Cpx* xa, const Cpx* xb, int warp, int lane,
                     Cpx (&acc)[kRowsPerWarp][kTile]) {
#pragma unroll
  for (int ra = 0; ra < kRowsPerWarp; ++ra) {
    const Cpx a = xa[(warp * kRowsPerWarp + ra) * kLanes + lane];
#pragma unroll
    for (int b = 0; b < kTile; ++b) {
      const Cpx x = xb[b * kLanes + lane];
      // conj(a) * x
      acc[ra][b].re += a.re * x.re + a.im * x.im;
      acc[ra][b].im += a.re * x.im - a.im * x.re;
    }
  }
}

// The stored value of a pair: (initial + sum) / count, the reference's
// in-place accumulation followed by its division (src/CrossCorr.cpp:122-144).
CC_HD Cpx pair_value(Cpx init, Cpx sum, int count) {
  const float n = (float)count;
  return cpx((init.re + sum.re) / n, (init.im + sum.im) / n);
}

}  // namespace xc
}  // namespace ccfj
