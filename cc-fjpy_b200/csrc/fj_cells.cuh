// Device-side building blocks of the station-amortised F-J kernels,
// shared by the single-data-set transform (fj_transform.cu) and the ragged
// batch (fj_batch.cu).
#pragma once

#include "ccfj_core.cuh"
#include "fj_frontend.cuh"
#include "fj_interval.cuh"

namespace ccfj {

using fjs::Station;
using fjs::ZB;

// Switch point of the interval rule (in k dr): the quintic Hermite rule's
// truncation error is about dx^6/1e5 relative, the closed form's rounding
// error about eps * 2/dx^2; these balance near 0.6 in FP32 and near 0.05 in
// FP64.
constexpr float kDefaultTau32 = 0.6f;
constexpr float kDefaultTau64 = 0.05f;
constexpr int kChunk = 64;           // stations per partial sum
// Unroll factor of the itype-1 station loop.
#ifndef CCFJ_STATION_UNROLL
#define CCFJ_STATION_UNROLL 2
#endif
#define CCFJ_PRAGMA_(x) _Pragma(#x)
#define CCFJ_PRAGMA(x) CCFJ_PRAGMA_(x)

template <int MODE>
struct ModeTraits;
template <>
struct ModeTraits<CCFJ_MODE_J> {
  static constexpr int NIN = 1, NACC = 1;
  static constexpr bool WJ = true, WY = false;
};
template <>
struct ModeTraits<CCFJ_MODE_Y> {
  static constexpr int NIN = 1, NACC = 1;
  static constexpr bool WJ = false, WY = true;
};
template <>
struct ModeTraits<CCFJ_MODE_J_MINUS_Y> {
  static constexpr int NIN = 2, NACC = 1;
  static constexpr bool WJ = true, WY = true;
};
template <>
struct ModeTraits<CCFJ_MODE_ABS_J> {
  static constexpr int NIN = 2, NACC = 2;
  static constexpr bool WJ = true, WY = false;
};
template <>
struct ModeTraits<CCFJ_MODE_ABS_H> {
  static constexpr int NIN = 2, NACC = 2;
  static constexpr bool WJ = true, WY = true;
};

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

// Per-thread constants of one (f, c) cell.
template <typename T>
struct Cell;
template <>
struct Cell<float> {
  float q_hi, q_lo;  // f / c as a double-float (cycles per unit distance)
  float k;           // 2 pi f / c
  float k2;          // k^2
  float inv_k;
  float inv_k2;
  // Set by prepare_folded() for the folded interval sum:
  // s8 = 8 / k: x = k r >= 8 where r >= s8, and an interval of length D
  // takes the closed form (k |D| >= tau) where |D| (8 / tau) >= s8.
  float s8;
  // The wavenumber exactly as init() rounds it (also used for the
  // per-frequency bounds of the folded interval sum).
  static __device__ __forceinline__ float wavenumber(float fl, float cl) {
    return (float)(fjs::kTwoPi * ((double)fl / (double)cl));
  }
  __device__ void init(float fl, float cl) {
    const double q = (double)fl / (double)cl;
    q_hi = (float)q;
    q_lo = (float)(q - (double)q_hi);
    const double kd = fjs::kTwoPi * q;
    k = wavenumber(fl, cl);
    k2 = (float)(kd * kd);
    inv_k = (float)(1.0 / kd);
    inv_k2 = (float)(1.0 / (kd * kd));
  }
  template <bool WJ, bool WY, bool WZ1>
  __device__ __forceinline__ void eval(float r, float x, bool need_b, ZB<float>& J,
                                       ZB<float>& Y) const {
    const float p_hi = q_hi * r;
    const float e = fmaf(q_hi, r, -p_hi);
    const float p_lo = fmaf(q_lo, r, e);
    fjs::eval_station_f32<WJ, WY, WZ1>(x, p_hi, p_lo, need_b, J, Y);
  }
  __device__ void prepare_folded() { s8 = (float)(8.0 / (fjs::kTwoPi * ((double)q_hi + (double)q_lo))); }
  // gam = sqrt(2 / (pi k)): the Hankel amplitude is M = gam / sqrt(r). At
  // k = 0 (f = 0) no station reaches x >= 8 and the scale is taken as 1.
  __device__ __forceinline__ float gamma() const {
    return k == 0.0f ? 1.0f : sqrtf((float)(2.0 / fjs::kPi) / k);
  }
  // Station values for the folded interval sum: y0 = Z0 / M, y1 = Z1 / M
  // with M = gam / sqrtr (rinv = 1/r and sqrtr = sqrt(r) per station;
  // sqrtr = 1 where r = 0). The range test uses s8, so x = k r is formed
  // only below 8; LARGE asserts x >= 8 and drops the test. B is not formed;
  // Z1 only with WZ1.
  template <bool WJ, bool WY, bool LARGE, bool WZ1 = true>
  __device__ __forceinline__ void eval_y(float r, float rinv, float sqrtr, ZB<float>& J,
                                         ZB<float>& Y) const {
    if (LARGE || r >= s8) {  // x >= 8
      const float p_hi = q_hi * r;
      const float e = fmaf(q_hi, r, -p_hi);
      const float p_lo = fmaf(q_lo, r, e);
      fjs::eval_large_scaled_f32<WJ, WY, WZ1>(s8 * rinv, p_hi, p_lo, false, 0.0f, J, Y);
    } else {
      fjs::eval_small_f32<WJ, WY, WZ1>(k * r, false, J, Y);
      // 1 / M = sqrtr sqrt(pi k / 2) (= sqrt(pi x / 2) for r > 0; 1 / gam)
      const float sc =
          k == 0.0f ? sqrtr : sqrtr * fjs::sqrt_fast((float)(fjs::kPi / 2.0) * k);
      if (WJ) {
        J.z0 *= sc;
        if (WZ1) J.z1 *= sc;
      }
      if (WY) {
        Y.z0 *= sc;
        if (WZ1) Y.z1 *= sc;
      }
    }
  }
  // B = int_0^x Z0 at a station whose eval_y values are in J / Y (only the
  // closed form of an interval needs it).
  template <bool WJ, bool WY>
  __device__ __forceinline__ void fill_b(float r, float rinv, ZB<float>& J, ZB<float>& Y) const {
    if (r >= s8) {
      // B_J = 1 + M (y1 rho0 - y0 rho1), B_Y = M (y1 rho0 - y0 rho1) with
      // M = sqrt(s / (4 pi)), s = 8 / x
      const float s = s8 * rinv;
      const float z = s * s;
      constexpr float cr0[] = FJC_F32_L_RHO0;
      constexpr float cr1[] = FJC_F32_L_RHO1;
      const float rho0 = fjs::horner(cr0, z);
      const float rho1 = fjs::horner(cr1, z) * s;
      const float m = fjs::sqrt_fast(s * (float)(0.25 / fjs::kPi));
      if (WJ) J.b = fmaf(m, fmaf(J.z1, rho0, -J.z0 * rho1), 1.0f);
      if (WY) Y.b = m * fmaf(Y.z1, rho0, -Y.z0 * rho1);
    } else {
      ZB<float> tJ{}, tY{};
      fjs::eval_small_f32<WJ, WY, true>(k * r, true, tJ, tY);
      J.b = tJ.b;
      Y.b = tY.b;
    }
  }
};
template <>
struct Cell<double> {
  double q, k, k2, inv_k, inv_k2;
  double s8;  // as Cell<float>
  static __device__ __forceinline__ double wavenumber(float fl, float cl) {
    return fjs::kTwoPi * ((double)fl / (double)cl);
  }
  __device__ void init(float fl, float cl) {
    q = (double)fl / (double)cl;
    k = wavenumber(fl, cl);
    k2 = k * k;
    inv_k = 1.0 / k;
    inv_k2 = 1.0 / k2;
  }
  template <bool WJ, bool WY, bool WZ1>
  __device__ __forceinline__ void eval(double r, double x, bool need_b, ZB<double>& J,
                                       ZB<double>& Y) const {
    (void)need_b;
    fjs::eval_station_f64<WJ, WY, WZ1>(x, q * r, J, Y);
  }
  __device__ void prepare_folded() { s8 = 8.0 / k; }
  __device__ __forceinline__ double gamma() const {
    return k == 0.0 ? 1.0 : sqrt(2.0 / (fjs::kPi * k));
  }
  // As Cell<float>::eval_y / fill_b (values divided by M = gam / sqrtr).
  template <bool WJ, bool WY, bool LARGE, bool WZ1 = true>
  __device__ __forceinline__ void eval_y(double r, double rinv, double sqrtr, ZB<double>& J,
                                         ZB<double>& Y) const {
    (void)rinv;
    fjs::eval_station_f64<WJ, WY, false>(k * r, q * r, J, Y);
    const double sc = k == 0.0 ? sqrtr : sqrtr * sqrt(0.5 * fjs::kPi * k);
    if (WJ) {
      J.z0 *= sc;
      J.z1 *= sc;
    }
    if (WY) {
      Y.z0 *= sc;
      Y.z1 *= sc;
    }
  }
  template <bool WJ, bool WY>
  __device__ __forceinline__ void fill_b(double r, double rinv, ZB<double>& J,
                                         ZB<double>& Y) const {
    (void)rinv;
    ZB<double> tJ{}, tY{};
    fjs::eval_station_f64<WJ, WY, true>(k * r, q * r, tJ, tY);
    J.b = tJ.b;
    Y.b = tY.b;
  }
};

struct FjDev {
  const float* rs;
  const float* drs;  // [nr + 1]: r_i - r_{i-1}, 0 at i = 0 and at i = nr
  // [nr]: (r_i, r_{i+1} - r_i (0 for the last pair), 1/r_i, sqrt(r_i)), with
  // 1/r = 0 and sqrt(r) = 1 where r = 0
  const float4* geo;
  // itype 1: StationCoef<T> [nr][nf] per input; itype 0: g * w [nr][nf]
  const void* gb[2];
  const void* kb;    // itype 1: fold threshold per frequency (T), see fold_threshold
  const float* f;
  const float* c;
  float* out;
  int nr, nf, nc;
  float tau;
  // Station range [i_lo, i_hi) of this launch (the whole set: 0, nr). With
  // `part` set, the raw sums of the range (before the amplitude gamma and
  // the magnitude) go to part[q][nc][nf] (q < the mode's accumulators)
  // instead of out, for a later fixed-order reduction over the ranges.
  int i_lo, i_hi;
  float* part;
  int split_len;  // stations per range when a launch splits the set (grid z)
};

// ------------------------------------------------- folded interval sum
// For an interval (A, B) of length D that takes the quintic Hermite rule,
// the term g_A I0 + (b/k) I1 of the per-interval integral (see
// fj_interval.cuh) is linear in the station values h, h', h'' with
// coefficients k^n times quantities that do not depend on the velocity:
//
//   k (a1 h_A + b1 h_B) + k^2 (a2 h_A' + b2 h_B') + k^3 (a3 h_A'' + b3 h_B'')
//   a1 = g_A D/2 + b D^2/10      b1 = g_A D/2 + 2 b D^2/5
//   a2 = g_A D^2/10 + b D^3/60   b2 = -g_A D^2/10 - b D^3/12
//   a3 = g_A D^3/120             b3 = (g_A D^3 + b D^4)/120
//
// Summed over the intervals, each station collects P_n = (a_n of the
// interval to its right) + (b_n of the interval to its left), and with
// x = k r, h = x Z0, h' = Z0 - x Z1, h'' = -Z1 - x Z0 the whole sum is
//
//   (1/k^2) sum = sum_s Z0(x_s) (A_s - k^2 C_s) - k Z1(x_s) B_s
//   A = P1 r + P2,   B = P2 r + P3,   C = P3 r.
//
// A, B, C are formed once per (station, frequency) in FP64 (the
// cancellation between neighbouring intervals happens there, exactly), so
// the kernel's per-(station, velocity) work is the special functions plus
// three FMAs. An interval is folded in when, at its frequency, it takes the
// Hermite rule at the smallest k (under the Y-basis rule, the stricter one)
// and k D stays below kFoldMax at the largest |k|; a folded interval that
// takes the closed form for some velocity has its Hermite part subtracted
// there again, and intervals not folded in are integrated explicitly.
// kFoldMax bounds that subtraction: the Hermite terms grow like (k D)^4/120
// relative to the interval's integral.
constexpr float kFoldMax = 4.0f;

// Per frequency: the interval length below which an interval is folded in,
// min(tau / min k, kFoldMax / max |k|) over the velocities. Below tau / k
// an interval takes the Hermite rule for wavenumber k.
template <typename T>
__device__ __forceinline__ T fold_threshold(T kmin, T kabs, T tau) {
  return fmin(tau / kmin, T(kFoldMax) / kabs);
}

// Whether interval (rA, rA + D) is folded in at a frequency with fold
// threshold thr: short enough, and not reaching closer to the origin than
// its own length (where the Y basis needs the closed form). The
// preparation and the kernels evaluate exactly this, so they agree.
template <typename T>
__device__ __forceinline__ bool folded_interval(T thr, T D, T rA) {
  return fabs(D) < thr && !(D > rA);
}

// Per (station, frequency): the folded-sum coefficients divided by the
// station's sqrt(r) (the r part of the Hankel amplitude; sqrt(r) := 1 where
// r = 0), and the station's spectrum value g (from which an explicit
// interval rebuilds its b).
template <typename T>
struct alignas(16) StationCoef {
  T A, B, C, g;
};
static_assert(sizeof(StationCoef<float>) == 16, "one 16-byte load per station");

__device__ __forceinline__ StationCoef<float> load_coef(const StationCoef<float>* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ StationCoef<double> load_coef(const StationCoef<double>* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 v0 = __ldg(q), v1 = __ldg(q + 1);
  return {v0.x, v0.y, v1.x, v1.y};
}

// b of the interval from g1 to g2: (g2 - g1) / max(D, 0.1) as
// src/FJcpu.cpp:259-261, in the kernel's precision.
template <typename T>
__device__ __forceinline__ T interval_slope(T g1, T g2, float D) {
  return (g2 - g1) / (T)fmaxf(D, 0.1f);
}

// Coefficients of station s with value g at r (sqrtr = geo.w), left
// neighbour (gl, rl) at distance Dl (if has_l) and right neighbour gr at
// distance Dr (if has_r); thr = the frequency's fold threshold.
template <typename T>
__device__ __forceinline__ StationCoef<T> station_coef(T g, T gl, T gr, bool has_l, bool has_r,
                                                       float r, float rl, float Dl, float Dr,
                                                       float sqrtr, T thr) {
  double P1 = 0.0, P2 = 0.0, P3 = 0.0;
  if (has_l && folded_interval<T>(thr, (T)Dl, (T)rl)) {  // s is B of (s-1, s)
    const double ga = gl, b = interval_slope<T>(gl, g, Dl), D = Dl;
    const double D2 = D * D, D3 = D2 * D;
    P1 += 0.5 * ga * D + 0.4 * b * D2;
    P2 -= 0.1 * ga * D2 + b * D3 / 12.0;
    P3 += (ga * D3 + b * D3 * D) / 120.0;
  }
  if (has_r && folded_interval<T>(thr, (T)Dr, (T)r)) {  // s is A of (s, s+1)
    const double ga = g, b = interval_slope<T>(g, gr, Dr), D = Dr;
    const double D2 = D * D, D3 = D2 * D;
    P1 += 0.5 * ga * D + 0.1 * b * D2;
    P2 += 0.1 * ga * D2 + b * D3 / 60.0;
    P3 += ga * D3 / 120.0;
  }
  const double rd = r, w = 1.0 / (double)sqrtr;
  return {(T)((P1 * rd + P2) * w), (T)((P2 * rd + P3) * w), (T)(P3 * rd * w), g};
}

// Fold threshold per frequency (one warp per frequency).
template <typename T>
__global__ void fj_kbounds_kernel(const float* __restrict__ f, const float* __restrict__ c,
                                  int nf, int nc, T tau, T* __restrict__ thr) {
  const int fi = blockIdx.x * blockDim.y + threadIdx.y;
  if (fi >= nf) return;
  const float fl = f[fi];
  T lo = T(INFINITY), hi = T(0);
  for (int j = threadIdx.x; j < nc; j += 32) {
    const T k = Cell<T>::wavenumber(fl, c[j]);
    lo = fmin(lo, k);
    hi = fmax(hi, fabs(k));
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if (threadIdx.x == 0) thr[fi] = fold_threshold<T>(lo, hi, tau);
}

// Station geometry for the itype-1 kernels (see FjDev::geo).
__device__ __forceinline__ float4 station_geometry(float r, float d_next) {
  const bool pos = r > 0.0f;
  return make_float4(r, d_next, pos ? 1.0f / r : 0.0f, pos ? sqrtf(r) : 1.0f);
}

// ------------------------------------------------------------ preparation
// itype 0: gathers row perm[i] (or i) of one input, takes every u_cs-th
// element, and writes g_i w_i / sqrt(r_i) per (pair, frequency): the
// trapezoid weight w (src/FJcpu.cpp:348-357) over the r part of the Hankel
// amplitude (sqrt(r) := 1 at r = 0).
template <typename T>
__global__ void fj_prep_u_kernel(InDesc in, int nr, int nf, const float* __restrict__ wtr,
                                 const float4* __restrict__ geo, T* __restrict__ dst) {
  // pairs on grid x (no 65535 limit), frequencies on grid y
  const int fi = blockIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  if (fi >= nf || i >= nr) return;
  const long long row = in.perm ? in.perm[i] : i;
  const T g = (T)in.p[row * in.ld + (long long)fi * in.cs];
  dst[(long long)i * nf + fi] = g * (T)wtr[i] / (T)geo[i].w;
}

// itype 1: gathers rows perm[i-1], perm[i], perm[i+1] (or i-1, i, i+1) of
// one input and writes station i's folded-sum coefficients.
template <typename T>
__global__ void fj_prep_coef_kernel(InDesc in, int nr, int nf, const float* __restrict__ rs,
                                    const float* __restrict__ drs,
                                    const float4* __restrict__ geo, const T* __restrict__ thr,
                                    StationCoef<T>* __restrict__ dst) {
  const int fi = blockIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  if (fi >= nf || i >= nr) return;
  const long long* perm = in.perm;
  const long long col = (long long)fi * in.cs;
  const bool hl = i > 0, hr = i + 1 < nr;
  const T g = (T)in.p[(perm ? perm[i] : i) * in.ld + col];
  const T gl = hl ? (T)in.p[(perm ? perm[i - 1] : i - 1) * in.ld + col] : T(0);
  const T gr = hr ? (T)in.p[(perm ? perm[i + 1] : i + 1) * in.ld + col] : T(0);
  dst[(long long)i * nf + fi] = station_coef<T>(g, gl, gr, hl, hr, rs[i], hl ? rs[i - 1] : 0.0f,
                                                drs[i], drs[i + 1], geo[i].w, thr[fi]);
}

// ------------------------------------------------- station-amortised kernel
// acc += g_{i-1} I0 + b_i I1 / k per input and basis (I1k = I1 / k); the
// sum is formed with one FMA per term.
template <int MODE, typename T>
__device__ __forceinline__ void accumulate_interval(T (&acc)[2], const typename Vec2<T>::type& g0,
                                                    const typename Vec2<T>::type& g1, T I0J,
                                                    T I1Jk, T I0Y, T I1Yk) {
  using fjs::fmaT;
  if (MODE == CCFJ_MODE_J) {
    acc[0] = fmaT(g0.y, I1Jk, fmaT(g0.x, I0J, acc[0]));
  } else if (MODE == CCFJ_MODE_Y) {
    acc[0] = fmaT(g0.y, I1Yk, fmaT(g0.x, I0Y, acc[0]));
  } else if (MODE == CCFJ_MODE_J_MINUS_Y) {
    acc[0] = fmaT(g0.y, I1Jk, fmaT(g0.x, I0J, acc[0]));
    acc[0] = fmaT(-g1.y, I1Yk, fmaT(-g1.x, I0Y, acc[0]));
  } else if (MODE == CCFJ_MODE_ABS_J) {
    acc[0] = fmaT(g0.y, I1Jk, fmaT(g0.x, I0J, acc[0]));
    acc[1] = fmaT(g1.y, I1Jk, fmaT(g1.x, I0J, acc[1]));
  } else {  // ABS_H: (J(u0) - Y(u1)) + i (J(u1) + Y(u0))
    acc[0] = fmaT(g0.y, I1Jk, fmaT(g0.x, I0J, acc[0]));
    acc[0] = fmaT(-g1.y, I1Yk, fmaT(-g1.x, I0Y, acc[0]));
    acc[1] = fmaT(g1.y, I1Jk, fmaT(g1.x, I0J, acc[1]));
    acc[1] = fmaT(g0.y, I1Yk, fmaT(g0.x, I0Y, acc[1]));
  }
}

template <int MODE, typename T>
__device__ __forceinline__ void accumulate_station(T (&acc)[2], T g0, T g1, T zJ, T zY) {
  if (MODE == CCFJ_MODE_J) {
    acc[0] = fjs::fmaT(g0, zJ, acc[0]);
  } else if (MODE == CCFJ_MODE_Y) {
    acc[0] = fjs::fmaT(g0, zY, acc[0]);
  } else {
    using fjs::fmaT;
    if (MODE == CCFJ_MODE_J_MINUS_Y) {
      acc[0] = fmaT(-g1, zY, fmaT(g0, zJ, acc[0]));
    } else if (MODE == CCFJ_MODE_ABS_J) {
      acc[0] = fmaT(g0, zJ, acc[0]);
      acc[1] = fmaT(g1, zJ, acc[1]);
    } else {  // ABS_H: (J(u0) - Y(u1)) + i (J(u1) + Y(u0))
      acc[0] = fmaT(-g1, zY, fmaT(g0, zJ, acc[0]));
      acc[1] = fmaT(g0, zY, fmaT(g1, zJ, acc[1]));
    }
  }
}

template <int MODE, typename T>
__device__ __forceinline__ float finish(const T (&tot)[2], T scale) {
  if (ModeTraits<MODE>::NACC == 1) return (float)(tot[0] * scale);
  const float re = (float)(tot[0] * scale);
  const float im = (float)(tot[1] * scale);
  return sqrtf(re * re + im * im);  // np.sqrt(outr**2 + outi**2) in float32
}

// Whether an interval of length dx starting at x1 takes the closed form
// (then B is needed at both of its stations): long intervals, and for the
// Y basis (Y0 is singular at x = 0) also intervals that reach close to the
// origin, where the Hermite rule's derivatives are not bounded.
template <typename T, bool IS_Y>
__device__ __forceinline__ bool closed_form(T dx, T x1, T tau) {
  return fabs(dx) >= tau || (IS_Y && dx > x1);
}

// I0, I1 of one interval between stations (xA, zA) and (xB, zB): the
// closed form or the Hermite rule, minus the Hermite part already in the
// folded sum when the interval was folded in.
template <typename T>
__device__ __forceinline__ void explicit_moments(T xA, const ZB<T>& zA, T xB, const ZB<T>& zB,
                                                 T dx, bool closed, bool folded, T& I0, T& I1) {
  const Station<T> sA = fjs::make_station(xA, zA);
  const Station<T> sB = fjs::make_station(xB, zB);
  fjs::interval_moments<T>(sA, sB, dx, closed, I0, I1);
  if (closed && folded) {
    T h0, h1;
    fjs::interval_moments<T>(sA, sB, dx, false, h0, h1);
    I0 -= h0;
    I1 -= h1;
  }
}

// Interval (A, B) of one cell for the bases that need explicit work
// (exJ / exY; lcJ / lcY its closed-form flags), in the units of the folded
// sums (output / gam). yA*, yB* are the stations' values from eval_scaled
// (Z / M, and B), at rA, rB with sqrt(r) = sqA, sqB; gA*, gB* the stations'
// spectrum values of inputs 0 and 1. Rarely taken: arguments and result by
// value.
template <typename T>
struct Acc2 {
  T v[2];
};
template <typename T>
__device__ __forceinline__ ZB<T> unscale(const ZB<T>& y, T m) {
  return ZB<T>{y.z0 * m, y.z1 * m, y.b};
}
template <int MODE, typename T>
__device__ __forceinline__ Acc2<T> explicit_interval(const Cell<T>& cell, bool exJ, bool exY,
                                                     bool lcJ, bool lcY, bool folded, T D, T rA,
                                                     T sqA, T rB, T sqB, ZB<T> yAJ, ZB<T> yBJ,
                                                     ZB<T> yAY, ZB<T> yBY, T gA0, T gB0, T gA1,
                                                     T gB1) {
  using T2 = typename Vec2<T>::type;
  const T k = cell.k;
  const T gam = cell.gamma();
  const T mA = gam / sqA, mB = gam / sqB;
  const T xA = k * rA, xB = k * rB, dx = k * D;
  T2 g0, g1;
  g0.x = gA0;
  g0.y = interval_slope<T>(gA0, gB0, (float)D);
  g1.x = gA1;
  g1.y = ModeTraits<MODE>::NIN > 1 ? interval_slope<T>(gA1, gB1, (float)D) : T(0);
  T I0J = 0, I1J = 0, I0Y = 0, I1Y = 0;
  if (ModeTraits<MODE>::WJ && exJ)
    explicit_moments<T>(xA, unscale(yAJ, mA), xB, unscale(yBJ, mB), dx, lcJ, folded, I0J, I1J);
  if (ModeTraits<MODE>::WY && exY)
    explicit_moments<T>(xA, unscale(yAY, mA), xB, unscale(yBY, mB), dx, lcY, folded, I0Y, I1Y);
  const T inv_k = T(1) / k;
  const T s0 = inv_k * inv_k / gam, s1 = s0 * inv_k;
  T acc[2] = {T(0), T(0)};
  accumulate_interval<MODE, T>(acc, g0, g1, I0J * s0, I1J * s1, I0Y * s0, I1Y * s1);
  return Acc2<T>{{acc[0], acc[1]}};
}

// Minimum resident 256-thread CTAs per SM of the kernels built on
// fj_cells. FP32: three CTAs, at most 85 registers. Two velocities per
// thread (the paired x >= 8 step) then fit without spilling; under four
// CTAs (64 registers) they spilled, and the large-array transform measured
// 5% slower, the small one 6%. The single-set and the batch kernels share
// the bound, so they compile the cell loop alike and agree bit for bit.
// FP64 cells hold twice the registers: a cap would only make them spill.
#ifndef CCFJ_FJ_MIN_BLOCKS
#define CCFJ_FJ_MIN_BLOCKS 3
#endif
template <typename T>
constexpr int fj_min_blocks() { return sizeof(T) == 4 ? CCFJ_FJ_MIN_BLOCKS : 1; }

template <bool B>
struct BoolTag {
  static constexpr bool value = B;
};

// Threads per CTA of the kernels built on fj_cells: 32 frequencies x 8
// velocity rows.
constexpr int kCellThreads = 256;

// Shared-memory stage of the FP32 itype-1 loop: per buffer, the station
// coefficients of a chunk for the CTA's 32 frequencies, and its geometry.
// 33 KB (one input, 32 stations) or 32.5 KB (two inputs, 16 stations).
template <int NIN>
struct StageBuf {
  static constexpr int kStations = NIN > 1 ? 16 : 32;
  float4 coef[2][NIN][kStations][32];
  float4 geo[2][kStations];
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
// Itype-0 stage: one prepared scalar per (station, frequency) per input.
// 2 x 64 stations: 16 KB (one input) or 32 KB (two), plus the geometry.
template <int NIN>
struct StageBuf0 {
  static constexpr int kStations = 64;
  float q[2][NIN][kStations][32];
  float4 geo[2][kStations];
};

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The x >= 8 station step of the J-basis modes for CPT cells, two cells per
// paired FP32 instruction (fjs::eval_large_scaled_pair_j): the station
// values y0, y1 of every cell (into Jzs) and the folded-sum accumulation of
// each input -- acc0 += (A - k^2 C) y0, acc1 += B y1 -- exactly as the
// scalar loop computes them. The primary template (FP64 cells, odd CPT) is
// never called.
template <bool PAIRED>
struct PairedStationJ {
  template <int NIN, int CPT, typename CellT, typename Q, typename AccT, typename ZT>
  __device__ __forceinline__ static void run(const CellT*, float, float, const Q&, const Q&, AccT&,
                                             AccT&, ZT&) {}
};
#if defined(FJS_HAVE_PAIRED)
template <>
struct PairedStationJ<true> {
  template <int NIN, int CPT>
  __device__ __forceinline__ static void run(const Cell<float>* cell, float r, float rinv,
                                             const StationCoef<float>& q0,
                                             const StationCoef<float>& q1, float (&acc0)[CPT][2],
                                             float (&acc1)[CPT][2], ZB<float> (&Jzs)[CPT]) {
#pragma unroll
    for (int j = 0; j < CPT; j += 2) {
      const fjs::PairPhase ph{make_float2(cell[j].q_hi, cell[j + 1].q_hi),
                              make_float2(-cell[j].q_hi, -cell[j + 1].q_hi),
                              make_float2(cell[j].q_lo, cell[j + 1].q_lo),
                              make_float2(cell[j].s8, cell[j + 1].s8)};
      fjs::ZB2 J2;
      fjs::eval_large_scaled_pair_j(ph, r, rinv, J2);
      Jzs[j] = ZB<float>{J2.z0.x, J2.z1.x, 0.0f};
      Jzs[j + 1] = ZB<float>{J2.z0.y, J2.z1.y, 0.0f};
      const float2 nk2 = make_float2(-cell[j].k2, -cell[j + 1].k2);
#pragma unroll
      for (int q = 0; q < NIN; ++q) {  // ABS_J: the second input shares the station values
        const StationCoef<float>& sc = q == 0 ? q0 : q1;
        const float2 u = fjs::pfma(nk2, fjs::psplat(sc.C), fjs::psplat(sc.A));
        const float2 a0 = fjs::pfma(u, J2.z0, make_float2(acc0[j][q], acc0[j + 1][q]));
        const float2 a1 =
            fjs::pfma(fjs::psplat(sc.B), J2.z1, make_float2(acc1[j][q], acc1[j + 1][q]));
        acc0[j][q] = a0.x;
        acc0[j + 1][q] = a0.y;
        acc1[j][q] = a1.x;
        acc1[j + 1][q] = a1.y;
      }
    }
  }
};
#endif

// CPT cells (f, c), (f, c + 1), ... per thread share the per-station loads.
// The transform of the CPT cells (fi, c0), (fi, c0 + 1), ... of one data
// set; shared by the grid kernel below and the persistent batch kernel.
template <int MODE, int ITYPE, typename T, int CPT>
__device__ __forceinline__ void fj_cells(const FjDev& a, int fi, int c0) {
  using MT = ModeTraits<MODE>;
  constexpr bool WJ = MT::WJ, WY = MT::WY;
  // c0 is uniform across a warp (its lanes are 32 frequencies); lanes past
  // the last frequency compute the last one and store nothing, so that all
  // 32 lanes stay active for the warp-wide steps below. The staged FP32
  // itype-1 loop has CTA-wide barriers: a warp past the last velocity stays
  // and helps with the staging.
  constexpr bool kStaged = sizeof(T) == 4;
  const bool c_valid = c0 < a.nc;
  if (!kStaged && !c_valid) return;
  c0 = c_valid ? c0 : 0;
  const bool f_valid = fi < a.nf;
  const int fbase = fi - (int)(threadIdx.x & 31);  // first frequency of the warp (and CTA)
  fi = f_valid ? fi : a.nf - 1;
  Cell<T> cell[CPT];
  const float fl = a.f[fi];
#pragma unroll
  for (int j = 0; j < CPT; ++j) cell[j].init(fl, a.c[min(c0 + j, a.nc - 1)]);
  T tot[CPT][2];
#pragma unroll
  for (int j = 0; j < CPT; ++j) tot[j][0] = tot[j][1] = T(0);
  if constexpr (ITYPE == 1) {
    const T thr_fold = static_cast<const T*>(a.kb)[fi];
    const StationCoef<T>* q0p = static_cast<const StationCoef<T>*>(a.gb[0]) + fi;
    const StationCoef<T>* q1p = static_cast<const StationCoef<T>*>(a.gb[MT::NIN > 1 ? 1 : 0]) + fi;
    const T d8 = T(8) / (T)a.tau;  // closed form where |D| d8 >= s8 (k |D| >= tau)
    T s8w = T(0);                  // largest s8 = 8 / k of the warp
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      cell[j].prepare_folded();
      s8w = fmax(s8w, cell[j].s8);
    }
    for (int o = 16; o > 0; o >>= 1) s8w = fmax(s8w, __shfl_xor_sync(0xffffffffu, s8w, o));
    // Paired FP32 arithmetic (two cells per FFMA2 / FMUL2 / FADD2) for the
    // J-basis modes with an even number of cells per thread; the Y basis
    // and the explicit path stay scalar.
#ifndef CCFJ_PAIRED
#define CCFJ_PAIRED 1
#endif
    constexpr bool kPaired = CCFJ_PAIRED && sizeof(T) == 4 && CPT % 2 == 0 && WJ && !WY &&
                             (MODE == CCFJ_MODE_J || MODE == CCFJ_MODE_ABS_J);
    // The explicit path needs station i-1's values: single-basis modes carry
    // them (2 registers per cell); two-basis modes, short of registers,
    // evaluate station i-1 again when an explicit interval comes.
    constexpr bool kCarry = !(WJ && WY);
    ZB<T> zpJ[kCarry ? CPT : 1], zpY[kCarry ? CPT : 1];
    // State of interval (i-1, i): length D, folded in, reaches near the
    // origin. Station 0 has no such interval.
    T D = T(0);
    bool fold_cur = true, near_cur = false;
    T acc0[CPT][2], acc1[CPT][2];
    // One station: out += gam (y0 (A - k^2 C) - k y1 B), plus the explicit
    // interval (i-1, i) where it is not (only) in the folded sum.
    auto station = [&](auto large_tag, int i, const float4 gm, const StationCoef<T> q0,
                       const StationCoef<T> q1) {
      constexpr bool LARGE = decltype(large_tag)::value;
      const T r = gm.x, D_next = gm.y;
      const long long qi = (long long)i * a.nf;
      const T dl8 = fabs(D) * d8;
      ZB<T> Jzs[CPT], Yzs[CPT];
#if defined(FJS_HAVE_PAIRED)
      if constexpr (kPaired && LARGE) {
        // two cells per paired instruction (x >= 8 in every cell of the warp)
        PairedStationJ<kPaired>::template run<MT::NIN, CPT>(cell, (float)r, (float)gm.z, q0, q1,
                                                             acc0, acc1, Jzs);
      } else
#endif
      {
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
          ZB<T> Jz{}, Yz{};
          cell[j].template eval_y<WJ, WY, LARGE>(r, (T)gm.z, (T)gm.w, Jz, Yz);
          const T u0 = fjs::fmaT(-cell[j].k2, q0.C, q0.A);
          const T u1 = MT::NIN > 1 ? fjs::fmaT(-cell[j].k2, q1.C, q1.A) : T(0);
          accumulate_station<MODE, T>(acc0[j], u0, u1, WJ ? Jz.z0 : T(0), WY ? Yz.z0 : T(0));
          accumulate_station<MODE, T>(acc1[j], q0.B, q1.B, WJ ? Jz.z1 : T(0), WY ? Yz.z1 : T(0));
          Jzs[j] = Jz;
          Yzs[j] = Yz;
        }
      }
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        ZB<T> Jz = Jzs[j], Yz = Yzs[j];
        const bool clJ = dl8 >= cell[j].s8;
        const bool clY = clJ || near_cur;  // Y0 is singular at 0
        const bool exJ = WJ && (clJ || !fold_cur), exY = WY && (clY || !fold_cur);
        if (i > 0 && (exJ || exY)) {
          const float4 gp = __ldg(a.geo + i - 1);
          ZB<T> pJ{}, pY{};
          if constexpr (kCarry) {
            pJ = zpJ[j];
            pY = zpY[j];
          } else {
            cell[j].template eval_y<WJ, WY, false>((T)gp.x, (T)gp.z, (T)gp.w, pJ, pY);
          }
          // B at both ends where the interval takes the closed form
          if ((WJ && exJ && clJ) || (WY && exY && clY)) {
            cell[j].template fill_b<WJ, WY>((T)gp.x, (T)gp.z, pJ, pY);
            cell[j].template fill_b<WJ, WY>(r, (T)gm.z, Jz, Yz);
          }
          const T gA0 = __ldg(&q0p[qi - a.nf].g);
          const T gA1 = MT::NIN > 1 ? __ldg(&q1p[qi - a.nf].g) : T(0);
          const Acc2<T> e = explicit_interval<MODE, T>(cell[j], exJ, exY, clJ, clY, fold_cur, D,
                                                       (T)gp.x, (T)gp.w, r, (T)gm.w, pJ, Jz, pY,
                                                       Yz, gA0, q0.g, gA1, q1.g);
          acc0[j][0] += e.v[0];
          acc0[j][1] += e.v[1];
        }
        if constexpr (kCarry) {
          if (WJ) zpJ[j] = Jz;
          if (WY) zpY[j] = Yz;
        }
      }
      fold_cur = folded_interval<T>(thr_fold, D_next, r);
      near_cur = D_next > r;
      D = D_next;
    };
    if (a.i_lo > 0) {
      // A station range that starts inside the set: the state of the
      // interval (i_lo - 1, i_lo) and, for the explicit path, the values of
      // station i_lo - 1, as the station before would have left them.
      const float4 gp = __ldg(a.geo + a.i_lo - 1);
      D = (T)gp.y;
      fold_cur = folded_interval<T>(thr_fold, D, (T)gp.x);
      near_cur = D > (T)gp.x;
      if constexpr (kCarry) {
#pragma unroll
        for (int j = 0; j < CPT; ++j)
          cell[j].template eval_y<WJ, WY, false>((T)gp.x, (T)gp.z, (T)gp.w, zpJ[j], zpY[j]);
      }
    }
    const int lane = threadIdx.x & 31;
    // Closes a chunk of stations: folds its partial sums into the totals.
    auto flush = [&]() {
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        tot[j][0] += fjs::fmaT(-cell[j].k, acc1[j][0], acc0[j][0]);
        tot[j][1] += fjs::fmaT(-cell[j].k, acc1[j][1], acc0[j][1]);
        acc0[j][0] = acc0[j][1] = acc1[j][0] = acc1[j][1] = T(0);
      }
    };
#pragma unroll
    for (int j = 0; j < CPT; ++j) acc0[j][0] = acc0[j][1] = acc1[j][0] = acc1[j][1] = T(0);
    if constexpr (kStaged) {
      // The CTA's 8 warps share the 32 frequencies of fbase..fbase+31, so
      // one copy of a chunk's station data in shared memory serves them all:
      // chunks of S stations (coefficients and geometry) are staged with
      // cp.async, double-buffered, while the previous chunk is computed.
      using SB = StageBuf<MT::NIN>;
      constexpr int S = SB::kStations;
      __shared__ SB sb;
      const int tid = threadIdx.y * 32 + threadIdx.x;
      const StationCoef<float>* g0 = static_cast<const StationCoef<float>*>(a.gb[0]);
      const StationCoef<float>* g1 = static_cast<const StationCoef<float>*>(a.gb[MT::NIN > 1 ? 1 : 0]);
      // chunks of S stations from i_lo (a multiple of S) to i_hi
      auto stage = [&](int ch, int buf) {
        const int i0 = a.i_lo + ch * S;
        const int n = min(S, a.i_hi - i0);
        for (int t = tid; t < n * 32; t += kCellThreads) {
          const int st = t >> 5;
          const long long src = (long long)(i0 + st) * a.nf + min(fbase + (t & 31), a.nf - 1);
          cp_async16(&sb.coef[buf][0][st][t & 31], g0 + src);
          if (MT::NIN > 1) cp_async16(&sb.coef[buf][MT::NIN > 1 ? 1 : 0][st][t & 31], g1 + src);
        }
        for (int t = tid; t < n; t += kCellThreads) cp_async16(&sb.geo[buf][t], a.geo + i0 + t);
        cp_async_commit();
      };
      const int nch = (a.i_hi - a.i_lo + S - 1) / S;
      stage(0, 0);
      for (int ch = 0; ch < nch; ++ch) {
        const int buf = ch & 1;
        if (ch + 1 < nch)
          stage(ch + 1, buf ^ 1);
        else
          cp_async_commit();  // one group per iteration keeps the count below
        cp_async_wait<1>();   // this thread's copies of chunk ch have landed
        __syncthreads();      // ... and everybody else's
        const int i0 = a.i_lo + ch * S;
        const int n = min(S, a.i_hi - i0);
        if (c_valid) {
          // smallest r of the chunk (the input need not be sorted): at or
          // above s8w every station of the chunk has x >= 8 in every cell of
          // the warp
          float rmin = lane < n ? sb.geo[buf][lane].x : INFINITY;
          for (int o = 16; o > 0; o >>= 1)
            rmin = fminf(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
          auto run = [&](auto large_tag) {
            CCFJ_PRAGMA(unroll CCFJ_STATION_UNROLL)
            for (int st = 0; st < n; ++st) {
              const float4 c0v = sb.coef[buf][0][st][lane];
              float4 c1v = c0v;
              if (MT::NIN > 1) c1v = sb.coef[buf][MT::NIN > 1 ? 1 : 0][st][lane];
              station(large_tag, i0 + st, sb.geo[buf][st], StationCoef<T>{c0v.x, c0v.y, c0v.z, c0v.w},
                      StationCoef<T>{c1v.x, c1v.y, c1v.z, c1v.w});
            }
          };
          if ((T)rmin >= s8w)
            run(BoolTag<true>{});
          else
            run(BoolTag<false>{});
          flush();
        }
        __syncthreads();  // buffer buf is refilled by the stage() of the next iteration
      }
    } else {
      for (int i0 = a.i_lo; i0 < a.i_hi; i0 += kChunk) {
        const int i1 = min(a.i_hi, i0 + kChunk);
        float rmin = INFINITY;
        for (int t = i0 + lane; t < i1; t += 32) rmin = fminf(rmin, __ldg(a.rs + t));
        for (int o = 16; o > 0; o >>= 1) rmin = fminf(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
        auto run = [&](auto large_tag) {
          for (int i = i0; i < i1; ++i) {
            const long long qi = (long long)i * a.nf;
            const StationCoef<T> q0 = load_coef(q0p + qi);
            StationCoef<T> q1{};
            if (MT::NIN > 1) q1 = load_coef(q1p + qi);
            station(large_tag, i, __ldg(a.geo + i), q0, q1);
          }
        };
        if ((T)rmin >= s8w)
          run(BoolTag<true>{});
        else
          run(BoolTag<false>{});
        flush();
      }
    }
    if (!c_valid) return;
    if (a.part) {  // raw sums of this station range
#pragma unroll
      for (int j = 0; j < CPT; ++j)
        if (f_valid && c0 + j < a.nc)
#pragma unroll
          for (int q = 0; q < MT::NACC; ++q)
            a.part[((long long)q * a.nc + c0 + j) * a.nf + fi] = (float)tot[j][q];
      return;
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const T gam = cell[j].gamma();
      T res[2];
      res[0] = gam * tot[j][0];
      res[1] = gam * tot[j][1];
      // k = 0 (f = 0) divides by zero in the reference: NaN
      const float v = cell[j].k == T(0) ? __int_as_float(0x7fffffff) : finish<MODE, T>(res, T(1));
      if (f_valid && c0 + j < a.nc) a.out[(long long)(c0 + j) * a.nf + fi] = v;
    }
  } else {
    // Trapezoid: out = gam sum_s y0(x_s) q_s with y0 = Z0 / M and the
    // prepared q = g w / sqrt(r) (w the trapezoid weight).
    T s8w = T(0);
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      cell[j].prepare_folded();
      s8w = fmax(s8w, cell[j].s8);
    }
    for (int o = 16; o > 0; o >>= 1) s8w = fmax(s8w, __shfl_xor_sync(0xffffffffu, s8w, o));
    const int lane = threadIdx.x & 31;
    T acc[CPT][2];
#pragma unroll
    for (int j = 0; j < CPT; ++j) acc[j][0] = acc[j][1] = T(0);
    auto station = [&](auto large_tag, const float4 gm, T q0, T q1) {
      constexpr bool LARGE = decltype(large_tag)::value;
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        ZB<T> Jz{}, Yz{};
        cell[j].template eval_y<WJ, WY, LARGE, false>((T)gm.x, (T)gm.z, (T)gm.w, Jz, Yz);
        accumulate_station<MODE, T>(acc[j], q0, q1, WJ ? Jz.z0 : T(0), WY ? Yz.z0 : T(0));
      }
    };
    auto flush = [&]() {
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        tot[j][0] += acc[j][0];
        tot[j][1] += acc[j][1];
        acc[j][0] = acc[j][1] = T(0);
      }
    };
    if constexpr (kStaged) {
      // staged as the itype-1 loop (one scalar per station and frequency)
      using SB = StageBuf0<MT::NIN>;
      constexpr int S = SB::kStations;
      __shared__ SB sb;
      const int tid = threadIdx.y * 32 + threadIdx.x;
      const float* g0 = static_cast<const float*>(a.gb[0]);
      const float* g1 = static_cast<const float*>(a.gb[MT::NIN > 1 ? 1 : 0]);
      auto stage = [&](int ch, int buf) {
        const int i0 = a.i_lo + ch * S;
        const int n = min(S, a.i_hi - i0);
        for (int t = tid; t < n * 32; t += kCellThreads) {
          const int st = t >> 5;
          const long long src = (long long)(i0 + st) * a.nf + min(fbase + (t & 31), a.nf - 1);
          cp_async4(&sb.q[buf][0][st][t & 31], g0 + src);
          if (MT::NIN > 1) cp_async4(&sb.q[buf][MT::NIN > 1 ? 1 : 0][st][t & 31], g1 + src);
        }
        for (int t = tid; t < n; t += kCellThreads) cp_async16(&sb.geo[buf][t], a.geo + i0 + t);
        cp_async_commit();
      };
      const int nch = (a.i_hi - a.i_lo + S - 1) / S;
      stage(0, 0);
      for (int ch = 0; ch < nch; ++ch) {
        const int buf = ch & 1;
        if (ch + 1 < nch)
          stage(ch + 1, buf ^ 1);
        else
          cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int n = min(S, a.i_hi - a.i_lo - ch * S);
        if (c_valid) {
          float rmin = INFINITY;
          for (int t = lane; t < n; t += 32) rmin = fminf(rmin, sb.geo[buf][t].x);
          for (int o = 16; o > 0; o >>= 1)
            rmin = fminf(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
          auto run = [&](auto large_tag) {
            CCFJ_PRAGMA(unroll CCFJ_STATION_UNROLL)
            for (int st = 0; st < n; ++st)
              station(large_tag, sb.geo[buf][st], sb.q[buf][0][st][lane],
                      MT::NIN > 1 ? sb.q[buf][MT::NIN > 1 ? 1 : 0][st][lane] : 0.0f);
          };
          if ((T)rmin >= s8w)
            run(BoolTag<true>{});
          else
            run(BoolTag<false>{});
          flush();
        }
        __syncthreads();
      }
    } else {
      for (int i0 = a.i_lo; i0 < a.i_hi; i0 += kChunk) {
        const int i1 = min(a.i_hi, i0 + kChunk);
        for (int i = i0; i < i1; ++i) {
          const long long gidx = (long long)i * a.nf + fi;
          const T q0 = __ldg(static_cast<const T*>(a.gb[0]) + gidx);
          const T q1 = MT::NIN > 1 ? __ldg(static_cast<const T*>(a.gb[1]) + gidx) : T(0);
          station(BoolTag<false>{}, __ldg(a.geo + i), q0, q1);
        }
        flush();
      }
    }
    if (!c_valid) return;
    if (a.part) {  // raw sums of this station range
#pragma unroll
      for (int j = 0; j < CPT; ++j)
        if (f_valid && c0 + j < a.nc)
#pragma unroll
          for (int q = 0; q < MT::NACC; ++q)
            a.part[((long long)q * a.nc + c0 + j) * a.nf + fi] = (float)tot[j][q];
      return;
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const T gam = cell[j].gamma();
      T res[2];
      res[0] = gam * tot[j][0];
      res[1] = gam * tot[j][1];
      if (f_valid && c0 + j < a.nc) a.out[(long long)(c0 + j) * a.nf + fi] = finish<MODE, T>(res, T(1));
    }
  }
}

// Launches fj_prep_geom_kernel: drs [nr + 1] (drs[0] = drs[nr] = 0) and the
// trapezoid weights wtr [nr] of the sorted r.
void fj_prep_geom_kernel_shared(const float* rs, int nr, float* drs, float* wtr, cudaStream_t s);
// Default velocities per thread of the FP32 kernel for a mode and itype.
int default_cpt_for(int mode, int itype);
// Per (set, frequency) column normalisation of out[nsets][nc][nf].
int normalize_sets(float* out, int nsets, int nc, int nf, cudaStream_t s);

}  // namespace ccfj
