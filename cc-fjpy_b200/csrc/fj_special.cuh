// Special functions of the F-J transform, in FP32 (fast path) and FP64
// (comparator path), compiled for both device and host (host copies back the
// CPU unit tests of the approximations).
//
// What the transform needs at every station x = k r:
//   Z0(x), Z1(x)   with Z = J (Bessel basis) or Y (Hankel imaginary part)
//   B(x) = int_0^x Z0(t) dt
// The reference evaluates these with Numerical-Recipes rational forms and
// Zhang & Jin Struve series (src/FJcpu.cpp:21-228), twice per interval and in
// loops of up to 60 terms. Here every function is a fixed-degree polynomial
// on four ranges (coefficients from gen_fj_special.py, fitted to mpmath
// values), and the oscillating factor of the x >= 8 range comes from ONE
// sin/cos pair of chi = x - pi/4 shared by J0, J1, Y0, Y1 and both B's.
//
// Phase accuracy: x reaches ~1e4 rad, where an FP32 x carries ~5e-4 rad of
// error. The caller therefore passes the phase in cycles, t = f r / c, as an
// unevaluated sum t = p_hi + p_lo (double-float, FP32 only) or as a double;
// the integer part of t is removed exactly before any rounding.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "fj_special_coeffs.h"

#ifdef __CUDACC__
#define FJ_HD __host__ __device__ __forceinline__
#else
#define FJ_HD inline
#endif

namespace fjs {

constexpr float kTwoPiF = 6.28318530717958647692f;
constexpr double kTwoPi = 6.28318530717958647692;
constexpr double kPi = 3.14159265358979323846;
constexpr float kSqrt2OverPiF = 0.79788456080286535588f;  // sqrt(2/pi)
constexpr double kSqrt2OverPi = 0.79788456080286535588;
constexpr float kTwoOverPiF = 0.63661977236758134308f;
constexpr double kTwoOverPi = 0.63661977236758134308;

// ------------------------------------------------------------- primitives
FJ_HD float fmaT(float a, float b, float c) { return fmaf(a, b, c); }
FJ_HD double fmaT(double a, double b, double c) { return fma(a, b, c); }

FJ_HD int32_t f2i_bits(float v) {
#ifdef __CUDA_ARCH__
  return __float_as_int(v);
#else
  int32_t i;
  memcpy(&i, &v, 4);
  return i;
#endif
}
FJ_HD float i2f_bits(int32_t i) {
#ifdef __CUDA_ARCH__
  return __int_as_float(i);
#else
  float v;
  memcpy(&v, &i, 4);
  return v;
#endif
}
FJ_HD float rcp_fast(float x) {
#ifdef __CUDA_ARCH__
  return __fdividef(1.0f, x);
#else
  return 1.0f / x;
#endif
}
// The SFU approximations below use their flush-to-zero forms: arguments and
// results here are never subnormal in any way that matters (a subnormal
// sine argument is 0 to within 1e-38), and the forms need no subnormal
// fix-up instructions.
FJ_HD float rsqrt_fast(float x) {
#ifdef __CUDA_ARCH__
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
#else
  return 1.0f / sqrtf(x);
#endif
}
// sqrt by the SFU's approximation (one MUFU op, relative error ~1 ulp).
FJ_HD float sqrt_fast(float x) {
#ifdef __CUDA_ARCH__
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
#else
  return sqrtf(x);
#endif
}
FJ_HD float log_fast(float x) {
#ifdef __CUDA_ARCH__
  return __logf(x);
#else
  return logf(x);
#endif
}

// Horner evaluation of a fixed coefficient list (lowest degree first).
template <typename T, int N>
FJ_HD T horner(const T (&c)[N], T v) {
  T acc = c[N - 1];
#pragma unroll
  for (int i = N - 2; i >= 0; --i) acc = fmaT(acc, v, c[i]);
  return acc;
}

// Values at one station for one basis: Z0, Z1 and B = int_0^x Z0.
template <typename T>
struct ZB {
  T z0, z1, b;
};

// ------------------------------------------------ phase reduction (FP64)
// t = x / (2 pi) in cycles as one double (|t| < 2^40 keeps >= 12 bits of
// fraction). Output: sin and cos of chi = x - pi/4 = 2 pi (t - 1/8). The
// integer part n of t is removed first (t - n is exact), the quarter-turn
// count q next (a - q exact); sin/cos of (pi/2) v, |v| <= 1/2, are
// polynomials and q mod 4 rotates them.
FJ_HD void sincos_chi_f64(double t, double& s_chi, double& c_chi) {
  const double n = rint(t);
  const double a = 4.0 * (t - n) - 0.5;  // exact up to the rounding of t
  const double qf = rint(a);
  const int q = (int)qf;
  const double v = a - qf;
  const double v2 = v * v;
  constexpr double cs[] = FJC_F64_SIN;
  constexpr double cc[] = FJC_F64_COS;
  const double s = v * horner(cs, v2);
  const double c = horner(cc, v2);
  const bool odd = (q & 1) != 0;
  double ss = odd ? c : s;
  double cc2 = odd ? s : c;
  if (q & 2) ss = -ss;
  if ((q + 1) & 2) cc2 = -cc2;
  s_chi = ss;
  c_chi = cc2;
}

// ------------------------------------------------ phase reduction, fast
// chi / (2 pi) = t - 1/8 reduced to [-5/8, 1/2] cycles: the integer part of
// p_hi is removed exactly (p_hi - n is exact), p_lo and the 1/8 shift are
// added after, so the only rounding is that of the final sum (< 3e-8 cycle).
FJ_HD float chi_cycles_f32(float p_hi, float p_lo) {
  const float kMagic = 12582912.0f;  // 1.5 * 2^23: x + M - M rounds |x| < 2^22
  const float n = (p_hi + kMagic) - kMagic;
  return (p_hi - n) + (p_lo - 0.125f);
}

// sin and cos of 2 pi u for |u| <= 5/8. On the device this is the SFU's
// sine/cosine (two MUFU ops, absolute error about 4e-7 on this range); the
// host build (used by the CPU tests of the polynomials) uses libm.
FJ_HD void sincos_cycles_f32(float u, float& s, float& c) {
#ifdef __CUDA_ARCH__
  const float a = kTwoPiF * u;
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(a));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(c) : "f"(a));
#else
  const double a = kTwoPi * (double)u;
  s = (float)sin(a);
  c = (float)cos(a);
#endif
}

// ------------------------------------------ station evaluation, FP32
// The x >= 8 range in Hankel form, returning the values divided by the
// Hankel amplitude M = sqrt(2 / (pi x)): y0 = Z0 / M, y1 = Z1 / M, and B
// itself (m = M is read only when need_b). s = 8 / x; p_hi + p_lo = x / (2 pi)
// in cycles (double-float). Without the amplitude the four polynomials need
// no scaling, and a caller that can fold M elsewhere (the folded interval
// sum does) never forms it.
template <bool WANT_J, bool WANT_Y, bool WANT_Z1>
FJ_HD void eval_large_scaled_f32(float s, float p_hi, float p_lo, bool need_b, float m,
                                 ZB<float>& J, ZB<float>& Y) {
  float sn, cs;
  sincos_cycles_f32(chi_cycles_f32(p_hi, p_lo), sn, cs);
  const float z = s * s;
  constexpr float cp0[] = FJC_F32_L_P0;
  constexpr float cq0[] = FJC_F32_L_Q0;
  const float P0 = horner(cp0, z);
  const float Q0 = horner(cq0, z) * s;
  float P1 = 0.f, Q1 = 0.f;
  if (WANT_Z1) {
    constexpr float cp1[] = FJC_F32_L_P1;
    constexpr float cq1[] = FJC_F32_L_Q1;
    P1 = horner(cp1, z);
    Q1 = horner(cq1, z) * s;
  }
  if (WANT_J) {
    J.z0 = fmaT(P0, cs, -Q0 * sn);
    if (WANT_Z1) J.z1 = fmaT(P1, sn, Q1 * cs);
  }
  if (WANT_Y) {
    Y.z0 = fmaT(P0, sn, Q0 * cs);
    if (WANT_Z1) Y.z1 = fmaT(Q1, sn, -P1 * cs);
  }
  if (WANT_Z1 && need_b) {
    constexpr float cr0[] = FJC_F32_L_RHO0;
    constexpr float cr1[] = FJC_F32_L_RHO1;
    const float rho0 = horner(cr0, z);
    const float rho1 = horner(cr1, z) * s;
    // B_J = 1 + J1 rho0 - J0 rho1, B_Y = Y1 rho0 - Y0 rho1 (Wronskian form)
    if (WANT_J) J.b = fmaT(m, fmaT(J.z1, rho0, -J.z0 * rho1), 1.0f);
    if (WANT_Y) Y.b = m * fmaT(Y.z1, rho0, -Y.z0 * rho1);
  }
}

// The x < 8 ranges: polynomials in (x - xc) / 1.5 for 2 <= x < 8, and in
// (x/2)^2 with the log term of Y for x < 2. Z0, Z1 and B themselves.
template <bool WANT_J, bool WANT_Y, bool WANT_Z1>
FJ_HD void eval_small_f32(float x, bool need_b, ZB<float>& J, ZB<float>& Y) {
  if (x >= 2.0f) {
    const bool hi = x >= 5.0f;
    const float u = (x - (hi ? 6.5f : 3.5f)) * (1.0f / 1.5f);
    if (hi) {
      if (WANT_J) {
        constexpr float c0[] = FJC_F32_S2_J0;
        J.z0 = horner(c0, u);
        if (WANT_Z1) {
          constexpr float c1[] = FJC_F32_S2_J1;
          J.z1 = horner(c1, u);
          if (need_b) {
            constexpr float cb[] = FJC_F32_S2_BJ;
            J.b = horner(cb, u);
          }
        }
      }
      if (WANT_Y) {
        constexpr float c0[] = FJC_F32_S2_Y0;
        Y.z0 = horner(c0, u);
        if (WANT_Z1) {
          constexpr float c1[] = FJC_F32_S2_Y1;
          Y.z1 = horner(c1, u);
          if (need_b) {
            constexpr float cb[] = FJC_F32_S2_BY;
            Y.b = horner(cb, u);
          }
        }
      }
    } else {
      if (WANT_J) {
        constexpr float c0[] = FJC_F32_S1_J0;
        J.z0 = horner(c0, u);
        if (WANT_Z1) {
          constexpr float c1[] = FJC_F32_S1_J1;
          J.z1 = horner(c1, u);
          if (need_b) {
            constexpr float cb[] = FJC_F32_S1_BJ;
            J.b = horner(cb, u);
          }
        }
      }
      if (WANT_Y) {
        constexpr float c0[] = FJC_F32_S1_Y0;
        Y.z0 = horner(c0, u);
        if (WANT_Z1) {
          constexpr float c1[] = FJC_F32_S1_Y1;
          Y.z1 = horner(c1, u);
          if (need_b) {
            constexpr float cb[] = FJC_F32_S1_BY;
            Y.b = horner(cb, u);
          }
        }
      }
    }
  } else {
    const float w = 0.25f * x * x;
    constexpr float ca[] = FJC_F32_S0_A;
    const float j0 = horner(ca, w);
    float j1 = 0.f, bj = 0.f;
    if (WANT_Z1) {
      constexpr float cb[] = FJC_F32_S0_B;
      j1 = x * horner(cb, w);
      if (need_b) {
        constexpr float cc[] = FJC_F32_S0_C;
        bj = x * horner(cc, w);
      }
    }
    if (WANT_J) {
      J.z0 = j0;
      if (WANT_Z1) {
        J.z1 = j1;
        if (need_b) J.b = bj;
      }
    }
    if (WANT_Y) {
      constexpr float cd[] = FJC_F32_S0_D;
      const float L = kTwoOverPiF * log_fast(0.5f * x);
      Y.z0 = fmaT(L, j0, horner(cd, w));
      if (WANT_Z1) {
        constexpr float ce[] = FJC_F32_S0_E;
        Y.z1 = fmaT(L, j1, fmaT(x, horner(ce, w), -kTwoOverPiF * rcp_fast(x)));
        if (need_b) {
          constexpr float cf[] = FJC_F32_S0_F;
          Y.b = fmaT(L, bj, x * horner(cf, w));
        }
      }
    }
  }
}

// x: the argument (FP32, for the smooth parts and the range choice);
// p_hi + p_lo: x / (2 pi) in cycles (double-float, for the phase).
// WANT_J / WANT_Y select the basis, WANT_Z1 adds Z1 (the integral forms
// need it, the trapezoid does not); B = int_0^x Z0 is computed only when
// need_b (the closed form of a long interval next to this station needs it;
// the Hermite rule of short intervals does not).
template <bool WANT_J, bool WANT_Y, bool WANT_Z1>
FJ_HD void eval_station_f32(float x, float p_hi, float p_lo, bool need_b, ZB<float>& J,
                            ZB<float>& Y) {
  if (x >= 8.0f) {
    const float rs = rsqrt_fast(x);  // one MUFU op gives both 1/sqrt(x) and 1/x
    const float M = kSqrt2OverPiF * rs;
    eval_large_scaled_f32<WANT_J, WANT_Y, WANT_Z1>(8.0f * (rs * rs), p_hi, p_lo, need_b, M, J, Y);
    if (WANT_J) {
      J.z0 *= M;
      if (WANT_Z1) J.z1 *= M;
    }
    if (WANT_Y) {
      Y.z0 *= M;
      if (WANT_Z1) Y.z1 *= M;
    }
  } else {
    eval_small_f32<WANT_J, WANT_Y, WANT_Z1>(x, need_b, J, Y);
  }
}

// ------------------------------------------ station evaluation, FP64
template <bool WANT_J, bool WANT_Y, bool WANT_B>
FJ_HD void eval_station_f64(double x, double t, ZB<double>& J, ZB<double>& Y) {
  if (x >= 8.0) {
    double sn, cs;
    sincos_chi_f64(t, sn, cs);
    const double s = 8.0 / x;
    const double z = s * s;
    const double M = kSqrt2OverPi / sqrt(x);
    constexpr double cp0[] = FJC_F64_L_P0;
    constexpr double cq0[] = FJC_F64_L_Q0;
    constexpr double cp1[] = FJC_F64_L_P1;
    constexpr double cq1[] = FJC_F64_L_Q1;
    const double P0 = horner(cp0, z) * M;
    const double Q0 = horner(cq0, z) * (s * M);
    const double P1 = horner(cp1, z) * M;
    const double Q1 = horner(cq1, z) * (s * M);
    double rho0 = 0, rho1 = 0;
    if (WANT_B) {
      constexpr double cr0[] = FJC_F64_L_RHO0;
      constexpr double cr1[] = FJC_F64_L_RHO1;
      rho0 = horner(cr0, z);
      rho1 = horner(cr1, z) * s;
    }
    if (WANT_J) {
      J.z0 = P0 * cs - Q0 * sn;
      J.z1 = P1 * sn + Q1 * cs;
      if (WANT_B) J.b = 1.0 + J.z1 * rho0 - J.z0 * rho1;
    }
    if (WANT_Y) {
      Y.z0 = P0 * sn + Q0 * cs;
      Y.z1 = Q1 * sn - P1 * cs;
      if (WANT_B) Y.b = Y.z1 * rho0 - Y.z0 * rho1;
    }
  } else if (x >= 2.0) {
    const bool hi = x >= 5.0;
    const double u = (x - (hi ? 6.5 : 3.5)) / 1.5;
    if (hi) {
      if (WANT_J) {
        constexpr double c0[] = FJC_F64_S2_J0;
        constexpr double c1[] = FJC_F64_S2_J1;
        J.z0 = horner(c0, u);
        J.z1 = horner(c1, u);
        if (WANT_B) {
          constexpr double cb[] = FJC_F64_S2_BJ;
          J.b = horner(cb, u);
        }
      }
      if (WANT_Y) {
        constexpr double c0[] = FJC_F64_S2_Y0;
        constexpr double c1[] = FJC_F64_S2_Y1;
        Y.z0 = horner(c0, u);
        Y.z1 = horner(c1, u);
        if (WANT_B) {
          constexpr double cb[] = FJC_F64_S2_BY;
          Y.b = horner(cb, u);
        }
      }
    } else {
      if (WANT_J) {
        constexpr double c0[] = FJC_F64_S1_J0;
        constexpr double c1[] = FJC_F64_S1_J1;
        J.z0 = horner(c0, u);
        J.z1 = horner(c1, u);
        if (WANT_B) {
          constexpr double cb[] = FJC_F64_S1_BJ;
          J.b = horner(cb, u);
        }
      }
      if (WANT_Y) {
        constexpr double c0[] = FJC_F64_S1_Y0;
        constexpr double c1[] = FJC_F64_S1_Y1;
        Y.z0 = horner(c0, u);
        Y.z1 = horner(c1, u);
        if (WANT_B) {
          constexpr double cb[] = FJC_F64_S1_BY;
          Y.b = horner(cb, u);
        }
      }
    }
  } else {
    const double w = 0.25 * x * x;
    constexpr double ca[] = FJC_F64_S0_A;
    constexpr double cb[] = FJC_F64_S0_B;
    constexpr double cc[] = FJC_F64_S0_C;
    const double j0 = horner(ca, w);
    const double j1 = x * horner(cb, w);
    const double bj = WANT_B ? x * horner(cc, w) : 0.0;
    if (WANT_J) {
      J.z0 = j0;
      J.z1 = j1;
      if (WANT_B) J.b = bj;
    }
    if (WANT_Y) {
      constexpr double cd[] = FJC_F64_S0_D;
      constexpr double ce[] = FJC_F64_S0_E;
      constexpr double cf[] = FJC_F64_S0_F;
      const double L = kTwoOverPi * log(0.5 * x);
      Y.z0 = L * j0 + horner(cd, w);
      Y.z1 = L * j1 + x * horner(ce, w) - kTwoOverPi / x;
      if (WANT_B) Y.b = L * bj + x * horner(cf, w);
    }
  }
}

// ------------------------------------------ paired evaluation (sm_100)
// Two cells (two velocities of one frequency) at one station: every FP32
// operation of eval_large_scaled_f32 on both lanes as one paired
// instruction (FFMA2 / FMUL2 / FADD2 on sm_100). Each lane performs exactly
// the scalar function's operations in the same order with the same
// rounding -- negated quantities come from negated inputs or coefficients,
// which round-to-nearest maps to exactly negated results -- with about half
// the instructions; tests/test_special_host.py holds it to the scalar path
// on the device.
#if defined(__CUDACC__)
#if !defined(__CUDA_ARCH__) || __CUDA_ARCH__ >= 1000
#define FJS_HAVE_PAIRED 1
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psplat(float v) { return make_float2(v, v); }

template <int N>
__device__ __forceinline__ float2 phorner(const float (&c)[N], float2 v) {
  float2 acc = psplat(c[N - 1]);
#pragma unroll
  for (int i = N - 2; i >= 0; --i) acc = pfma(acc, v, psplat(c[i]));
  return acc;
}
// The same with every coefficient negated: exactly -phorner(c, v).
template <int N>
__device__ __forceinline__ float2 phorner_neg(const float (&c)[N], float2 v) {
  float2 acc = psplat(-c[N - 1]);
#pragma unroll
  for (int i = N - 2; i >= 0; --i) acc = pfma(acc, v, psplat(-c[i]));
  return acc;
}

struct ZB2 {
  float2 z0, z1;
};

// Per-pair constants: the phase factor q = f / c as a double-float
// (q_hi, q_lo), -q_hi, and s8 = 8 / k of each lane's cell.
struct PairPhase {
  float2 qhi, nqhi, qlo, s8;
};

// sincos_cycles_f32(chi_cycles_f32(p_hi, p_lo)) of both lanes: the
// reduction to cycles (the magic-number rounding and the sums after it) and
// the 2 pi scaling are round-to-nearest adds and a multiply, so the paired
// forms give each lane's bits; the sine and cosine stay per lane.
__device__ __forceinline__ void sincos_cycles_pair(float2 p_hi, float2 p_lo, float2& sn,
                                                   float2& cs) {
  const float kMagic = 12582912.0f;  // as chi_cycles_f32
  const float2 n = padd(padd(p_hi, psplat(kMagic)), psplat(-kMagic));
  const float2 u = padd(pfma(psplat(-1.0f), n, p_hi), padd(p_lo, psplat(-0.125f)));
#ifdef __CUDA_ARCH__
  const float2 arg = pmul(psplat(kTwoPiF), u);
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(sn.x) : "f"(arg.x));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(cs.x) : "f"(arg.x));
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(sn.y) : "f"(arg.y));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(cs.y) : "f"(arg.y));
#else
  sincos_cycles_f32(u.x, sn.x, cs.x);
  sincos_cycles_f32(u.y, sn.y, cs.y);
#endif
}

// eval_large_scaled_f32<true, false, true> (need_b false) of both lanes at
// the station r (1/r = rinv): y0 = J0 / M and y1 = J1 / M, x >= 8 in both.
__device__ __forceinline__ void eval_large_scaled_pair_j(const PairPhase& ph, float r, float rinv,
                                                         ZB2& J) {
  // The double-float phase in cycles, per lane with the scalar code (p_hi =
  // q_hi r, p_lo = fma(q_lo, r, fma(q_hi, r, -p_hi))): written with paired
  // operations it measured about 2e-3 rad less accurate at x = 3e4, as if
  // the low part had been lost. Its reduction to cycles is paired.
  float2 p_hi, p_lo;
  p_hi.x = ph.qhi.x * r;
  p_lo.x = fmaf(ph.qlo.x, r, fmaf(ph.qhi.x, r, -p_hi.x));
  p_hi.y = ph.qhi.y * r;
  p_lo.y = fmaf(ph.qlo.y, r, fmaf(ph.qhi.y, r, -p_hi.y));
  float2 sn, cs;
  sincos_cycles_pair(p_hi, p_lo, sn, cs);
  const float2 sv = pmul(ph.s8, psplat(rinv));  // s = 8 / x
  const float2 z = pmul(sv, sv);
  constexpr float cp0[] = FJC_F32_L_P0;
  constexpr float cq0[] = FJC_F32_L_Q0;
  constexpr float cp1[] = FJC_F32_L_P1;
  constexpr float cq1[] = FJC_F32_L_Q1;
  const float2 P0 = phorner(cp0, z);
  const float2 nQ0 = pmul(phorner_neg(cq0, z), sv);  // -Q0
  const float2 P1 = phorner(cp1, z);
  const float2 Q1 = pmul(phorner(cq1, z), sv);
  J.z0 = pfma(P0, cs, pmul(nQ0, sn));  // fma(P0, cs, -Q0 sn)
  J.z1 = pfma(P1, sn, pmul(Q1, cs));   // fma(P1, sn, Q1 cs)
}

// eval_station_f32<true, false, true> at two stations of one cell, x >= 8
// in both (lanes are stations): J0, J1 (times the amplitude) and, with
// need_b, B of both lanes. p_hi / p_lo: each lane's phase x / (2 pi) in
// cycles, formed by the caller with the scalar code.
__device__ __forceinline__ void eval_large_pair_stations_j(float2 x, float2 p_hi, float2 p_lo,
                                                           bool need_b, ZB2& J, float2& B) {
  float2 sn, cs;
  sincos_cycles_pair(p_hi, p_lo, sn, cs);
  const float2 rs = make_float2(rsqrt_fast(x.x), rsqrt_fast(x.y));
  const float2 M = pmul(psplat(kSqrt2OverPiF), rs);
  const float2 s = pmul(psplat(8.0f), pmul(rs, rs));
  const float2 z = pmul(s, s);
  constexpr float cp0[] = FJC_F32_L_P0;
  constexpr float cq0[] = FJC_F32_L_Q0;
  constexpr float cp1[] = FJC_F32_L_P1;
  constexpr float cq1[] = FJC_F32_L_Q1;
  const float2 P0 = phorner(cp0, z);
  const float2 nQ0 = pmul(phorner_neg(cq0, z), s);  // -Q0
  const float2 P1 = phorner(cp1, z);
  const float2 Q1 = pmul(phorner(cq1, z), s);
  const float2 y0 = pfma(P0, cs, pmul(nQ0, sn));
  const float2 y1 = pfma(P1, sn, pmul(Q1, cs));
  if (need_b) {
    // B_J = 1 + M (y1 rho0 - y0 rho1)
    constexpr float cr0[] = FJC_F32_L_RHO0;
    constexpr float cr1[] = FJC_F32_L_RHO1;
    const float2 rho0 = phorner(cr0, z);
    const float2 nrho1 = pmul(phorner_neg(cr1, z), s);  // -rho1
    B = pfma(M, pfma(y1, rho0, pmul(y0, nrho1)), psplat(1.0f));
  }
  J.z0 = pmul(y0, M);
  J.z1 = pmul(y1, M);
}
#endif
#endif

}  // namespace fjs
