// Per-interval integral of the F-J transform, shared by the FP32 and FP64
// station-amortised kernels.
//
// The reference (src/FJcpu.cpp:253-268) sums, over the intervals [r1, r2] of
// the distance-sorted stations, the exact integral of the linearly
// interpolated spectrum times r Z0(k r):
//
//   int_{r1}^{r2} (a + b r) r Z0(k r) dr,   b = (g2 - g1) / max(r2 - r1, 0.1),
//                                            a = g1 - r1 b
//
// which, with x = k r and g1 + b (r - r1) = a + b r, is
//
//   (1/k^2) [ g1 I0 + (b/k) I1 ],   I0 = int_{x1}^{x2} h(x) dx,
//                                   I1 = int_{x1}^{x2} (x - x1) h(x) dx,
//                                   h(x) = x Z0(x).
//
// Closed forms (the reference's, regrouped): I0 = [x Z1] and
// I1 = x2 dx Z1(x2) + [x Z0] - [B], with B = int_0^x Z0. They lose about
// log10(2/dx^2) digits to cancellation when dx = k (r2 - r1) is small, which
// is why the FP32 reference is only ~1e-3 accurate at low frequency. For
// dx < tau this code uses instead the two-point quintic Hermite rule
//
//   int_0^H F = H/2 (F0 + F1) + H^2/10 (F0' - F1') + H^3/120 (F0'' + F1'')
//               - H^7/100800 F^(6)
//
// on h and (x - x1) h, whose derivatives follow from Z0' = -Z1,
// (x Z1)' = x Z0: h' = Z0 - x Z1, h'' = -Z1 - x Z0. It uses only the values
// already computed at the two stations, so both branches cost a handful of
// FMAs and the special functions stay evaluated once per station.
#pragma once

#include "fj_special.cuh"

namespace fjs {

// What one station contributes to its two intervals, for one basis.
template <typename T>
struct Station {
  T h;    // x Z0
  T hp;   // h'  = Z0 - x Z1
  T hpp;  // h'' = -Z1 - x Z0
  T xz1;  // x Z1
  T b;    // int_0^x Z0
};

template <typename T>
FJ_HD Station<T> make_station(T x, const ZB<T>& z) {
  Station<T> s;
  s.h = x * z.z0;
  s.xz1 = x * z.z1;
  s.hp = z.z0 - s.xz1;
  s.hpp = -(z.z1 + s.h);
  s.b = z.b;
  return s;
}

// I0, I1 of the interval from station a (at x1) to station b (dx = x2 - x1,
// negative for the reversed intervals of unsorted input), by the closed form
// when `closed` (long intervals: see the kernels' closed_form) and by the
// quintic Hermite rule otherwise.
template <typename T>
FJ_HD void interval_moments(const Station<T>& a, const Station<T>& b, T dx, bool closed, T& I0,
                            T& I1) {
  if (closed) {
    I0 = b.xz1 - a.xz1;
    I1 = fmaT(dx, b.xz1, (b.h - a.h) - (b.b - a.b));
  } else {
    const T c1 = T(0.5) * dx;
    const T d2 = dx * dx;
    const T c2 = T(0.1) * d2;
    const T c3 = d2 * dx * T(1.0 / 120.0);
    I0 = fmaT(c1, a.h + b.h, fmaT(c2, a.hp - b.hp, c3 * (a.hpp + b.hpp)));
    const T g0 = dx * b.h;                               // G(x2),   G = (x - x1) h
    const T g0p = fmaT(dx, b.hp, b.h);                   // G'(x2)
    const T g0pp = fmaT(dx, b.hpp, T(2) * b.hp);         // G''(x2)
    // G(x1) = 0, G'(x1) = h1, G''(x1) = 2 h1'
    I1 = fmaT(c1, g0, fmaT(c2, a.h - g0p, c3 * fmaT(T(2), a.hp, g0pp)));
  }
}

#if defined(FJS_HAVE_PAIRED)
// Two stations (or two intervals) per paired FP32 instruction: the lanes
// carry independent values, each computed with make_station's and
// interval_moments' operations (a - b as fma(-1, b, a), a single rounding
// like the subtraction).
struct Station2 {
  float2 h, hp, hpp, xz1, b;
};

__device__ __forceinline__ float2 psub(float2 a, float2 b) { return pfma(psplat(-1.0f), b, a); }

__device__ __forceinline__ Station2 make_station_pair(float2 x, const ZB2& z, float2 b) {
  Station2 s;
  s.h = pmul(x, z.z0);
  s.xz1 = pmul(x, z.z1);
  s.hp = psub(z.z0, s.xz1);
  s.hpp = pmul(psplat(-1.0f), padd(z.z1, s.h));
  s.b = b;
  return s;
}

__device__ __forceinline__ Station<float> station_lane(const Station2& s, int lane) {
  return lane == 0 ? Station<float>{s.h.x, s.hp.x, s.hpp.x, s.xz1.x, s.b.x}
                   : Station<float>{s.h.y, s.hp.y, s.hpp.y, s.xz1.y, s.b.y};
}

// interval_moments of two intervals (a.x -> b.x, a.y -> b.y) that take the
// same rule.
__device__ __forceinline__ void interval_moments_pair(const Station2& a, const Station2& b,
                                                      float2 dx, bool closed, float2& I0,
                                                      float2& I1) {
  if (closed) {
    I0 = psub(b.xz1, a.xz1);
    I1 = pfma(dx, b.xz1, psub(psub(b.h, a.h), psub(b.b, a.b)));
  } else {
    const float2 c1 = pmul(psplat(0.5f), dx);
    const float2 d2 = pmul(dx, dx);
    const float2 c2 = pmul(psplat(0.1f), d2);
    const float2 c3 = pmul(pmul(d2, dx), psplat((float)(1.0 / 120.0)));
    I0 = pfma(c1, padd(a.h, b.h), pfma(c2, psub(a.hp, b.hp), pmul(c3, padd(a.hpp, b.hpp))));
    const float2 g0 = pmul(dx, b.h);
    const float2 g0p = pfma(dx, b.hp, b.h);
    const float2 g0pp = pfma(dx, b.hpp, pmul(psplat(2.0f), b.hp));
    I1 = pfma(c1, g0, pfma(c2, psub(a.h, g0p), pmul(c3, pfma(psplat(2.0f), a.hp, g0pp))));
  }
}
#endif

}  // namespace fjs
