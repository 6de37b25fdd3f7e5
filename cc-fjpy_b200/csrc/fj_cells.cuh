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
  float inv_k;
  float inv_k2;
  __device__ void init(float fl, float cl) {
    const double q = (double)fl / (double)cl;
    q_hi = (float)q;
    q_lo = (float)(q - (double)q_hi);
    const double kd = fjs::kTwoPi * q;
    k = (float)kd;
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
};
template <>
struct Cell<double> {
  double q, k, inv_k, inv_k2;
  __device__ void init(float fl, float cl) {
    q = (double)fl / (double)cl;
    k = fjs::kTwoPi * q;
    inv_k = 1.0 / k;
    inv_k2 = 1.0 / (k * k);
  }
  template <bool WJ, bool WY, bool WZ1>
  __device__ __forceinline__ void eval(double r, double x, bool need_b, ZB<double>& J,
                                       ZB<double>& Y) const {
    (void)need_b;
    fjs::eval_station_f64<WJ, WY, WZ1>(x, q * r, J, Y);
  }
};

struct FjDev {
  const float* rs;
  const float* drs;  // [nr + 1]: r_i - r_{i-1}, 0 at i = 0 and at i = nr
  const void* gb[2];
  const float* f;
  const float* c;
  float* out;
  int nr, nf, nc;
  float tau;
};

// ------------------------------------------------------------ preparation
// Gathers row perm[i] (or i) of one input, takes every u_cs-th element, and
// writes the per-interval pair (g_{i-1}, b_i) with b_i = (g_i - g_{i-1}) /
// max(r_i - r_{i-1}, 0.1) (src/FJcpu.cpp:259-261), or g_i * wtr_i for the
// trapezoid.
template <typename T>
__global__ void fj_prep_u_kernel(InDesc in, int nr, int nf, const float* __restrict__ drs,
                                 const float* __restrict__ wtr, int itype, void* __restrict__ dst) {
  // pairs on grid x (no 65535 limit), frequencies on grid y
  const int fi = blockIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  if (fi >= nf || i >= nr) return;
  const long long* perm = in.perm;
  const long long row = perm ? perm[i] : i;
  const T g = (T)in.p[row * in.ld + (long long)fi * in.cs];
  if (itype == 1) {
    using T2 = typename Vec2<T>::type;
    T2 v;
    if (i == 0) {
      v.x = 0;
      v.y = 0;
    } else {
      const long long rowp = perm ? perm[i - 1] : i - 1;
      const T gp = (T)in.p[rowp * in.ld + (long long)fi * in.cs];
      const T dr0 = (T)fmaxf(drs[i], 0.1f);
      v.x = gp;
      v.y = (g - gp) / dr0;
    }
    static_cast<T2*>(dst)[(long long)i * nf + fi] = v;
  } else {
    static_cast<T*>(dst)[(long long)i * nf + fi] = g * (T)wtr[i];
  }
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
    if (MODE == CCFJ_MODE_J_MINUS_Y) {
      acc[0] += g0 * zJ - g1 * zY;
    } else if (MODE == CCFJ_MODE_ABS_J) {
      acc[0] = fjs::fmaT(g0, zJ, acc[0]);
      acc[1] = fjs::fmaT(g1, zJ, acc[1]);
    } else {
      acc[0] += g0 * zJ - g1 * zY;
      acc[1] += g1 * zJ + g0 * zY;
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

// CPT cells (f, c), (f, c + 1), ... per thread share the per-station loads.
// The transform of the CPT cells (fi, c0), (fi, c0 + 1), ... of one data
// set; shared by the grid kernel below and the persistent batch kernel.
template <int MODE, int ITYPE, typename T, int CPT>
__device__ __forceinline__ void fj_cells(const FjDev& a, int fi, int c0) {
  using MT = ModeTraits<MODE>;
  constexpr bool WJ = MT::WJ, WY = MT::WY;
  if (fi >= a.nf || c0 >= a.nc) return;
  Cell<T> cell[CPT];
  const float fl = a.f[fi];
#pragma unroll
  for (int j = 0; j < CPT; ++j) cell[j].init(fl, a.c[min(c0 + j, a.nc - 1)]);
  T tot[CPT][2];
#pragma unroll
  for (int j = 0; j < CPT; ++j) tot[j][0] = tot[j][1] = T(0);
  ZB<T> Jz{}, Yz{};
  if (ITYPE == 1) {
    const T tau = (T)a.tau;
    Station<T> sJp[CPT], sYp[CPT];
    T xp[CPT];
    T r_cur = (T)__ldg(a.rs);
    T dr_next = (T)__ldg(a.drs + 1);  // drs has nr + 1 entries, the last 0
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      xp[j] = cell[j].k * r_cur;
      const bool nb = closed_form<T, WY>(cell[j].k * dr_next, xp[j], tau);  // Y rule: superset
      cell[j].template eval<WJ, WY, true>(r_cur, xp[j], nb, Jz, Yz);
      if (WJ) sJp[j] = fjs::make_station(xp[j], Jz);
      if (WY) sYp[j] = fjs::make_station(xp[j], Yz);
    }
    // lnJ/lnY[j]: interval (i, i+1) of cell j takes the closed form in the
    // J / Y basis (the Y rule also sends near-origin intervals there)
    bool lnJ[CPT], lnY[CPT];
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      lnJ[j] = closed_form<T, false>(cell[j].k * dr_next, xp[j], tau);
      lnY[j] = closed_form<T, true>(cell[j].k * dr_next, xp[j], tau);
    }
    for (int i0 = 1; i0 < a.nr; i0 += kChunk) {
      const int i1 = min(a.nr, i0 + kChunk);
      T acc[CPT][2];
#pragma unroll
      for (int j = 0; j < CPT; ++j) acc[j][0] = acc[j][1] = T(0);
#pragma unroll 2
      for (int i = i0; i < i1; ++i) {
        const T r = (T)__ldg(a.rs + i);
        const T dr = dr_next;
        dr_next = (T)__ldg(a.drs + i + 1);
        using T2 = typename Vec2<T>::type;
        const long long gidx = (long long)i * a.nf + fi;
        const T2 g0 = __ldg(static_cast<const T2*>(a.gb[0]) + gidx);
        T2 g1;
        if (MT::NIN > 1) g1 = __ldg(static_cast<const T2*>(a.gb[1]) + gidx);
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
          const T x = cell[j].k * r;
          const T dx = cell[j].k * dr;
          const bool lcJ = lnJ[j], lcY = lnY[j];
          const T dxn = cell[j].k * dr_next;
          if (WJ) lnJ[j] = closed_form<T, false>(dxn, x, tau);
          if (WY) lnY[j] = closed_form<T, true>(dxn, x, tau);
          // B is needed where an adjacent interval takes the closed form
          const bool nb = WY ? (lcY || lnY[j]) : (lcJ || lnJ[j]);
          cell[j].template eval<WJ, WY, true>(r, x, nb, Jz, Yz);
          T I0J = 0, I1J = 0, I0Y = 0, I1Y = 0;
          if (WJ) {
            const Station<T> sJ = fjs::make_station(x, Jz);
            fjs::interval_moments<T>(sJp[j], sJ, dx, lcJ, I0J, I1J);
            sJp[j] = sJ;
          }
          if (WY) {
            const Station<T> sY = fjs::make_station(x, Yz);
            fjs::interval_moments<T>(sYp[j], sY, dx, lcY, I0Y, I1Y);
            sYp[j] = sY;
          }
          accumulate_interval<MODE, T>(acc[j], g0, g1, I0J, I1J * cell[j].inv_k, I0Y,
                                       I1Y * cell[j].inv_k);
          xp[j] = x;
        }
      }
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        tot[j][0] += acc[j][0];
        tot[j][1] += acc[j][1];
      }
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j)
      if (c0 + j < a.nc) a.out[(long long)(c0 + j) * a.nf + fi] = finish<MODE, T>(tot[j], cell[j].inv_k2);
  } else {
    for (int i0 = 0; i0 < a.nr; i0 += kChunk) {
      const int i1 = min(a.nr, i0 + kChunk);
      T acc[CPT][2];
#pragma unroll
      for (int j = 0; j < CPT; ++j) acc[j][0] = acc[j][1] = T(0);
      for (int i = i0; i < i1; ++i) {
        const T r = (T)__ldg(a.rs + i);
        const long long gidx = (long long)i * a.nf + fi;
        const T g0 = __ldg(static_cast<const T*>(a.gb[0]) + gidx);
        T g1 = T(0);
        if (MT::NIN > 1) g1 = __ldg(static_cast<const T*>(a.gb[1]) + gidx);
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
          cell[j].template eval<WJ, WY, false>(r, cell[j].k * r, false, Jz, Yz);
          accumulate_station<MODE, T>(acc[j], g0, g1, WJ ? Jz.z0 : T(0), WY ? Yz.z0 : T(0));
        }
      }
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        tot[j][0] += acc[j][0];
        tot[j][1] += acc[j][1];
      }
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j)
      if (c0 + j < a.nc) a.out[(long long)(c0 + j) * a.nf + fi] = finish<MODE, T>(tot[j], T(1));
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
