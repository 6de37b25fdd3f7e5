// The F-J transform on one B200: data preparation, the station-amortised
// FP32 / FP64 kernels, the FP64 comparator with the reference's loop
// structure, the per-frequency normalisation, and the C-ABI entries
// FJ / FHr / FHi / FH / ccfj_fj_v1.
//
// Reference path (file:line in CC-FJpy):
//   fj_noise / fj_earthquake         src/ccfj-gpu.pyx:241-295
//   FJ / FHr / FHi host launchers    src/FJgpu.cu:390-483
//   integral_J / integral_Y          src/FJcpu.cpp:230-319  (the oracle)
//   trap_J / trap_Y                  src/FJcpu.cpp:323-399
//
// Layout in HBM (all row-major, frequency fastest, as in the reference):
//   rs   [nr]        float   sorted distances
//   drs  [nr + 1]    float   r_i - r_{i-1} (drs[0] = drs[nr] = 0)
//   wtr  [nr]        float   trapezoid weight r_i (dr0_i + dr0_{i+1}) / 2
//   geo  [nr]        float4  (r_i, r_{i+1} - r_i, 1/r_i, sqrt(r_i))
//   kb   [nf]        T       itype 1: fold threshold per frequency
//   gb   [nr][nf]    StationCoef<T> (A, B, C, g) per station, itype 1
//                    T       g_i wtr_i / sqrt(r_i), itype 0
//   out  [nc][nf]    float
// A thread owns CPT velocities of one frequency and walks all stations in
// order; a warp spans 32 consecutive frequencies of one velocity row and a
// CTA 8 rows, which share the chunks of station data staged in shared
// memory (fj_cells.cuh).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "ccfj_core.cuh"
#include "fj_cells.cuh"
#include "fj_frontend.cuh"
#include "fj_interval.cuh"

namespace ccfj {

using fjs::Station;
using fjs::ZB;

// ------------------------------------------------------------ preparation
// drs, wtr, and (if geo) the itype-1 station geometry.
__global__ void fj_prep_geom_kernel(const float* __restrict__ rs, int nr, float* __restrict__ drs,
                                    float* __restrict__ wtr, float4* __restrict__ geo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == nr) drs[nr] = 0.0f;  // padding read by the kernels' one-station lookahead
  if (i >= nr) return;
  const float r = rs[i];
  const float dl = i > 0 ? r - rs[i - 1] : 0.0f;
  const float dr = i + 1 < nr ? rs[i + 1] - r : 0.0f;
  drs[i] = dl;
  if (geo) geo[i] = station_geometry(r, dr);
  // dr0 = fmaxf(r2 - r1, 0.1) per interval, as src/FJcpu.cpp:354
  const float w0 = i > 0 ? fmaxf(dl, 0.1f) : 0.0f;
  const float w1 = i + 1 < nr ? fmaxf(dr, 0.1f) : 0.0f;
  wtr[i] = (w0 + w1) * 0.5f * r;
}

template <int MODE, int ITYPE, typename T, int CPT>
__global__ void __launch_bounds__(256, fj_min_blocks<T>()) fj_amortized_kernel(FjDev a) {
  if (gridDim.z > 1) {
    // split launch: CTA layer z sums stations [z L, (z + 1) L) into its own
    // partial sums (fj_split_finish_kernel adds the layers in order)
    a.i_lo = blockIdx.z * a.split_len;
    a.i_hi = min(a.nr, a.i_lo + a.split_len);
    a.part += (long long)blockIdx.z * ModeTraits<MODE>::NACC * a.nc * a.nf;
  }
  // velocity tiles on grid x: the CTAs of one frequency tile run side by
  // side and share its station coefficients in L2
  fj_cells<MODE, ITYPE, T, CPT>(a, blockIdx.y * blockDim.x + threadIdx.x,
                                (blockIdx.x * blockDim.y + threadIdx.y) * CPT);
}

// Sum of the station ranges of a split launch, in range order (the result
// does not depend on how the ranges were scheduled), then the amplitude
// gamma(k), the mode's combination and NaN at k = 0, as fj_cells finishes
// an unsplit sum.
template <int MODE>
__global__ void fj_split_finish_kernel(const float* __restrict__ part, int nsplit,
                                       const float* __restrict__ f, const float* __restrict__ c,
                                       int nc, int nf, float* __restrict__ out) {
  const int fi = blockIdx.x * 32 + threadIdx.x;
  const int ci = blockIdx.y * 8 + threadIdx.y;
  if (fi >= nf || ci >= nc) return;
  constexpr int NACC = ModeTraits<MODE>::NACC;
  const long long plane = (long long)nc * nf, at = (long long)ci * nf + fi;
  float tot[2] = {0.f, 0.f};
  for (int z = 0; z < nsplit; ++z)
#pragma unroll
    for (int q = 0; q < NACC; ++q) tot[q] += part[((long long)z * NACC + q) * plane + at];
  Cell<float> cell;
  cell.init(f[fi], c[ci]);
  const float gam = cell.gamma();
  float res[2] = {gam * tot[0], gam * tot[1]};
  out[at] = cell.k == 0.0f ? __int_as_float(0x7fffffff) : finish<MODE, float>(res, 1.0f);
}

// ------------------------------------------ FP64 comparator (plain form)
// The reference loop of src/FJcpu.cpp:253-268 (integral) and :348-357
// (trapezoid) in FP64: every interval re-evaluates the special functions at
// both of its ends and combines them with a = g1 - r1 b and b as the
// reference does. Only the special functions differ (the accurate FP64 ones
// above instead of Numerical Recipes / Zhang-Jin loops).
template <bool IS_Y, int ITYPE>
__device__ __forceinline__ double plain_interval(const Cell<double>& cell, double g1, double g2,
                                                 double r1, double r2, double dr0) {
  ZB<double> J, Y, J2, Y2;
  if (ITYPE == 0) {
    cell.eval<!IS_Y, IS_Y, false>(r1, cell.k * r1, false, J, Y);
    cell.eval<!IS_Y, IS_Y, false>(r2, cell.k * r2, false, J2, Y2);
    const double z1 = IS_Y ? Y.z0 : J.z0, z2 = IS_Y ? Y2.z0 : J2.z0;
    return (g1 * z1 * r1 + g2 * z2 * r2) * dr0 * 0.5;
  }
  cell.eval<!IS_Y, IS_Y, true>(r1, cell.k * r1, true, J, Y);
  cell.eval<!IS_Y, IS_Y, true>(r2, cell.k * r2, true, J2, Y2);
  const ZB<double>& A = IS_Y ? Y : J;
  const ZB<double>& B = IS_Y ? Y2 : J2;
  const double k = cell.k;
  const double b = (g2 - g1) / dr0;
  const double a = g1 - r1 * b;
  double s = a * (r2 * B.z1 - r1 * A.z1) / k;
  s += b * (r2 * r2 * B.z1 - r1 * r1 * A.z1) / k;
  s += b * (r2 * B.z0 - r1 * A.z0) / k / k;
  s += -b * (B.b - A.b) / k / k / k;
  return s;
}

template <int MODE, int ITYPE>
__global__ void __launch_bounds__(256) fj_plain64_kernel(FjDev a, const float* g0p,
                                                         const float* g1p) {
  const int fi = blockIdx.x * blockDim.x + threadIdx.x;
  const int ci = blockIdx.y * blockDim.y + threadIdx.y;
  if (fi >= a.nf || ci >= a.nc) return;
  Cell<double> cell;
  cell.init(a.f[fi], a.c[ci]);
  double acc[2] = {0, 0};
  for (int i = 1; i < a.nr; ++i) {
    const double r1 = a.rs[i - 1], r2 = a.rs[i];
    const double dr0 = fmaxf(a.rs[i] - a.rs[i - 1], 0.1f);
    const long long i1 = (long long)(i - 1) * a.nf + fi, i2 = (long long)i * a.nf + fi;
    const double u1 = g0p[i1], u2 = g0p[i2];
    if (MODE == CCFJ_MODE_J) {
      acc[0] += plain_interval<false, ITYPE>(cell, u1, u2, r1, r2, dr0);
    } else if (MODE == CCFJ_MODE_Y) {
      acc[0] += plain_interval<true, ITYPE>(cell, u1, u2, r1, r2, dr0);
    } else {
      const double v1 = g1p[i1], v2 = g1p[i2];
      if (MODE == CCFJ_MODE_J_MINUS_Y) {
        acc[0] += plain_interval<false, ITYPE>(cell, u1, u2, r1, r2, dr0) -
                  plain_interval<true, ITYPE>(cell, v1, v2, r1, r2, dr0);
      } else if (MODE == CCFJ_MODE_ABS_J) {
        acc[0] += plain_interval<false, ITYPE>(cell, u1, u2, r1, r2, dr0);
        acc[1] += plain_interval<false, ITYPE>(cell, v1, v2, r1, r2, dr0);
      } else {
        acc[0] += plain_interval<false, ITYPE>(cell, u1, u2, r1, r2, dr0) -
                  plain_interval<true, ITYPE>(cell, v1, v2, r1, r2, dr0);
        acc[1] += plain_interval<false, ITYPE>(cell, v1, v2, r1, r2, dr0) +
                  plain_interval<true, ITYPE>(cell, u1, u2, r1, r2, dr0);
      }
    }
  }
  a.out[(long long)ci * a.nf + fi] = finish<MODE, double>(acc, 1.0);
}

void fj_prep_geom_kernel_shared(const float* rs, int nr, float* drs, float* wtr, cudaStream_t s) {
  fj_prep_geom_kernel<<<div_up(nr + 1, 256), 256, 0, s>>>(rs, nr, drs, wtr, nullptr);
}

// Gathered plain copy of one input, [nr][nf] float (for the comparator).
__global__ void fj_gather_kernel(InDesc in, int nr, int nf, float* __restrict__ dst) {
  const int fi = blockIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  if (fi >= nf || i >= nr) return;
  const long long row = in.perm ? in.perm[i] : i;
  dst[(long long)i * nf + fi] = in.p[row * in.ld + (long long)fi * in.cs];
}

// ------------------------------------------------------- normalisation
// out[:, i] /= max(|out[:, i]|) with Python's builtin max over the column
// (src/ccfj-gpu.pyx:266-267): the running maximum starts at row 0 and is
// replaced only by a strictly larger value, so a NaN in row 0 makes the
// column NaN while NaNs in later rows are skipped.
__global__ void fj_normalize_kernel(float* __restrict__ out, int nc, int nf) {
  __shared__ float red[8][33];
  __shared__ float colmax[32];
  const int fi = blockIdx.x * 32 + threadIdx.x;
  float m = -INFINITY;
  if (fi < nf)
    for (int c = threadIdx.y; c < nc; c += blockDim.y) m = fmaxf(m, fabsf(out[(long long)c * nf + fi]));
  red[threadIdx.y][threadIdx.x] = m;
  __syncthreads();
  if (threadIdx.y == 0) {
    for (int y = 1; y < (int)blockDim.y; ++y) m = fmaxf(m, red[y][threadIdx.x]);
    if (fi < nf) {
      const float first = fabsf(out[fi]);
      colmax[threadIdx.x] = isnan(first) ? first : m;
    }
  }
  __syncthreads();
  if (fi < nf) {
    const float d = colmax[threadIdx.x];
    for (int c = threadIdx.y; c < nc; c += blockDim.y) {
      const long long k = (long long)c * nf + fi;
      out[k] = out[k] / d;
    }
  }
}

// ------------------------------------------------------------ dispatch
namespace {

// Velocities per thread of the FP32 kernel (1, 2 or 4): more share the
// per-station loads and loop overhead, fewer keep more warps resident.
// 0 = automatic: the tuned choice for the problem class if one is recorded
// (ccfj_autotune_fj_v1), else the default of default_cpt_for.
std::atomic<int> g_force_cpt{0};

template <int MODE, typename T, int CPT>
void launch_amortized_cpt(int itype, const FjDev& d, cudaStream_t s) {
  const dim3 block(32, 8);
  const int nsplit = d.part ? div_up(d.nr, d.split_len) : 1;
  const dim3 grid(div_up(d.nc, 8 * CPT), div_up(d.nf, 32), nsplit);
  if (itype == 1)
    fj_amortized_kernel<MODE, 1, T, CPT><<<grid, block, 0, s>>>(d);
  else
    fj_amortized_kernel<MODE, 0, T, CPT><<<grid, block, 0, s>>>(d);
}

template <int MODE, typename T>
void launch_amortized(int itype, const FjDev& d, int cpt, cudaStream_t s) {
  if (sizeof(T) == 8 || cpt == 1)
    launch_amortized_cpt<MODE, T, 1>(itype, d, s);
  else if (cpt == 4)
    launch_amortized_cpt<MODE, T, 4>(itype, d, s);
  else
    launch_amortized_cpt<MODE, T, 2>(itype, d, s);
}

template <int MODE>
void launch_plain(int itype, const FjDev& d, const float* g0, const float* g1, cudaStream_t s) {
  const dim3 block(32, 8);
  const dim3 grid(div_up(d.nf, 32), div_up(d.nc, 8));
  if (itype == 1)
    fj_plain64_kernel<MODE, 1><<<grid, block, 0, s>>>(d, g0, g1);
  else
    fj_plain64_kernel<MODE, 0><<<grid, block, 0, s>>>(d, g0, g1);
}

template <int MODE>
void launch_mode(int prec, int itype, const FjDev& d, const float* g0, const float* g1, int cpt,
                 cudaStream_t s) {
  if (prec == CCFJ_PREC_FP32)
    launch_amortized<MODE, float>(itype, d, cpt, s);
  else if (prec == CCFJ_PREC_FP64)
    launch_amortized<MODE, double>(itype, d, 1, s);
  else
    launch_plain<MODE>(itype, d, g0, g1, s);
}

int nin_of(int mode) { return (mode == CCFJ_MODE_J || mode == CCFJ_MODE_Y) ? 1 : 2; }

}  // namespace

// ------------------------------------------------------------ autotuner
// The tuned table maps a problem class to the fastest tile choice --
// velocities per thread and station ranges -- on a device; classes are
// (mode, itype, log2 of nr, of nf, of nc).
namespace {
long long tune_key(const ccfj_fj_args& a) {
  auto lg = [](long long v) {
    int b = 0;
    while ((1LL << (b + 1)) <= v) ++b;
    return (long long)b;
  };
  return ((((long long)a.mode * 2 + a.itype) * 64 + lg(a.nr)) * 64 + lg(a.nf)) * 64 + lg(a.nc);
}
}  // namespace

// Untuned default (measured on the large-array workload, with the stations
// staged in shared memory): two velocities per thread in every itype-1 mode,
// four for the trapezoid.
int default_cpt_for(int mode, int itype) {
  (void)mode;
  return itype == 0 ? 4 : 2;
}


// A tuned choice is stored as cpt + 8 * nsplit (tuner "fj" of the table).
int tuned_cpt(const ccfj_fj_args& a) {
  int choice = 0;
  return tune_lookup("fj", tune_key(a), &choice) ? choice % 8 : default_cpt_for(a.mode, a.itype);
}

int tuned_split(const ccfj_fj_args& a) {
  int choice = 0;
  return tune_lookup("fj", tune_key(a), &choice) ? choice / 8 : 0;
}

// The variant a transform runs: the caller's choice (the autotuner's
// candidate), else ccfj_set_fj_variant's, else the tuned or default one.
static int variant_for(const ccfj_fj_args& a, int cpt) {
  if (cpt > 0) return cpt;
  const int forced = g_force_cpt.load(std::memory_order_relaxed);
  return forced > 0 ? forced : tuned_cpt(a);
}

// Station ranges of one FP32 transform (split launches): split_choice if
// given, else the tuned choice for the problem class, else enough ranges
// that the grid fills the SMs' resident slots when the (velocity tile x
// frequency tile) grid alone leaves them idle -- the largest n <= 4 with
// n x CTAs <= slots (one more CTA would start a second wave) and ranges of
// at least two station chunks.
constexpr int kSplitAlign = 32;  // multiple of every staged chunk (16 or 32 stations)
static int sm_count() {
  static std::atomic<int> cached{0};
  int v = cached.load(std::memory_order_relaxed);
  if (v == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cached.store(v, std::memory_order_relaxed);
  }
  return v;
}
std::atomic<int> g_force_split{0};
static int split_for(const ccfj_fj_args& a, int cpt, int split_choice) {
  if (split_choice > 0) return split_choice;
  const int forced = g_force_split.load(std::memory_order_relaxed);
  if (forced > 0) return forced;
  const int tuned = tuned_split(a);
  if (tuned > 0) return tuned;
  // a window of frequencies (col_begin, nf_total) decides as its whole
  // problem does, so that windows reproduce the full transform
  const int nf_all = a.nf_total > 0 ? a.nf_total : a.nf;
  const long long ctas = (long long)div_up(a.nc, 8 * cpt) * div_up(nf_all, 32);
  const long long slots = (long long)sm_count() * CCFJ_FJ_MIN_BLOCKS;
  int n = 1;
  for (int k = 2; k <= 4; ++k)
    if (k * ctas <= slots && a.nr >= 2 * kSplitAlign * k) n = k;
  return n;
}

// Bytes of the itype-1 per-station geometry and per-frequency fold
// thresholds, and of one input's interval data.
size_t geometry_bytes(const ccfj_fj_args& a) { return sizeof(float4) * (size_t)a.nr; }
size_t kbounds_bytes(const ccfj_fj_args& a) {
  return a.itype == 1 ? (a.precision == CCFJ_PREC_FP32 ? 4 : 8) * (size_t)a.nf : 0;
}
size_t interval_data_bytes(const ccfj_fj_args& a) {
  const size_t t = a.precision == CCFJ_PREC_FP32 ? 4 : 8;
  return (size_t)a.nr * a.nf * (a.itype == 1 ? 4 * t : t);
}

// Fills d.kb (itype 1) and d.gb[0..nin) from the inputs: the per-frequency
// fold thresholds and the station coefficients of the folded interval sum
// (itype 1), or g * w (itype 0). kb and gbuf[] are device buffers of the
// sizes above; d.rs, d.drs, d.geo (itype 1), d.nr, d.nf, d.tau must be set.
int prep_interval_data(const ccfj_fj_args& a, FjDev& d, const InDesc* in, int nin, void* kb,
                       void* const* gbuf, const float* wtr, cudaStream_t s) {
  const bool fp32 = a.precision == CCFJ_PREC_FP32;
  if (a.itype == 1) {
    const dim3 kbb(32, 8);
    if (fp32)
      fj_kbounds_kernel<float><<<div_up(a.nf, 8), kbb, 0, s>>>(a.f, a.c, a.nf, a.nc, d.tau,
                                                               static_cast<float*>(kb));
    else
      fj_kbounds_kernel<double><<<div_up(a.nf, 8), kbb, 0, s>>>(a.f, a.c, a.nf, a.nc,
                                                                (double)d.tau,
                                                                static_cast<double*>(kb));
    count_launch();
    CCFJ_LAUNCH_CHECK("fj_kbounds_kernel");
    d.kb = kb;
  }
  const dim3 pb(32, 8), pg(div_up(a.nr, 8), div_up(a.nf, 32));
  for (int j = 0; j < nin; ++j) {
    void* g = gbuf[j];
    if (a.itype == 1) {
      if (fp32)
        fj_prep_coef_kernel<float><<<pg, pb, 0, s>>>(in[j], a.nr, a.nf, d.rs, d.drs, d.geo,
                                                     static_cast<const float*>(kb),
                                                     static_cast<StationCoef<float>*>(g));
      else
        fj_prep_coef_kernel<double><<<pg, pb, 0, s>>>(in[j], a.nr, a.nf, d.rs, d.drs, d.geo,
                                                      static_cast<const double*>(kb),
                                                      static_cast<StationCoef<double>*>(g));
      count_launch();
      CCFJ_LAUNCH_CHECK("fj_prep_coef_kernel");
    } else {
      if (fp32)
        fj_prep_u_kernel<float><<<pg, pb, 0, s>>>(in[j], a.nr, a.nf, wtr, d.geo,
                                                  static_cast<float*>(g));
      else
        fj_prep_u_kernel<double><<<pg, pb, 0, s>>>(in[j], a.nr, a.nf, wtr, d.geo,
                                                   static_cast<double*>(g));
      count_launch();
      CCFJ_LAUNCH_CHECK("fj_prep_u_kernel");
    }
    d.gb[j] = g;
  }
  return CCFJ_OK;
}

// Device-resident transform: every pointer in `a` is a device pointer.
// cpt > 0 runs that variant (velocities per thread) of the FP32 kernel.
int fj_device(const ccfj_fj_args& a, cudaStream_t s, int cpt_choice, int split_choice) {
  const int nin = nin_of(a.mode);
  Scratch sc(s);
  float* drs = sc.get_n<float>(a.nr + 1);
  float* wtr = sc.get_n<float>(a.nr);
  const bool amortized = a.precision != CCFJ_PREC_FP64_PLAIN;
  float4* geo = amortized ? sc.get_n<float4>(a.nr) : nullptr;
  if (!drs || !wtr || (amortized && !geo)) return CCFJ_ERR_ALLOC;
  fj_prep_geom_kernel<<<div_up(a.nr + 1, 256), 256, 0, s>>>(a.r, a.nr, drs, wtr, geo);
  count_launch();
  CCFJ_LAUNCH_CHECK("fj_prep_geom_kernel");

  FjDev d{};
  d.rs = a.r;
  d.drs = drs;
  d.geo = geo;
  d.f = a.f;
  d.c = a.c;
  d.out = a.out;
  d.nr = a.nr;
  d.nf = a.nf;
  d.nc = a.nc;
  d.tau = a.tau > 0 ? a.tau : (a.precision == CCFJ_PREC_FP32 ? kDefaultTau32 : kDefaultTau64);
  d.i_lo = 0;
  d.i_hi = a.nr;
  d.part = nullptr;
  d.split_len = a.nr;

  InDesc in[2];
  const long long col0 = (long long)a.col_begin * a.fstride * a.u_es;  // first computed column
  for (int j = 0; j < 2; ++j)
    in[j] = InDesc{a.u[j] ? a.u[j] + col0 : nullptr, a.u_ld, (long long)a.u_es * a.fstride, a.perm};
  if (a.hilbert) {
    float* hb = sc.get_n<float>((size_t)a.nr * a.nf);
    if (!hb) return CCFJ_ERR_ALLOC;
    const int st = hilbert_rows(InDesc{a.u[0], a.u_ld, a.u_es, a.perm}, a.u_ncols, a.u_es, a.nr,
                                a.nf, a.fstride, a.col_begin, hb, s, sc);
    if (st != CCFJ_OK) return st;
    in[1] = InDesc{hb, a.nf, 1, nullptr};
  }

  const float* plain[2] = {nullptr, nullptr};
  if (a.precision == CCFJ_PREC_FP64_PLAIN) {
    const dim3 pb(32, 8), pg(div_up(a.nr, 8), div_up(a.nf, 32));
    for (int j = 0; j < nin; ++j) {
      float* g = sc.get_n<float>((size_t)a.nr * a.nf);
      if (!g) return CCFJ_ERR_ALLOC;
      fj_gather_kernel<<<pg, pb, 0, s>>>(in[j], a.nr, a.nf, g);
      count_launch();
      CCFJ_LAUNCH_CHECK("fj_gather_kernel");
      plain[j] = g;
    }
  } else {
    void* kb = nullptr;
    if (a.itype == 1) {
      kb = sc.get(kbounds_bytes(a));
      if (!kb) return CCFJ_ERR_ALLOC;
    }
    void* gbuf[2] = {nullptr, nullptr};
    for (int j = 0; j < nin; ++j) {
      gbuf[j] = sc.get(interval_data_bytes(a));
      if (!gbuf[j]) return CCFJ_ERR_ALLOC;
    }
    const int st = prep_interval_data(a, d, in, nin, kb, gbuf, wtr, s);
    if (st != CCFJ_OK) return st;
  }

  const int cpt = variant_for(a, cpt_choice);
  if (a.precision == CCFJ_PREC_FP32) {
    const int nsplit = split_for(a, cpt, split_choice);
    if (nsplit > 1) {
      d.split_len = (int)div_up(div_up(a.nr, nsplit), kSplitAlign) * kSplitAlign;
      const int n = (int)div_up(a.nr, d.split_len);
      if (n > 1) {
        d.part = sc.get_n<float>((size_t)n * nin_of(a.mode) * a.nc * a.nf);
        if (!d.part) return CCFJ_ERR_ALLOC;
      }
    }
  }
  prof_begin(s);
  switch (a.mode) {
    case CCFJ_MODE_J:
      launch_mode<CCFJ_MODE_J>(a.precision, a.itype, d, plain[0], plain[1], cpt, s);
      break;
    case CCFJ_MODE_Y:
      launch_mode<CCFJ_MODE_Y>(a.precision, a.itype, d, plain[0], plain[1], cpt, s);
      break;
    case CCFJ_MODE_J_MINUS_Y:
      launch_mode<CCFJ_MODE_J_MINUS_Y>(a.precision, a.itype, d, plain[0], plain[1], cpt, s);
      break;
    case CCFJ_MODE_ABS_J:
      launch_mode<CCFJ_MODE_ABS_J>(a.precision, a.itype, d, plain[0], plain[1], cpt, s);
      break;
    default:
      launch_mode<CCFJ_MODE_ABS_H>(a.precision, a.itype, d, plain[0], plain[1], cpt, s);
      break;
  }
  prof_end(s);
  count_launch();
  CCFJ_LAUNCH_CHECK("fj transform kernel");
  if (d.part) {
    const int n = (int)div_up(a.nr, d.split_len);
    const dim3 fg(div_up(a.nf, 32), div_up(a.nc, 8)), fb(32, 8);
    switch (a.mode) {
      case CCFJ_MODE_J:
        fj_split_finish_kernel<CCFJ_MODE_J><<<fg, fb, 0, s>>>(d.part, n, a.f, a.c, a.nc, a.nf, a.out);
        break;
      case CCFJ_MODE_Y:
        fj_split_finish_kernel<CCFJ_MODE_Y><<<fg, fb, 0, s>>>(d.part, n, a.f, a.c, a.nc, a.nf, a.out);
        break;
      case CCFJ_MODE_J_MINUS_Y:
        fj_split_finish_kernel<CCFJ_MODE_J_MINUS_Y><<<fg, fb, 0, s>>>(d.part, n, a.f, a.c, a.nc,
                                                                     a.nf, a.out);
        break;
      case CCFJ_MODE_ABS_J:
        fj_split_finish_kernel<CCFJ_MODE_ABS_J><<<fg, fb, 0, s>>>(d.part, n, a.f, a.c, a.nc, a.nf,
                                                                 a.out);
        break;
      default:
        fj_split_finish_kernel<CCFJ_MODE_ABS_H><<<fg, fb, 0, s>>>(d.part, n, a.f, a.c, a.nc, a.nf,
                                                                 a.out);
        break;
    }
    count_launch();
    CCFJ_LAUNCH_CHECK("fj_split_finish_kernel");
  }

  if (a.normalize) {
    fj_normalize_kernel<<<div_up(a.nf, 32), dim3(32, 8), 0, s>>>(a.out, a.nc, a.nf);
    count_launch();
    CCFJ_LAUNCH_CHECK("fj_normalize_kernel");
  }
  return CCFJ_OK;
}

static int validate(const ccfj_fj_args* a) {
  CCFJ_REQUIRE(a != nullptr, "ccfj_fj_v1: args is NULL");
  CCFJ_REQUIRE(a->struct_size == (int)sizeof(ccfj_fj_args),
               "ccfj_fj_v1: struct_size %d != %d (header mismatch)", a->struct_size,
               (int)sizeof(ccfj_fj_args));
  CCFJ_REQUIRE(a->nr >= 1 && a->nf >= 1 && a->nc >= 1, "ccfj_fj_v1: nr=%d nf=%d nc=%d must be >= 1",
               a->nr, a->nf, a->nc);
  // frequency tiles of 32 and velocity rows of 8 are grid dimensions y
  CCFJ_REQUIRE(a->nf <= 65535 * 32 && a->nc <= 65535 * 8,
               "ccfj_fj_v1: nf=%d (max %d) or nc=%d (max %d) too large for one launch", a->nf,
               65535 * 32, a->nc, 65535 * 8);
  CCFJ_REQUIRE(a->itype == 0 || a->itype == 1, "ccfj_fj_v1: itype must be 0 or 1 (got %d)",
               a->itype);
  CCFJ_REQUIRE(a->mode >= CCFJ_MODE_J && a->mode <= CCFJ_MODE_ABS_H, "ccfj_fj_v1: bad mode %d",
               a->mode);
  CCFJ_REQUIRE(a->precision >= CCFJ_PREC_FP32 && a->precision <= CCFJ_PREC_FP64_PLAIN,
               "ccfj_fj_v1: bad precision %d", a->precision);
  CCFJ_REQUIRE(a->r && a->f && a->c && a->out && a->u[0], "ccfj_fj_v1: NULL array");
  CCFJ_REQUIRE(a->fstride >= 1 && a->u_es >= 1 && a->u_ld >= 1,
               "ccfj_fj_v1: fstride, u_es and u_ld must be >= 1");
  const int nf_total = a->nf_total > 0 ? a->nf_total : a->nf;
  CCFJ_REQUIRE(a->u_ncols >= 1 && (a->u_ncols + a->fstride - 1) / a->fstride == nf_total,
               "ccfj_fj_v1: %d columns with fstride %d give %d frequencies, not %d", a->u_ncols,
               a->fstride, (a->u_ncols + a->fstride - 1) / a->fstride, nf_total);
  CCFJ_REQUIRE(a->col_begin >= 0 && a->col_begin + a->nf <= nf_total,
               "ccfj_fj_v1: frequencies %d..%d outside the %d the rows hold", a->col_begin,
               a->col_begin + a->nf - 1, nf_total);
  CCFJ_REQUIRE(a->u_ld >= (long long)(a->u_ncols - 1) * a->u_es + 1,
               "ccfj_fj_v1: u_ld=%lld too small for %d columns of stride %d", a->u_ld, a->u_ncols,
               a->u_es);
  CCFJ_REQUIRE(a->u_rows >= a->nr, "ccfj_fj_v1: u_rows=%lld < nr=%d", a->u_rows, a->nr);
  if (a->hilbert) {
    CCFJ_REQUIRE(a->mode == CCFJ_MODE_J_MINUS_Y && a->u[1] == nullptr,
                 "ccfj_fj_v1: hilbert=1 needs mode J_MINUS_Y and u[1] == NULL");
  } else {
    CCFJ_REQUIRE(nin_of(a->mode) == 1 || a->u[1], "ccfj_fj_v1: mode %d needs two inputs",
                 a->mode);
  }
  return CCFJ_OK;
}

int fj_validate(const ccfj_fj_args* a) { return validate(a); }

// ------------------------------------------ host memory, in frequency blocks
// Frequency columns are independent (the per-frequency normalisation
// included), so a large host-memory transform without the Hilbert transform
// (which needs whole rows) runs in column blocks. The host gathers block
// p+1's columns into one of two pinned staging buffers while the upload (one
// contiguous DMA) and the transform of block p run on the GPU. Blocks
// alternate between two library-owned streams so that one block's last wave
// overlaps the next block's first; all downloads are issued after the last
// upload (a pageable download would otherwise hold the host until its block
// finished, and the next gather with it). The staging buffers (2 x 64 MiB of
// pinned host memory per device) are allocated on first use and kept.
namespace {
constexpr int kHostMaxDevices = 64;
constexpr size_t kStageBytes = size_t(64) << 20;
constexpr int kMaxHostBlocks = 32;
std::mutex g_host_mu;
struct HostPipe {
  cudaStream_t st[2] = {nullptr, nullptr};
  void* stage[2] = {nullptr, nullptr};
  cudaEvent_t staged[2] = {nullptr, nullptr};  // the upload from stage[k] has finished
  std::mutex use;  // one blocked transform at a time uses the staging buffers
};
HostPipe g_host_pipe[kHostMaxDevices];

int host_pipe(HostPipe** out) {
  int dev = 0;
  CCFJ_CUDA_TRY(cudaGetDevice(&dev));
  CCFJ_REQUIRE(dev >= 0 && dev < kHostMaxDevices, "ccfj_fj_v1: device ordinal %d", dev);
  std::lock_guard<std::mutex> lk(g_host_mu);
  HostPipe& hp = g_host_pipe[dev];
  for (int k = 0; k < 2; ++k) {
    if (!hp.st[k]) CCFJ_CUDA_TRY(cudaStreamCreateWithFlags(&hp.st[k], cudaStreamNonBlocking));
    if (!hp.stage[k]) CCFJ_CUDA_TRY(cudaHostAlloc(&hp.stage[k], kStageBytes, cudaHostAllocDefault));
    if (!hp.staged[k])
      CCFJ_CUDA_TRY(cudaEventCreateWithFlags(&hp.staged[k], cudaEventDisableTiming));
  }
  *out = &hp;
  return CCFJ_OK;
}

// Host threads for gathering one block: up to 8 (half the hardware
// threads), for blocks of at least 1024 rows.
int gather_threads(long long rows) {
  const unsigned hw = std::thread::hardware_concurrency();
  const int n = (int)std::min<unsigned>(8u, hw > 1 ? hw / 2 : 1u);
  return rows >= 1024 ? n : 1;
}

// Blocks worth splitting into: about 40 MB of spectra each (each must fit a
// staging buffer), at least 128 frequencies each.
// First frequency of block p (p = nblk gives nf): equal shares, with
// boundaries on whole warps of 32 frequencies.
static int block_start(int nf, int nblk, int p) {
  if (p <= 0) return 0;
  if (p >= nblk) return nf;
  return (int)(((long long)nf * p / nblk) & ~31ll);
}

int host_block_count(const ccfj_fj_args& a, long long span_floats) {
  if (a.hilbert) return 1;
  const long long bytes = 4 * span_floats;
  int n = (int)std::min<long long>(kMaxHostBlocks, (bytes + (40ll << 20) - 1) / (40ll << 20));
  n = std::min(n, a.nf / 128);
  if (n < 2) return 1;
  // every block (its frequencies' share of the bytes, plus two columns of
  // slack) must fit a staging buffer
  for (int p = 0; p < n; ++p) {
    const long long w = block_start(a.nf, n, p + 1) - block_start(a.nf, n, p);
    if (bytes / a.nf * (w + 2) > (long long)kStageBytes) return 1;
  }
  return n;
}
}  // namespace

static int fj_host_blocks(const ccfj_fj_args& a, cudaStream_t s, int nblk, int nin, bool merged) {
  HostPipe* hp = nullptr;
  int st = host_pipe(&hp);
  if (st != CCFJ_OK) return st;
  // one call at a time per device uses the staging buffers
  std::lock_guard<std::mutex> pipe_lock(hp->use);
  cudaStream_t hs[2] = {hp->st[0], hp->st[1]};
  const int full_cpt = variant_for(a, 0);
  const int full_split = a.precision == CCFJ_PREC_FP32 ? split_for(a, full_cpt, 0) : 1;
  Scratch sc(s);
  float* dr = sc.get_n<float>(a.nr);
  float* df = sc.get_n<float>(a.nf);
  float* dc = sc.get_n<float>(a.nc);
  long long* dp = a.perm ? sc.get_n<long long>(a.nr) : nullptr;
  if (!dr || !df || !dc || (a.perm && !dp)) return CCFJ_ERR_ALLOC;
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dr, a.r, sizeof(float) * a.nr, cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(df, a.f, sizeof(float) * a.nf, cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dc, a.c, sizeof(float) * a.nc, cudaMemcpyHostToDevice, s));
  if (dp)
    CCFJ_CUDA_TRY(cudaMemcpyAsync(dp, a.perm, sizeof(long long) * a.nr, cudaMemcpyHostToDevice, s));
  // The regions one block copies: every input's columns of the block over
  // all rows, as one region when the inputs interleave (Re / Im).
  const int nreg = merged ? 1 : nin;
  const float* reg_base[2] = {a.u[0], a.u[1]};
  long long reg_extra = 0;  // floats between the first and the last input of a merged region
  if (merged && nin == 2) {
    reg_base[0] = std::min(a.u[0], a.u[1]);
    reg_extra = std::max(a.u[0], a.u[1]) - reg_base[0];
  }
  struct Block {
    int b0, b1;
    long long width;  // floats per row of the block's device copy
    float* du[2];
    float* dout;
  };
  // Two device allocations hold every block's upload and output (one
  // scratch entry each, whatever the number of blocks).
  Block blk[kMaxHostBlocks];
  size_t u_total = 0;
  for (int p = 0; p < nblk; ++p) {
    Block& B = blk[p];
    B.b0 = block_start(a.nf, nblk, p);
    B.b1 = block_start(a.nf, nblk, p + 1);
    const long long c_lo = (long long)(a.col_begin + B.b0) * a.fstride * a.u_es;
    const long long c_hi = (long long)(a.col_begin + B.b1 - 1) * a.fstride * a.u_es;
    B.width = c_hi - c_lo + 1 + reg_extra;
    const size_t floats = (size_t)nreg * B.width * a.u_rows;
    if (floats * sizeof(float) > kStageBytes)
      return set_error(CCFJ_ERR_UNSUPPORTED, "ccfj_fj_v1: host block exceeds the staging buffer");
    u_total += (floats + 63) & ~size_t(63);  // blocks start on 256-byte boundaries
  }
  float* du_all = sc.get_n<float>(u_total);
  float* dout_all = sc.get_n<float>((size_t)a.nc * a.nf);
  if (!du_all || !dout_all) return CCFJ_ERR_ALLOC;
  size_t u_off = 0;
  for (int p = 0; p < nblk; ++p) {
    Block& B = blk[p];
    const size_t floats = (size_t)nreg * B.width * a.u_rows;
    // the block's regions are contiguous on the device (one DMA)
    B.du[0] = du_all + u_off;
    B.du[1] = B.du[0] + (size_t)B.width * a.u_rows;
    u_off += (floats + 63) & ~size_t(63);
    B.dout = dout_all + (size_t)a.nc * B.b0;  // [nc][b1 - b0]
  }
  cudaEvent_t ready = nullptr, done[2] = {nullptr, nullptr};
  CCFJ_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  for (int k = 0; k < 2; ++k) CCFJ_CUDA_TRY(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming));
  auto destroy = [&]() {
    cudaEventDestroy(ready);
    for (int k = 0; k < 2; ++k) cudaEventDestroy(done[k]);
  };
  auto fail = [&](int status) {
    // leave no work of this call running on the library's streams
    for (int k = 0; k < 2; ++k) cudaStreamSynchronize(hs[k]);
    destroy();
    return status;
  };
  if (cudaEventRecord(ready, s) != cudaSuccess)
    return fail(set_error(CCFJ_ERR_CUDA, "ccfj_fj_v1: cudaEventRecord failed"));
  for (int k = 0; k < 2; ++k)
    if (cudaStreamWaitEvent(hs[k], ready, 0) != cudaSuccess)
      return fail(set_error(CCFJ_ERR_CUDA, "ccfj_fj_v1: cudaStreamWaitEvent failed"));
  for (int p = 0; p < nblk; ++p) {
    Block& B = blk[p];
    cudaStream_t cs = hs[p & 1];
    const long long c_lo = (long long)(a.col_begin + B.b0) * a.fstride * a.u_es;
    // gather the block's columns into staging buffer p % 2 once its previous
    // upload has finished, then upload it in one piece
    const int k = p & 1;
    cudaError_t e = cudaEventSynchronize(hp->staged[k]);
    if (e != cudaSuccess)
      return fail(set_error(CCFJ_ERR_CUDA, "ccfj_fj_v1: staging wait failed: %s",
                            cudaGetErrorString(e)));
    float* stg = static_cast<float*>(hp->stage[k]);
    const size_t row_bytes = B.width * sizeof(float);
    // the gather of the first block is on the critical path: split the rows
    // over a few host threads
    auto gather = [&](long long r0, long long r1) {
      for (int g = 0; g < nreg; ++g) {
        const float* src = reg_base[g] + c_lo;
        float* dst = stg + (size_t)g * B.width * a.u_rows;
        for (long long row = r0; row < r1; ++row)
          memcpy(dst + row * B.width, src + row * a.u_ld, row_bytes);
      }
    };
    const int nthr = gather_threads(a.u_rows);
    if (nthr <= 1) {
      gather(0, a.u_rows);
    } else {
      // row ranges [start[t], start[t+1]); a thread that cannot be created
      // leaves its range to this one (no exception crosses the C ABI)
      std::vector<std::thread> pool;
      std::vector<long long> mine;
      for (int t = 1; t < nthr; ++t) {
        const long long r0 = a.u_rows * t / nthr, r1 = a.u_rows * (t + 1) / nthr;
        try {
          pool.emplace_back(gather, r0, r1);
        } catch (...) {
          mine.push_back(r0);
          mine.push_back(r1);
        }
      }
      gather(0, a.u_rows / nthr);
      for (size_t q = 0; q < mine.size(); q += 2) gather(mine[q], mine[q + 1]);
      for (auto& th : pool) th.join();
    }
    e = cudaMemcpyAsync(B.du[0], stg, (size_t)nreg * row_bytes * a.u_rows, cudaMemcpyHostToDevice,
                        cs);
    if (e == cudaSuccess) e = cudaEventRecord(hp->staged[k], cs);
    if (e != cudaSuccess)
      return fail(set_error(CCFJ_ERR_CUDA, "ccfj_fj_v1: block upload failed: %s",
                            cudaGetErrorString(e)));
    ccfj_fj_args d = a;
    d.device_ptrs = 1;
    for (int j = 0; j < nin; ++j)
      d.u[j] = merged ? B.du[0] + (a.u[j] - reg_base[0]) : B.du[j];
    d.u_ld = B.width;
    d.col_begin = 0;
    d.nf = B.b1 - B.b0;
    d.nf_total = d.nf;
    d.u_ncols = (d.nf - 1) * a.fstride + 1;
    d.r = dr;
    d.f = df + B.b0;
    d.c = dc;
    d.perm = dp;
    d.out = B.dout;
    // every block runs the whole problem's tile choice, so the blocks give
    // the device path's result bit for bit
    st = fj_device(d, cs, full_cpt, full_split);
    if (st != CCFJ_OK) return fail(st);
  }
  for (int p = 0; p < nblk; ++p) {
    const Block& B = blk[p];
    const int w = B.b1 - B.b0;
    const cudaError_t e = cudaMemcpy2DAsync(a.out + B.b0, a.nf * sizeof(float), B.dout,
                                            w * sizeof(float), w * sizeof(float), a.nc,
                                            cudaMemcpyDeviceToHost, hs[p & 1]);
    if (e != cudaSuccess)
      return fail(set_error(CCFJ_ERR_CUDA, "ccfj_fj_v1: block download failed: %s",
                            cudaGetErrorString(e)));
  }
  // the scratch is freed on s: s waits for both streams
  for (int k = 0; k < 2; ++k) {
    if (cudaEventRecord(done[k], hs[k]) != cudaSuccess || cudaStreamWaitEvent(s, done[k], 0) != cudaSuccess)
      return fail(set_error(CCFJ_ERR_CUDA, "ccfj_fj_v1: stream join failed"));
  }
  const cudaError_t e = cudaStreamSynchronize(s);
  destroy();
  if (e != cudaSuccess)
    return set_error(CCFJ_ERR_CUDA, "ccfj_fj_v1: %s", cudaGetErrorString(e));
  return CCFJ_OK;
}

// Host-memory variant: copies the inputs in, runs the device path, copies
// out back and waits (in frequency blocks when that pays, see above).
static int fj_host(const ccfj_fj_args& a, cudaStream_t s) {
  const int nin = a.hilbert ? 1 : nin_of(a.mode);
  const long long rows = a.u_rows;
  if (a.perm)
    for (int i = 0; i < a.nr; ++i)
      CCFJ_REQUIRE(a.perm[i] >= 0 && a.perm[i] < rows, "ccfj_fj_v1: perm[%d]=%lld out of [0,%lld)",
                   i, a.perm[i], rows);
  // Input span(s): the two inputs may be the real and imaginary parts of
  // one complex array; copy the union once.
  const long long span = (rows - 1) * a.u_ld + (long long)(a.u_ncols - 1) * a.u_es + 1;
  const float* lo = a.u[0];
  const float* hi = a.u[0] + span;
  bool merged = nin == 1;
  if (nin == 2) {
    const float* lo1 = a.u[1];
    const float* hi1 = a.u[1] + span;
    if (lo1 < hi && lo < hi1) {
      lo = std::min(lo, lo1);
      hi = std::max(hi, hi1);
      merged = true;
    }
  }
  const int nblk = host_block_count(a, merged ? (long long)(hi - lo) : nin * span);
  if (nblk > 1) return fj_host_blocks(a, s, nblk, nin, merged);
  Scratch sc(s);
  ccfj_fj_args d = a;
  d.device_ptrs = 1;
  float* dr = sc.get_n<float>(a.nr);
  float* df = sc.get_n<float>(a.nf);
  float* dc = sc.get_n<float>(a.nc);
  float* dout = sc.get_n<float>((size_t)a.nc * a.nf);
  if (!dr || !df || !dc || !dout) return CCFJ_ERR_ALLOC;
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dr, a.r, sizeof(float) * a.nr, cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(df, a.f, sizeof(float) * a.nf, cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dc, a.c, sizeof(float) * a.nc, cudaMemcpyHostToDevice, s));
  if (merged) {
    float* du = sc.get_n<float>(hi - lo);
    if (!du) return CCFJ_ERR_ALLOC;
    const int cst = copy_from_host(du, lo, sizeof(float) * (hi - lo), s);
    if (cst != CCFJ_OK) return cst;
    for (int j = 0; j < nin; ++j) d.u[j] = du + (a.u[j] - lo);
  } else {
    for (int j = 0; j < nin; ++j) {
      float* du = sc.get_n<float>(span);
      if (!du) return CCFJ_ERR_ALLOC;
      const int cst = copy_from_host(du, a.u[j], sizeof(float) * span, s);
      if (cst != CCFJ_OK) return cst;
      d.u[j] = du;
    }
  }
  if (a.perm) {
    long long* dp = sc.get_n<long long>(a.nr);
    if (!dp) return CCFJ_ERR_ALLOC;
    CCFJ_CUDA_TRY(cudaMemcpyAsync(dp, a.perm, sizeof(long long) * a.nr, cudaMemcpyHostToDevice, s));
    d.perm = dp;
  }
  d.r = dr;
  d.f = df;
  d.c = dc;
  d.out = dout;
  int st = fj_device(d, s);
  if (st != CCFJ_OK) return st;
  return copy_to_host(a.out, dout, sizeof(float) * a.nc * a.nf, 0, s);
}

int fj_entry(const ccfj_fj_args* a, cudaStream_t s) {
  clear_error();
  int st = validate(a);
  if (st != CCFJ_OK) return st;
  if (a->device_ptrs) return fj_device(*a, s);
  return fj_host(*a, s);
}

static int compat(float* u_f, float* r, float* f, float* out, float* c, int nc, int nr, int nf,
                  int type, int mode) {
  ccfj_fj_args a{};
  a.struct_size = sizeof(a);
  a.nr = nr;
  a.nf = nf;
  a.nc = nc;
  a.itype = type;
  a.mode = mode;
  a.precision = CCFJ_PREC_FP32;
  a.normalize = 0;
  a.device_ptrs = 0;
  a.u[0] = u_f;
  a.u_ld = nf;
  a.u_es = 1;
  a.u_ncols = nf;
  a.fstride = 1;
  a.u_rows = nr;
  a.r = r;
  a.f = f;
  a.c = c;
  a.out = out;
  return fj_entry(&a, 0);
}

}  // namespace ccfj

CCFJ_API int ccfj_fj_v1(const ccfj_fj_args* args, void* stream) {
  return ccfj::fj_entry(args, (cudaStream_t)stream);
}

CCFJ_API int ccfj_set_fj_variant(int cpt) {
  if (cpt != 0 && cpt != 1 && cpt != 2 && cpt != 4)
    return ccfj::set_error(CCFJ_ERR_INVALID, "ccfj_set_fj_variant: cpt must be 0, 1, 2 or 4");
  ccfj::g_force_cpt.store(cpt, std::memory_order_relaxed);
  return CCFJ_OK;
}

CCFJ_API int ccfj_autotune_fj_v1(const ccfj_fj_args* args, void* stream, int* best_cpt,
                                 float* best_ms) {
  ccfj::clear_error();
  int st = ccfj::validate(args);
  if (st != CCFJ_OK) return st;
  if (!args->device_ptrs)
    return ccfj::set_error(CCFJ_ERR_INVALID, "ccfj_autotune_fj_v1: needs device pointers");
  cudaStream_t s = (cudaStream_t)stream;
  // candidates: 1, 2 or 4 velocities per thread, times 1 to 8 station
  // ranges where the unsplit grid leaves resident slots idle
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long slots = (long long)sms * CCFJ_FJ_MIN_BLOCKS;
  int best = 2, best_split = 1;
  float best_t = 1e30f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return ccfj::set_error(CCFJ_ERR_CUDA, "ccfj_autotune_fj_v1: cudaEventCreate failed: %s",
                           cudaGetErrorString(cudaGetLastError()));
  }
  const int cands[3] = {1, 2, 4};
  const int splits[6] = {1, 2, 3, 4, 6, 8};
  for (int c : cands) {
    const long long ctas = (long long)ccfj::div_up(args->nc, 8 * c) * ccfj::div_up(args->nf, 32);
    for (int n : splits) {
      if (n > 1 && (n * ctas > 2 * slots || args->nr < 2 * 32 * n)) continue;
      float t = 1e30f;
      for (int rep = 0; rep < 3 && st == CCFJ_OK; ++rep) {
        cudaEventRecord(e0, s);
        st = ccfj::fj_device(*args, s, c, n);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = CCFJ_ERR_CUDA;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) t = std::min(t, ms);  // the first run is a warm-up
      }
      if (st != CCFJ_OK) break;
      if (t < best_t) {
        best_t = t;
        best = c;
        best_split = n;
      }
    }
    if (st != CCFJ_OK) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != CCFJ_OK) return st;
  st = ccfj::tune_record("fj", ccfj::tune_key(*args), best + 8 * best_split, best_t);
  if (best_cpt) *best_cpt = best;
  if (best_ms) *best_ms = best_t;
  return st;
}

CCFJ_API int ccfj_set_fj_split(int nsplit) {
  if (nsplit < 0 || nsplit > 64)
    return ccfj::set_error(CCFJ_ERR_INVALID, "ccfj_set_fj_split: nsplit must be 0..64");
  ccfj::g_force_split.store(nsplit, std::memory_order_relaxed);
  return CCFJ_OK;
}

CCFJ_API int ccfj_tuned_choice_fj(const ccfj_fj_args* args, int* cpt, int* nsplit) {
  ccfj::clear_error();
  int st = ccfj::validate(args);
  if (st != CCFJ_OK) return st;
  const int c = ccfj::variant_for(*args, 0);
  if (cpt) *cpt = c;
  if (nsplit) *nsplit = args->precision == CCFJ_PREC_FP32 ? ccfj::split_for(*args, c, 0) : 1;
  return CCFJ_OK;
}

CCFJ_API int FJ(float* u_f, float* r, float* f, float* out, float* c, int nc, int nr, int nf,
                int type) {
  return ccfj::compat(u_f, r, f, out, c, nc, nr, nf, type, CCFJ_MODE_J);
}
CCFJ_API int FHr(float* u_f, float* r, float* f, float* out, float* c, int nc, int nr, int nf,
                 int type) {
  return ccfj::compat(u_f, r, f, out, c, nc, nr, nf, type, CCFJ_MODE_J);
}
CCFJ_API int FHi(float* u_f, float* r, float* f, float* out, float* c, int nc, int nr, int nf,
                 int type) {
  return ccfj::compat(u_f, r, f, out, c, nc, nr, nf, type, CCFJ_MODE_Y);
}
CCFJ_API int FH(float* u_f, float* r, float* f, float* out, float* c, int nc, int nr, int nf,
                int type, int /*nThread*/) {
  return ccfj::compat(u_f, r, f, out, c, nc, nr, nf, type, CCFJ_MODE_Y);
}

// --------------------------------------------------- allocation-free entry
// ccfj_fj_noalloc_v1 runs the same FP32 transform as ccfj_fj_v1 with device
// pointers, but takes its scratch (pair geometry and the per-interval
// spectrum data) from one fixed array that lives in the library's device
// image instead of allocating it. It exists for callers that cannot
// allocate device memory while they run: a host that has handed all free
// device memory to its own pool allocator (so cudaMalloc/cudaMallocAsync
// would fail or fragment it), code that must not incur the device-wide
// synchronisation that cudaMalloc/cudaFree may cause, or code running
// where only kernel launches on the caller's stream are allowed.
namespace ccfj {

// 16 MiB, held by every GPU that loads this library until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_dev_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device. In host code
// the array's name is only a host-side stand-in, so the address must come
// from cudaGetSymbolAddress, once per device, with that device current.
int noalloc_scratch_address(void** out) {
  int dev = 0;
  CCFJ_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return set_error(CCFJ_ERR_UNSUPPORTED, "ccfj_fj_noalloc_v1: device ordinal %d >= %d", dev,
                     kNoAllocMaxDevices);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_dev_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return set_error(CCFJ_ERR_CUDA, "ccfj_fj_noalloc_v1: cudaGetSymbolAddress failed: %s",
                       cudaGetErrorString(e));
    g_noalloc_dev_ptr[dev] = p;
  }
  *out = g_noalloc_dev_ptr[dev];
  return CCFJ_OK;
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
}  // namespace

static int fj_noalloc(const ccfj_fj_args& a, cudaStream_t s) {
  CCFJ_REQUIRE(a.device_ptrs == 1, "ccfj_fj_noalloc_v1: needs device pointers (device_ptrs = 1)");
  if (a.precision != CCFJ_PREC_FP32)
    return set_error(CCFJ_ERR_UNSUPPORTED, "ccfj_fj_noalloc_v1: only precision CCFJ_PREC_FP32");
  if (a.hilbert)
    return set_error(CCFJ_ERR_UNSUPPORTED,
                     "ccfj_fj_noalloc_v1: hilbert = 1 is not supported; pass the transformed "
                     "spectrum as u[1]");
  const int nin = nin_of(a.mode);
  const size_t geom = round256(sizeof(float) * ((size_t)a.nr + 1));
  const size_t gbytes = round256(geometry_bytes(a));
  const size_t kbytes = round256(kbounds_bytes(a));
  const size_t per_input = round256(interval_data_bytes(a));
  const size_t fixed = 2 * geom + gbytes + kbytes;
  const size_t need = fixed + nin * per_input;
  if (need > kNoAllocScratchBytes)
    return set_error(CCFJ_ERR_INVALID,
                     "ccfj_fj_noalloc_v1: nr=%d nf=%d (%d input%s, itype %d) needs %zu bytes of "
                     "scratch; the fixed scratch holds %zu bytes (nr*nf up to about %zu for one "
                     "itype-1 input)",
                     a.nr, a.nf, nin, nin > 1 ? "s" : "", a.itype, need, kNoAllocScratchBytes,
                     (kNoAllocScratchBytes - fixed) / 16);
  void* base = nullptr;
  int st = noalloc_scratch_address(&base);
  if (st != CCFJ_OK) return st;
  unsigned char* p = static_cast<unsigned char*>(base);
  // Every scratch byte read below is first written by the preparation
  // kernels of this call, so nothing needs clearing between calls.
  float* drs = reinterpret_cast<float*>(p);
  float* wtr = reinterpret_cast<float*>(p + geom);
  float4* geo = reinterpret_cast<float4*>(p + 2 * geom);
  fj_prep_geom_kernel<<<div_up(a.nr + 1, 256), 256, 0, s>>>(a.r, a.nr, drs, wtr, geo);
  count_launch();
  CCFJ_LAUNCH_CHECK("fj_prep_geom_kernel");

  FjDev d{};
  d.rs = a.r;
  d.drs = drs;
  d.geo = geo;
  d.f = a.f;
  d.c = a.c;
  d.out = a.out;
  d.nr = a.nr;
  d.nf = a.nf;
  d.nc = a.nc;
  d.tau = a.tau > 0 ? a.tau : kDefaultTau32;
  d.i_lo = 0;
  d.i_hi = a.nr;
  d.part = nullptr;
  d.split_len = a.nr;
  InDesc in[2];
  void* gbuf[2] = {nullptr, nullptr};
  for (int j = 0; j < nin; ++j) {
    in[j] = InDesc{a.u[j] + (long long)a.col_begin * a.fstride * a.u_es, a.u_ld,
                   (long long)a.u_es * a.fstride, a.perm};
    gbuf[j] = p + fixed + j * per_input;
  }
  st = prep_interval_data(a, d, in, nin, a.itype == 1 ? p + 2 * geom + gbytes : nullptr, gbuf,
                          wtr, s);
  if (st != CCFJ_OK) return st;
  const int cpt = variant_for(a, 0);
  switch (a.mode) {
    case CCFJ_MODE_J:
      launch_mode<CCFJ_MODE_J>(a.precision, a.itype, d, nullptr, nullptr, cpt, s);
      break;
    case CCFJ_MODE_Y:
      launch_mode<CCFJ_MODE_Y>(a.precision, a.itype, d, nullptr, nullptr, cpt, s);
      break;
    case CCFJ_MODE_J_MINUS_Y:
      launch_mode<CCFJ_MODE_J_MINUS_Y>(a.precision, a.itype, d, nullptr, nullptr, cpt, s);
      break;
    case CCFJ_MODE_ABS_J:
      launch_mode<CCFJ_MODE_ABS_J>(a.precision, a.itype, d, nullptr, nullptr, cpt, s);
      break;
    default:
      launch_mode<CCFJ_MODE_ABS_H>(a.precision, a.itype, d, nullptr, nullptr, cpt, s);
      break;
  }
  count_launch();
  CCFJ_LAUNCH_CHECK("fj transform kernel");
  if (a.normalize) {
    fj_normalize_kernel<<<div_up(a.nf, 32), dim3(32, 8), 0, s>>>(a.out, a.nc, a.nf);
    count_launch();
    CCFJ_LAUNCH_CHECK("fj_normalize_kernel");
  }
  return CCFJ_OK;
}

}  // namespace ccfj

CCFJ_API int ccfj_fj_noalloc_v1(const ccfj_fj_args* args, void* stream) {
  ccfj::clear_error();
  const int st = ccfj::validate(args);
  if (st != CCFJ_OK) return st;
  return ccfj::fj_noalloc(*args, (cudaStream_t)stream);
}
