// Ambient-noise cross-correlation on the device: the reference's
// CrossCorrelation (src/CrossCorr.cpp:33-159), which produces the
// cross-spectra that fj_noise takes.
//
// Three kernels per call:
//   xc_spectra_kernel   one CTA per kept (shift, station) window: the
//                       window's samples (one-bit on load) as M = F/2
//                       complex points in shared memory, self-sorting
//                       Stockham passes of radix 8/4/2/3/5 in place, then
//                       the real-FFT split at bins j*fstride, whitening, and
//                       a store to X[k][i][j] (complex FP32, frequency
//                       fastest, rows padded to 32);
//   xc_spectra_direct_kernel   the same bins by a direct transform (FP64
//                       accumulation) for windows the shared-memory FFT
//                       does not take (odd, longer than 16384 samples, or
//                       a prime factor above 5 in F/2);
//   xc_gram_kernel      per 16 x 16 station tile and 32 frequencies, the
//                       sums over shifts of conj(X_a) X_b, staged 4 shifts
//                       at a time in shared memory; windows a station does
//                       not keep are zero in X, so the sums need no mask, and
//                       each pair's count is the overlap of two shift
//                       intervals. The epilogue divides and stores every
//                       pair of the caller's list that falls in the tile.
// The arithmetic lives in cc_core.cuh and the planning in cc_plan.h, which
// the tests also run on the host.
#include <algorithm>
#include <string>
#include <vector>

#include "cc_core.cuh"
#include "cc_plan.h"
#include "ccfj_core.cuh"
#include "fj_frontend.cuh"

namespace ccfj {
namespace xc {

// exp(-2 pi i u / n) for u < count, from FP64 sincospi
__global__ void xc_twiddle_kernel(int n, int count, Cpx* __restrict__ out) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= count) return;
  double s, c;
  sincospi(-2.0 * (double)u / (double)n, &s, &c);
  out[u] = cpx((float)c, (float)s);
}

struct SpecJob {
  const float* data;      // [nsta][npts]
  long long npts;
  long long steplen;
  int F, M;
  int npass_r[5];         // passes of radix 8, 4, 2, 3, 5, in that order
  const Cpx* tw;          // [M] exp(-2 pi i u/M) (Stockham) or [F] (direct)
  const Cpx* twh;         // [M + 1] exp(-i pi k/M) (Stockham)
  const Window* windows;  // [gridDim.x]
  int nf, fstride, whiten, onebit;
  int nsta, ldj;
  Cpx* X;                 // [nshifts][nsta][ldj]
};

// One in-place Stockham pass over s[0 .. M): every thread loads all of its
// butterflies' inputs, then (after the barrier) twiddles, transforms and
// stores them.
template <int R>
__device__ __forceinline__ void spec_pass(Cpx* s, int M, int Ns, const Cpx* tw) {
  constexpr int B = (kMaxM + R * kFftThreads - 1) / (R * kFftThreads);
  Cpx v[B][R];
  const int nb = M / R;
#pragma unroll
  for (int b = 0; b < B; ++b) {
    const int t = threadIdx.x + b * kFftThreads;
    if (t < nb) bf_load<R>(s, M, t, v[b]);
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < B; ++b) {
    const int t = threadIdx.x + b * kFftThreads;
    if (t < nb) bf_finish<R>(s, M, Ns, tw, t, v[b]);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kFftThreads, 2) xc_spectra_kernel(SpecJob j) {
  extern __shared__ Cpx s[];  // [M]
  const Window w = j.windows[blockIdx.x];
  // a kept window lies inside the record: k*steplen + F <= npts
  const float* x = j.data + (long long)w.i * j.npts + (long long)w.k * j.steplen;
  for (int m = threadIdx.x; m < j.M; m += kFftThreads) {
    float a = x[2 * m], b = x[2 * m + 1];
    if (j.onebit) {
      a = onebit(a);
      b = onebit(b);
    }
    s[m] = cpx(a, b);
  }
  __syncthreads();
  // the plan's passes in its order: 8s, a 4 or a 2, 3s, 5s (one loop per
  // radix keeps each radix's registers apart)
  int Ns = 1;
  for (int p = 0; p < j.npass_r[0]; ++p, Ns *= 8) spec_pass<8>(s, j.M, Ns, j.tw);
  for (int p = 0; p < j.npass_r[1]; ++p, Ns *= 4) spec_pass<4>(s, j.M, Ns, j.tw);
  for (int p = 0; p < j.npass_r[2]; ++p, Ns *= 2) spec_pass<2>(s, j.M, Ns, j.tw);
  for (int p = 0; p < j.npass_r[3]; ++p, Ns *= 3) spec_pass<3>(s, j.M, Ns, j.tw);
  for (int p = 0; p < j.npass_r[4]; ++p, Ns *= 5) spec_pass<5>(s, j.M, Ns, j.tw);
  Cpx* out = j.X + ((long long)w.k * j.nsta + w.i) * j.ldj;
  for (int q = threadIdx.x; q < j.nf; q += kFftThreads) {
    const int k = q * j.fstride;  // <= M (checked by the plan)
    Cpx v = real_bin(s, j.M, k, j.twh[k]);
    if (j.whiten) v = whiten(v);
    out[q] = v;
  }
}

constexpr int kDirectThreads = 128;

__global__ void __launch_bounds__(kDirectThreads) xc_spectra_direct_kernel(SpecJob j) {
  const Window w = j.windows[blockIdx.x];
  const int q = blockIdx.y * kDirectThreads + threadIdx.x;
  if (q >= j.nf) return;
  const float* x = j.data + (long long)w.i * j.npts + (long long)w.k * j.steplen;
  const long long k = (long long)q * j.fstride;  // <= F/2 < F
  double re = 0.0, im = 0.0;
  long long ph = 0;  // k*n mod F
  for (int n = 0; n < j.F; ++n) {
    float v = x[n];
    if (j.onebit) v = onebit(v);
    const Cpx t = j.tw[ph];
    re += (double)v * (double)t.re;
    im += (double)v * (double)t.im;
    ph += k;
    if (ph >= j.F) ph -= j.F;
  }
  Cpx v = cpx((float)re, (float)im);
  if (j.whiten) v = whiten(v);
  j.X[((long long)w.k * j.nsta + w.i) * j.ldj + q] = v;
}

struct GramJob {
  const Cpx* X;
  int nsta, ldj, nf;
  const Tile* tiles;
  const int* lo;
  const int* hi;
  const int* pmap;   // [nsta * nsta]
  const int* pnext;  // [npairs]
  float* out_re;
  float* out_im;
  long long out_ld;  // floats between pairs
  int out_es;        // floats between bins
  int accumulate;
};

__global__ void __launch_bounds__(kGramThreads) xc_gram_kernel(GramJob g) {
  __shared__ Cpx xs[kShiftChunk][2][kTile][kLanes];  // 32 KiB
  const Tile t = g.tiles[blockIdx.x];
  const int j0 = blockIdx.y * kLanes;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  Cpx acc[kRowsPerWarp][kTile];
#pragma unroll
  for (int ra = 0; ra < kRowsPerWarp; ++ra)
#pragma unroll
    for (int b = 0; b < kTile; ++b) acc[ra][b] = cpx(0.f, 0.f);

  for (int kc = t.k0; kc <= t.k1; kc += kShiftChunk) {
    __syncthreads();
    for (int e = threadIdx.x; e < kShiftChunk * 2 * kTile * kLanes; e += kGramThreads) {
      const int l = e % kLanes;
      const int row = (e / kLanes) % kTile;
      const int side = (e / (kLanes * kTile)) % 2;
      const int kk = e / (2 * kTile * kLanes);
      const int k = kc + kk;
      const int st = (side ? t.b0 : t.a0) + row;
      Cpx v = cpx(0.f, 0.f);
      if (k <= t.k1 && st < g.nsta) v = g.X[((long long)k * g.nsta + st) * g.ldj + j0 + l];
      xs[kk][side][row][l] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kShiftChunk; ++kk)
      gram_step(&xs[kk][0][0][0], &xs[kk][1][0][0], warp, lane, acc);
  }

  const int j = j0 + lane;
  if (j >= g.nf) return;
#pragma unroll
  for (int ra = 0; ra < kRowsPerWarp; ++ra) {
    const int a = t.a0 + warp * kRowsPerWarp + ra;
    if (a >= g.nsta) continue;
#pragma unroll
    for (int b = 0; b < kTile; ++b) {
      const int bb = t.b0 + b;
      if (bb >= g.nsta) continue;
      int p = g.pmap[(long long)a * g.nsta + bb];
      if (p < 0) continue;
      const int cnt = pair_count(g.lo[a], g.hi[a], g.lo[bb], g.hi[bb]);
      if (cnt == 0) continue;
      for (; p >= 0; p = g.pnext[p]) {
        float* re = g.out_re + (long long)p * g.out_ld + (long long)j * g.out_es;
        float* im = g.out_im + (long long)p * g.out_ld + (long long)j * g.out_es;
        const Cpx init = g.accumulate ? cpx(*re, *im) : cpx(0.f, 0.f);
        const Cpx v = pair_value(init, acc[ra][b], cnt);
        *re = v.re;
        *im = v.im;
      }
    }
  }
}

template <typename T>
static T* upload(Scratch& sc, const std::vector<T>& v, cudaStream_t s, int* status) {
  T* d = sc.get_n<T>(v.empty() ? 1 : v.size());
  if (!d) {
    *status = CCFJ_ERR_ALLOC;
    return nullptr;
  }
  if (!v.empty()) {
    cudaError_t e = cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      *status = set_error(CCFJ_ERR_CUDA, "cudaMemcpyAsync (plan upload): %s", cudaGetErrorString(e));
      return nullptr;
    }
  }
  return d;
}

static int twiddles(Cpx* out, int n, int count, cudaStream_t s) {
  xc_twiddle_kernel<<<div_up(count, 256), 256, 0, s>>>(n, count, out);
  count_launch();
  CCFJ_LAUNCH_CHECK("xc_twiddle_kernel");
  return CCFJ_OK;
}

static int run(const ccfj_cc_args& a, cudaStream_t s) {
  CCFJ_REQUIRE(a.struct_size == (int)sizeof(ccfj_cc_args),
               "ccfj_cc_v1: struct_size=%d, expected %d", a.struct_size, (int)sizeof(ccfj_cc_args));
  CCFJ_REQUIRE(a.data != nullptr, "ccfj_cc_v1: data is NULL");
  Plan p;
  std::string err;
  const int pst = make_plan(a, &p, &err);
  if (pst != CCFJ_OK) return set_error(pst, "ccfj_cc_v1: %s", err.c_str());
  const long long nout = (long long)a.npairs * a.nf;
  CCFJ_REQUIRE(nout == 0 || (a.out_re && (a.out_layout == 1 || a.out_im)),
               "ccfj_cc_v1: output pointer is NULL");
  CCFJ_REQUIRE(a.nf <= 65535LL * kLanes, "ccfj_cc_v1: nf=%d too large", a.nf);
  CCFJ_REQUIRE(p.windows.size() <= (size_t)0x7fffffff, "ccfj_cc_v1: too many windows");
  const long long nrec = (long long)a.nsta * a.npts;
  if (!a.device_ptrs && a.onebit)  // the reference rewrites the caller's samples
    for (long long n = 0; n < nrec; ++n) a.data[n] = onebit(a.data[n]);
  if (nout == 0) return CCFJ_OK;  // no pairs or no bins: nothing for the device

  Scratch sc(s);
  int status = CCFJ_OK;
  const float* d_data = a.data;
  if (!a.device_ptrs) {
    float* d = sc.get_n<float>(nrec);
    if (!d) return CCFJ_ERR_ALLOC;
    const int cst = copy_from_host(d, a.data, nrec * sizeof(float), s);
    if (cst != CCFJ_OK) return cst;
    d_data = d;
  }
  // outputs: planes (re, im) [npairs][nf] or interleaved complex [npairs][nf]
  const size_t plane = (size_t)nout * sizeof(float);
  float* d_re = a.out_re;
  float* d_im = a.out_layout == 1 ? (a.out_re ? a.out_re + 1 : nullptr) : a.out_im;
  if (!a.device_ptrs && nout > 0) {
    if (a.out_layout == 1) {
      d_re = sc.get_n<float>(2 * nout);
      if (!d_re) return CCFJ_ERR_ALLOC;
      d_im = d_re + 1;
    } else {
      d_re = sc.get_n<float>(nout);
      d_im = sc.get_n<float>(nout);
      if (!d_re || !d_im) return CCFJ_ERR_ALLOC;
    }
  }
  if (nout > 0) {
    if (a.accumulate && !a.device_ptrs) {
      if (a.out_layout == 1) {
        CCFJ_CUDA_TRY(cudaMemcpyAsync(d_re, a.out_re, 2 * plane, cudaMemcpyHostToDevice, s));
      } else {
        CCFJ_CUDA_TRY(cudaMemcpyAsync(d_re, a.out_re, plane, cudaMemcpyHostToDevice, s));
        CCFJ_CUDA_TRY(cudaMemcpyAsync(d_im, a.out_im, plane, cudaMemcpyHostToDevice, s));
      }
    } else if (!a.accumulate) {
      if (a.out_layout == 1) {
        CCFJ_CUDA_TRY(cudaMemsetAsync(d_re, 0, 2 * plane, s));
      } else {
        CCFJ_CUDA_TRY(cudaMemsetAsync(d_re, 0, plane, s));
        CCFJ_CUDA_TRY(cudaMemsetAsync(d_im, 0, plane, s));
      }
    }
  }

  if (nout > 0 && !p.tiles.empty()) {
    // window spectra
    const size_t xcount = (size_t)p.nshifts * a.nsta * p.ldj;
    Cpx* X = sc.get_n<Cpx>(xcount);
    if (!X) return CCFJ_ERR_ALLOC;
    CCFJ_CUDA_TRY(cudaMemsetAsync(X, 0, xcount * sizeof(Cpx), s));
    const Window* d_win = upload(sc, p.windows, s, &status);
    if (!d_win) return status;
    SpecJob j = {};
    j.data = d_data;
    j.npts = a.npts;
    j.steplen = a.steplen;
    j.F = p.F;
    j.M = p.M;
    for (int i = 0; i < p.npass; ++i) {
      const int r = p.radix[i];
      ++j.npass_r[r == 8 ? 0 : r == 4 ? 1 : r == 2 ? 2 : r == 3 ? 3 : 4];
    }
    j.windows = d_win;
    j.nf = a.nf;
    j.fstride = a.fstride;
    j.whiten = a.whiten ? 1 : 0;
    j.onebit = a.onebit ? 1 : 0;
    j.nsta = a.nsta;
    j.ldj = p.ldj;
    j.X = X;
    const unsigned nwin = (unsigned)p.windows.size();
    if (p.stockham) {
      Cpx* tw = sc.get_n<Cpx>(p.M);
      Cpx* twh = sc.get_n<Cpx>(p.M + 1);
      if (!tw || !twh) return CCFJ_ERR_ALLOC;
      if (int e = twiddles(tw, p.M, p.M, s)) return e;
      if (int e = twiddles(twh, 2 * p.M, p.M + 1, s)) return e;
      j.tw = tw;
      j.twh = twh;
      const size_t smem = (size_t)p.M * sizeof(Cpx);
      CCFJ_CUDA_TRY(cudaFuncSetAttribute(xc_spectra_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      if (nwin > 0) {
        xc_spectra_kernel<<<nwin, kFftThreads, smem, s>>>(j);
        count_launch();
        CCFJ_LAUNCH_CHECK("xc_spectra_kernel");
      }
    } else {
      Cpx* tw = sc.get_n<Cpx>(p.F);
      if (!tw) return CCFJ_ERR_ALLOC;
      if (int e = twiddles(tw, p.F, p.F, s)) return e;
      j.tw = tw;
      if (nwin > 0) {
        xc_spectra_direct_kernel<<<dim3(nwin, div_up(a.nf, kDirectThreads)), kDirectThreads, 0,
                                   s>>>(j);
        count_launch();
        CCFJ_LAUNCH_CHECK("xc_spectra_direct_kernel");
      }
    }
    // pair products
    const Tile* d_tiles = upload(sc, p.tiles, s, &status);
    const int* d_lo = d_tiles ? upload(sc, p.lo, s, &status) : nullptr;
    const int* d_hi = d_lo ? upload(sc, p.hi, s, &status) : nullptr;
    const int* d_pmap = d_hi ? upload(sc, p.pmap, s, &status) : nullptr;
    const int* d_pnext = d_pmap ? upload(sc, p.pnext, s, &status) : nullptr;
    if (!d_pnext) return status;
    GramJob g = {};
    g.X = X;
    g.nsta = a.nsta;
    g.ldj = p.ldj;
    g.nf = a.nf;
    g.tiles = d_tiles;
    g.lo = d_lo;
    g.hi = d_hi;
    g.pmap = d_pmap;
    g.pnext = d_pnext;
    g.out_re = d_re;
    g.out_im = d_im;
    g.out_ld = a.out_layout == 1 ? 2LL * a.nf : a.nf;
    g.out_es = a.out_layout == 1 ? 2 : 1;
    g.accumulate = a.accumulate ? 1 : 0;
    xc_gram_kernel<<<dim3((unsigned)p.tiles.size(), div_up(a.nf, kLanes)), kGramThreads, 0, s>>>(g);
    count_launch();
    CCFJ_LAUNCH_CHECK("xc_gram_kernel");
  }

  if (!a.device_ptrs) {
    int st = CCFJ_OK;
    if (nout > 0 && a.out_layout == 1) {
      st = copy_to_host(a.out_re, d_re, 2 * plane, 0, s);
    } else if (nout > 0) {
      st = copy_to_host(a.out_re, d_re, plane, 0, s);
      if (st == CCFJ_OK) st = copy_to_host(a.out_im, d_im, plane, 0, s);
    } else {
      CCFJ_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (st != CCFJ_OK) return st;
  }
  return CCFJ_OK;
}

// Records to dispersion spectrum: the cross-correlation writes its
// complex64 cross-spectra into device scratch, and the transform reads
// their real parts there (perm, r, f, c and out as the caller gives them).
static int cc_fj_noise(const ccfj_cc_args& cc, const ccfj_fj_args& fj, cudaStream_t s) {
  CCFJ_REQUIRE(cc.struct_size == (int)sizeof(ccfj_cc_args),
               "ccfj_cc_fj_noise_v1: cc struct_size=%d, expected %d", cc.struct_size,
               (int)sizeof(ccfj_cc_args));
  CCFJ_REQUIRE(!cc.accumulate, "ccfj_cc_fj_noise_v1: cc->accumulate must be 0");
  CCFJ_REQUIRE(cc.device_ptrs == fj.device_ptrs,
               "ccfj_cc_fj_noise_v1: cc->device_ptrs (%d) != fj->device_ptrs (%d)",
               cc.device_ptrs, fj.device_ptrs);
  CCFJ_REQUIRE(cc.data != nullptr, "ccfj_cc_fj_noise_v1: data is NULL");
  CCFJ_REQUIRE(fj.nr == cc.npairs && fj.nf == cc.nf,
               "ccfj_cc_fj_noise_v1: fj nr=%d nf=%d must equal the pairs (%d) and bins (%d)",
               fj.nr, fj.nf, cc.npairs, cc.nf);
  CCFJ_REQUIRE(fj.mode == CCFJ_MODE_J || fj.mode == CCFJ_MODE_J_MINUS_Y,
               "ccfj_cc_fj_noise_v1: mode must be CCFJ_MODE_J (func 0) or CCFJ_MODE_J_MINUS_Y "
               "(func 1)");
  CCFJ_REQUIRE(cc.npairs >= 1 && cc.nf >= 1, "ccfj_cc_fj_noise_v1: npairs=%d nf=%d", cc.npairs,
               cc.nf);
  Scratch sc(s);
  float* spec = sc.get_n<float>(2 * (size_t)cc.npairs * cc.nf);
  if (!spec) return CCFJ_ERR_ALLOC;
  ccfj_cc_args c = cc;
  c.device_ptrs = 1;
  c.out_layout = 1;
  c.out_re = spec;
  c.out_im = nullptr;
  const long long nrec = (long long)cc.nsta * cc.npts;
  if (!cc.device_ptrs) {  // the records cross to the device once
    CCFJ_REQUIRE(cc.nsta >= 1 && cc.npts >= 1, "ccfj_cc_fj_noise_v1: nsta=%d npts=%d", cc.nsta,
                 cc.npts);
    float* d = sc.get_n<float>(nrec);
    if (!d) return CCFJ_ERR_ALLOC;
    const int cst = copy_from_host(d, cc.data, nrec * sizeof(float), s);
    if (cst != CCFJ_OK) return cst;
    c.data = d;
  }
  ccfj_fj_args f = fj;
  f.u[0] = spec;
  f.u[1] = nullptr;
  f.u_ld = 2LL * cc.nf;
  f.u_rows = cc.npairs;
  f.u_es = 2;
  f.u_ncols = cc.nf;
  f.fstride = 1;
  f.hilbert = fj.mode == CCFJ_MODE_J_MINUS_Y ? 1 : 0;
  f.col_begin = 0;
  f.nf_total = 0;
  f.device_ptrs = 1;
  int st = fj_validate(&f);
  if (st != CCFJ_OK) return st;
  if (!fj.device_ptrs) {  // the small per-pair and grid arrays, and the result
    float* dr = sc.get_n<float>(fj.nr);
    float* df = sc.get_n<float>(fj.nf);
    float* dc = sc.get_n<float>(fj.nc);
    float* dout = sc.get_n<float>((size_t)fj.nc * fj.nf);
    long long* dp = fj.perm ? sc.get_n<long long>(fj.nr) : nullptr;
    if (!dr || !df || !dc || !dout || (fj.perm && !dp)) return CCFJ_ERR_ALLOC;
    if (fj.perm)
      for (int i = 0; i < fj.nr; ++i)
        CCFJ_REQUIRE(fj.perm[i] >= 0 && fj.perm[i] < fj.nr,
                     "ccfj_cc_fj_noise_v1: perm[%d]=%lld out of range", i, fj.perm[i]);
    CCFJ_CUDA_TRY(cudaMemcpyAsync(dr, fj.r, sizeof(float) * fj.nr, cudaMemcpyHostToDevice, s));
    CCFJ_CUDA_TRY(cudaMemcpyAsync(df, fj.f, sizeof(float) * fj.nf, cudaMemcpyHostToDevice, s));
    CCFJ_CUDA_TRY(cudaMemcpyAsync(dc, fj.c, sizeof(float) * fj.nc, cudaMemcpyHostToDevice, s));
    if (dp)
      CCFJ_CUDA_TRY(cudaMemcpyAsync(dp, fj.perm, sizeof(long long) * fj.nr, cudaMemcpyHostToDevice,
                                    s));
    f.r = dr;
    f.f = df;
    f.c = dc;
    f.out = dout;
    f.perm = dp;
  }
  st = run(c, s);
  if (st != CCFJ_OK) return st;
  st = fj_device(f, s);
  if (st != CCFJ_OK) return st;
  if (!fj.device_ptrs) return copy_to_host(fj.out, f.out, sizeof(float) * fj.nc * fj.nf, 0, s);
  return CCFJ_OK;
}

}  // namespace xc
}  // namespace ccfj

CCFJ_API int ccfj_cc_fj_noise_v1(const ccfj_cc_args* cc, const ccfj_fj_args* fj, void* stream) {
  ccfj::clear_error();
  if (!cc || !fj) return ccfj::set_error(CCFJ_ERR_INVALID, "ccfj_cc_fj_noise_v1: NULL args");
  if (fj->struct_size != (int)sizeof(ccfj_fj_args))
    return ccfj::set_error(CCFJ_ERR_INVALID, "ccfj_cc_fj_noise_v1: fj struct_size=%d, expected %d",
                           fj->struct_size, (int)sizeof(ccfj_fj_args));
  return ccfj::xc::cc_fj_noise(*cc, *fj, (cudaStream_t)stream);
}

CCFJ_API int ccfj_cc_v1(const ccfj_cc_args* args, void* stream) {
  ccfj::clear_error();
  if (!args) return ccfj::set_error(CCFJ_ERR_INVALID, "ccfj_cc_v1: args is NULL");
  return ccfj::xc::run(*args, (cudaStream_t)stream);
}

CCFJ_API int CrossCorrelation(ccfj_cc_data d) {
  ccfj_cc_args a = {};
  a.struct_size = (int)sizeof(a);
  a.nsta = d.nsta;
  a.npts = d.npts;
  a.nf = d.nf;
  a.npairs = d.npairs;
  a.fstride = d.fstride;
  a.fftlen = d.fftlen;
  a.steplen = d.steplen;
  a.onebit = d.ifonebit;
  a.whiten = d.ifspecwhitenning;
  a.device_ptrs = 0;
  a.accumulate = 1;
  a.out_layout = 0;
  a.pairs = d.Pairs;
  a.startend = d.startend;
  a.data = d.data;
  a.out_re = d.ncfsr;
  a.out_im = d.ncfsi;
  return ccfj_cc_v1(&a, nullptr);
}
