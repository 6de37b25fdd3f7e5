// Time-domain front end of fj_earthquake and MWFJ on the device: optional
// taper window, real FFT, selection of the first nbins bins.
//
// The reference does this on the host with numpy (src/ccfj-gpu.pyx:274-278:
// argsort, np.fft.rfft of every trace, uf[:, 0:len(f)*fstride:fstride]) and,
// for MWFJ, multiplies every trace by `win` first (src/ccfj-gpu.pyx:168-178,
// 307-311).
//
// Power-of-two lengths N <= 32768 use an in-place radix-2 FFT of the N/2
// complex points z[m] = x[2m] + i x[2m+1] in shared memory (one CTA per
// trace) followed by the standard split that recovers the real transform,
//   X[k] = (Z[k] + conj Z[M-k]) / 2 - (i/2) e^{-2 pi i k/N} (Z[k] - conj Z[M-k]),
// M = N/2. Other lengths use a direct DFT of the requested bins whose phase
// index (k n mod N) is formed in integers.
//
// Output: complex [rows][nbins] as interleaved float pairs, row = sorted
// trace i (times window w for MWFJ: row = w * ntr + i).
#include <stdint.h>

#include "ccfj_core.cuh"
#include "fj_fft.cuh"
#include "fj_frontend.cuh"

namespace ccfj {

// Window value at sample t for the reference's `win`, given its integer
// n1, n2 and delta (computed on the host in float64 exactly as `win` does)
// and the trace length npts. `win` zeroes out[0:n1] and out[n2:npts] (a
// negative n2 counts from the end), then for i < delta writes
// sin(pi/2 i/delta) to out[n1 + i] and out[n2 - 1 - i] (a negative index
// again counts from the end; the host rejects loops that leave the array).
// The value at t is that of the last write to it -- the largest iteration
// index among t - n1, n2 - 1 - t and n2 - 1 - t + npts that lies in
// [0, delta) -- or, without one, the zero-filled head / tail or 1.
__device__ __forceinline__ float taper_value(int t, const TaperSpec& w, int npts) {
  int best = -1;
  const int ia = t - w.n1;
  if (ia >= 0 && ia < w.delta) best = ia;
  const int ib = w.n2 - 1 - t;
  if (ib >= 0 && ib < w.delta) best = max(best, ib);
  const int ibw = ib + npts;
  if (ibw >= 0 && ibw < w.delta) best = max(best, ibw);
  if (best >= 0) return sinpif(0.5f * (float)best / (float)w.delta);
  const int tail = w.n2 >= 0 ? w.n2 : max(npts + w.n2, 0);
  return (t < w.n1 || t >= tail) ? 0.0f : 1.0f;
}

// A sample range [lo, hi) outside which taper_value is zero: the hull of
// the ramps [n1, n1 + delta), [n2 - delta, n2), [n2 + npts - delta,
// n2 + npts) and the plateau [n1, tail), clipped to the trace. The FFT load
// skips the samples outside it (a window of 200-2000 samples in a trace of
// 16384 touches one eighth of the trace or less).
__device__ __forceinline__ void taper_support(const TaperSpec& w, int npts, int& lo, int& hi) {
  const int tail = w.n2 >= 0 ? w.n2 : max(npts + w.n2, 0);
  const int s[4] = {w.n1, w.n2 - w.delta, w.n2 + npts - w.delta, w.n1};
  const int e[4] = {w.n1 + w.delta, w.n2, w.n2 + npts, tail};
  lo = npts;
  hi = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int a = max(s[j], 0), b = min(e[j], npts);
    if (a < b) {
      lo = min(lo, a);
      hi = max(hi, b);
    }
  }
}

// Twiddles e^{-2 pi i t / M} for t < M/2, from FP64 sinpi/cospi.
__global__ void fft_twiddle_kernel(int M, float2* __restrict__ tw) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M / 2) return;
  double s, c;
  sincospi(-2.0 * t / M, &s, &c);
  tw[t] = make_float2((float)c, (float)s);
}

__device__ __forceinline__ unsigned bitrev(unsigned v, int bits) { return __brev(v) >> (32 - bits); }

constexpr int kFftThreads = 512;

// One CTA per output row. Shared memory: M float2.
__global__ void __launch_bounds__(kFftThreads) rfft_pow2_kernel(FftJob job, const float2* __restrict__ tw) {
  extern __shared__ float2 z[];
  const int M = job.npts / 2;
  const int bits = job.log2n - 1;
  const int row = blockIdx.x;
  const int i = row % job.ntr;  // sorted trace
  const long long src_row = job.perm ? job.perm[i] : i;
  const float* x = job.u + src_row * job.u_ld;
  TaperSpec tp;
  const bool taper = job.taper != nullptr;
  if (taper) tp = job.taper[row];
  // bit-reversed load of z[m] = x[2m] + i x[2m+1]
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    float a = x[2 * m], b = x[2 * m + 1];
    if (taper) {
      a *= taper_value(2 * m, tp, job.npts);
      b *= taper_value(2 * m + 1, tp, job.npts);
    }
    z[bits > 0 ? bitrev(m, bits) : 0] = make_float2(a, b);
  }
  __syncthreads();
  // radix-2 DIT butterflies
  for (int half = 1, tstride = M / 2; half < M; half *= 2, tstride /= 2) {
    for (int b = threadIdx.x; b < M / 2; b += blockDim.x) {
      const int grp = b / half, j = b - grp * half;
      const int p = grp * 2 * half + j, q = p + half;
      const float2 w = __ldg(tw + j * tstride);
      const float2 u = z[p], v = z[q];
      const float2 vw = make_float2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
      z[p] = make_float2(u.x + vw.x, u.y + vw.y);
      z[q] = make_float2(u.x - vw.x, u.y - vw.y);
    }
    __syncthreads();
  }
  // real-transform split, bins k < nbins (k <= M)
  float2* out = job.out + (long long)row * job.nbins;
  for (int kk = threadIdx.x; kk < job.nbins; kk += blockDim.x) {
    const int k = kk * job.bin_stride;
    if (k > M) {
      out[kk] = make_float2(0.f, 0.f);
      continue;
    }
    const float2 zk = z[k == M ? 0 : k];
    const float2 zm = z[k == 0 ? 0 : M - k];
    // E = (Z[k] + conj Z[M-k]) / 2, O = (Z[k] - conj Z[M-k]) / (2i)
    const float er = 0.5f * (zk.x + zm.x), ei = 0.5f * (zk.y - zm.y);
    const float orr = 0.5f * (zk.y + zm.y), oi = -0.5f * (zk.x - zm.x);
    float s, c;
    sincospif(-2.0f * (float)k / (float)job.npts, &s, &c);  // k/N exact (N = 2^p)
    out[kk] = make_float2(er + c * orr - s * oi, ei + c * oi + s * orr);
  }
}

// ------------------------------------------ Stockham FFT, 16 points per thread
// For 512 <= M <= 8192 complex points (N = 2M real samples): M/16 threads per
// row, each holding 16 points in registers. The passes follow Stockham's
// autosort formulation (no bit reversal): a pass of radix R over sub-
// transforms of size Ns reads in[j + r M/R] (r < R), multiplies by
// e^{-2 pi i r (j mod Ns) / (Ns R)}, takes an R-point DFT and writes
// out[(j / Ns) Ns R + (j mod Ns) + r Ns]. Radix 16 while at least 16 remain,
// then one pass of the remaining radix (2, 4 or 8, each thread doing 16/R
// butterflies): 4 passes for M = 8192 instead of 13 radix-2 stages. The
// first pass reads the (tapered) trace straight from global memory; the
// others go through one shared-memory buffer with a pad slot per 16
// entries, so that the strided writes of the early passes do not collide
// in the banks.
constexpr int kStockMinM = 512, kStockMaxM = 8192;

__device__ __forceinline__ int spad(int i) { return i + (i >> 4); }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-register R-point DFT (R = 2, 4, 8, 16), natural order in and out:
// radix-2 decimation in time over bit-reversed register indices, with the
// 16th roots of unity as constants.
template <int R>
__device__ __forceinline__ void dft_pow2(float2* v) {
  // cos and -sin of 2 pi m / 16, m = 0..7
  constexpr float kC[8] = {1.0f, 0.92387953251128674f, 0.70710678118654752f,
                           0.38268343236508977f, 0.0f, -0.38268343236508977f,
                           -0.70710678118654752f, -0.92387953251128674f};
  constexpr float kS[8] = {0.0f, -0.38268343236508977f, -0.70710678118654752f,
                           -0.92387953251128674f, -1.0f, -0.92387953251128674f,
                           -0.70710678118654752f, -0.38268343236508977f};
  constexpr int LOG = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
  float2 t[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    int rev = 0;
#pragma unroll
    for (int b = 0; b < LOG; ++b) rev |= ((i >> b) & 1) << (LOG - 1 - b);
    t[rev] = v[i];
  }
#pragma unroll
  for (int h = 1; h < R; h *= 2) {
#pragma unroll
    for (int g = 0; g < R; g += 2 * h) {
#pragma unroll
      for (int jj = 0; jj < h; ++jj) {
        const int m = jj * (8 / h);  // e^{-2 pi i jj / (2h)} = W16^m
        const float2 w = make_float2(kC[m], kS[m]);
        const float2 u = t[g + jj];
        const float2 x = h == 1 ? t[g + jj + h] : cmul(t[g + jj + h], w);
        t[g + jj] = make_float2(u.x + x.x, u.y + x.y);
        t[g + jj + h] = make_float2(u.x - x.x, u.y - x.y);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = t[i];
}

// e^{-2 pi i t / M} for t < M from the half table tw (t < M/2).
__device__ __forceinline__ float2 twiddle_full(const float2* __restrict__ tw, int t, int M) {
  const int h = M >> 1;
  const float2 w = __ldg(tw + (t < h ? t : t - h));
  return t < h ? w : make_float2(-w.x, -w.y);
}

// w[r] = e^{-2 pi i r t / M} for r < R (r t < M): the table entries of t,
// 2t, 4t and 8t, the other powers as products of those (at most three
// products deep, a few ulp). The twiddle indices of a warp's lanes are far
// apart in the table, so each table read costs one L1 wavefront per lane
// group; four reads per butterfly instead of R - 1.
template <int R>
__device__ __forceinline__ void twiddle_powers(const float2* __restrict__ tw, int t, int M,
                                               float2 (&w)[R]) {
  w[0] = make_float2(1.0f, 0.0f);
  w[1] = twiddle_full(tw, t, M);
  if (R >= 4) {
    w[2 % R] = twiddle_full(tw, 2 * t, M);
    w[3 % R] = cmul(w[1], w[2 % R]);
  }
  if (R >= 8) {
    w[4 % R] = twiddle_full(tw, 4 * t, M);
#pragma unroll
    for (int r = 5; r < 8; ++r) w[r % R] = cmul(w[4 % R], w[(r - 4) % R]);
  }
  if (R >= 16) {
    w[8 % R] = twiddle_full(tw, 8 * t, M);
#pragma unroll
    for (int r = 9; r < 16; ++r) w[r % R] = cmul(w[8 % R], w[(r - 8) % R]);
  }
}

// One Stockham pass of radix R over the 16 registers of thread tid (16/R
// butterflies j = tid + g P), writing the outputs to shared memory. In the
// last pass (Ns R = M) butterfly j writes outputs j + r Ns; one none of
// whose outputs is at most kneed or at least M - kneed is skipped (the
// real-FFT split reads only those).
template <int R>
__device__ __forceinline__ void stockham_pass(float2 (&v)[16], float2* sz, int M, int Ns,
                                              const float2* __restrict__ tw, int tid, int P,
                                              int kneed) {
#pragma unroll
  for (int g = 0; g < 16 / R; ++g) {
    const int j = tid + g * P;
    if (Ns * R == M && j > kneed && j + (R - 1) * Ns < M - kneed) continue;
    const int k = j % Ns;
    float2* u = v + g * R;
    if (Ns > 1) {
      float2 w[R];
      twiddle_powers<R>(tw, k * (M / (Ns * R)), M, w);
#pragma unroll
      for (int r = 1; r < R; ++r) u[r] = cmul(u[r], w[r]);
    }
    dft_pow2<R>(u);
    const int o = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) sz[spad(o + r * Ns)] = u[r];
  }
}

// Reads the inputs of a radix-R pass from shared memory.
template <int R>
__device__ __forceinline__ void stockham_load(float2 (&v)[16], const float2* sz, int M, int tid,
                                              int P) {
#pragma unroll
  for (int g = 0; g < 16 / R; ++g) {
    const int j = tid + g * P;
#pragma unroll
    for (int r = 0; r < R; ++r) v[g * R + r] = sz[spad(j + r * (M / R))];
  }
}

// The whole M-point FFT of the 16 points per thread in v (the first pass's
// inputs, in[tid + r P]); the result is left in natural order in sz (padded
// indices) and the CTA is synchronised. Only outputs at most kneed or at
// least M - kneed are guaranteed (kneed >= M: all of them).
__device__ __forceinline__ void stockham_fft(float2 (&v)[16], float2* sz, int M,
                                             const float2* __restrict__ tw, int tid, int P,
                                             int kneed) {
  stockham_pass<16>(v, sz, M, 1, tw, tid, P, kneed);
  __syncthreads();
  int Ns = 16;
  while (Ns < M) {
    const int rem = M / Ns;
    if (rem >= 16) {
      stockham_load<16>(v, sz, M, tid, P);
      __syncthreads();
      stockham_pass<16>(v, sz, M, Ns, tw, tid, P, kneed);
      Ns *= 16;
    } else if (rem == 8) {
      stockham_load<8>(v, sz, M, tid, P);
      __syncthreads();
      stockham_pass<8>(v, sz, M, Ns, tw, tid, P, kneed);
      Ns *= 8;
    } else if (rem == 4) {
      stockham_load<4>(v, sz, M, tid, P);
      __syncthreads();
      stockham_pass<4>(v, sz, M, Ns, tw, tid, P, kneed);
      Ns *= 4;
    } else {
      stockham_load<2>(v, sz, M, tid, P);
      __syncthreads();
      stockham_pass<2>(v, sz, M, Ns, tw, tid, P, kneed);
      Ns *= 2;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kStockMaxM / 16, 2)
    rfft_stockham_kernel(FftJob job, const float2* __restrict__ tw) {
  extern __shared__ float2 sz[];
  const int M = job.npts >> 1;
  const int P = M >> 4;
  const int tid = threadIdx.x;
  const int row = blockIdx.x;
  const int i = row % job.ntr;  // sorted trace
  const long long src_row = job.perm ? job.perm[i] : i;
  const float2* x = reinterpret_cast<const float2*>(job.u + src_row * job.u_ld);
  const bool taper = job.taper != nullptr;
  TaperSpec tp;
  if (taper) tp = job.taper[row];
  // first pass (radix 16, Ns = 1): z[m] = x[2m] + i x[2m+1], m = tid + r P
  // all 16 loads are issued before any taper arithmetic, so they overlap;
  // with a taper, points whose two samples lie outside the window's support
  // are zero and are not loaded
  float2 v[16];
  if (taper) {
    int lo, hi;
    taper_support(tp, job.npts, lo, hi);
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int m = tid + r * P;
      v[r] = (2 * m + 1 >= lo && 2 * m < hi) ? __ldg(x + m) : make_float2(0.0f, 0.0f);
    }
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int m = tid + r * P;
      if (2 * m + 1 >= lo && 2 * m < hi) {
        v[r].x *= taper_value(2 * m, tp, job.npts);
        v[r].y *= taper_value(2 * m + 1, tp, job.npts);
      }
    }
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = __ldg(x + tid + r * P);
  }
  // the split below reads bins up to (nbins - 1) bin_stride and their mirrors
  const long long kmax = (long long)(job.nbins - 1) * job.bin_stride;
  stockham_fft(v, sz, M, tw, tid, P, kmax < M ? (int)kmax : M);
  // real-transform split, bins k < nbins (k <= M)
  float2* out = job.out + (long long)row * job.nbins;
  for (int kk = tid; kk < job.nbins; kk += P) {
    const int k = kk * job.bin_stride;
    if (k > M) {
      out[kk] = make_float2(0.f, 0.f);
      continue;
    }
    const float2 zk = sz[spad(k == M ? 0 : k)];
    const float2 zm = sz[spad(k == 0 ? 0 : M - k)];
    const float er = 0.5f * (zk.x + zm.x), ei = 0.5f * (zk.y - zm.y);
    const float orr = 0.5f * (zk.y + zm.y), oi = -0.5f * (zk.x - zm.x);
    float s, c;
    sincospif(-2.0f * (float)k / (float)job.npts, &s, &c);  // k/N exact (N = 2^p)
    out[kk] = make_float2(er + c * orr - s * oi, ei + c * oi + s * orr);
  }
}

// ------------------------------------------ Hilbert transform by FFT
// For rows of n = 512..8192 (a power of two) columns: two rows per CTA,
// packed as z = x_a + i x_b (the transform is linear over complex scalars);
// Z = FFT(z); bin k times +i sign(k) (scipy.fftpack.hilbert's multiplier
// with numpy's forward sign convention; 0 at k = 0 and k = n/2); then the
// inverse as y = conj(FFT(conj(Z'))) / n, so H(x_a) = Re y and H(x_b) = Im y.
// O(n log n) per row instead of the direct convolution's O(n^2).
__global__ void __launch_bounds__(kStockMaxM / 16, 2)
    hilbert_fft_kernel(InDesc in, int n, int es, int nr, int nf, int fstride, int col_begin,
                       const float2* __restrict__ tw, float* __restrict__ dst) {
  extern __shared__ float2 sz[];
  const int M = n, P = M >> 4, tid = threadIdx.x;
  const int ia = 2 * blockIdx.x, ib = ia + 1;
  const bool has_b = ib < nr;
  const float* xa = in.p + (in.perm ? in.perm[ia] : ia) * in.ld;
  const float* xb = has_b ? in.p + (in.perm ? in.perm[ib] : ib) * in.ld : xa;
  float2 v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const long long m = tid + r * P;
    v[r] = make_float2(xa[m * es], has_b ? xb[m * es] : 0.0f);
  }
  stockham_fft(v, sz, M, tw, tid, P, M);
  const int h = M >> 1;
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const int m = tid + r * P;
    const float2 z = sz[spad(m)];
    // conj(Z +i) = (-z.y, -z.x) for 0 < m < n/2; conj(Z -i) = (z.y, z.x) above
    v[r] = (m == 0 || m == h) ? make_float2(0.0f, 0.0f)
           : m < h            ? make_float2(-z.y, -z.x)
                              : make_float2(z.y, z.x);
  }
  __syncthreads();  // every read of Z is done before the second FFT writes sz
  stockham_fft(v, sz, M, tw, tid, P, M);
  const float inv_n = 1.0f / (float)n;
  for (int j = tid; j < n; j += P) {
    if (j % fstride) continue;
    const int col = j / fstride - col_begin;
    if (col < 0 || col >= nf) continue;
    const float2 y = sz[spad(j)];
    dst[(long long)ia * nf + col] = y.x * inv_n;
    if (has_b) dst[(long long)ib * nf + col] = -y.y * inv_n;
  }
}

bool hilbert_fft_supported(int n) {
  return n >= kStockMinM && n <= kStockMaxM && (n & (n - 1)) == 0;
}

int hilbert_rows_fft(const InDesc& in, int n, int es, int nr, int nf, int fstride, int col_begin,
                     float* dst, cudaStream_t s, Scratch& sc) {
  float2* tw = sc.get_n<float2>(n / 2);
  if (!tw) return CCFJ_ERR_ALLOC;
  fft_twiddle_kernel<<<div_up(n / 2, 256), 256, 0, s>>>(n, tw);
  count_launch();
  CCFJ_LAUNCH_CHECK("fft_twiddle_kernel");
  const size_t smem = sizeof(float2) * (size_t)(n + n / 16);
  CCFJ_CUDA_TRY(cudaFuncSetAttribute(hilbert_fft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  hilbert_fft_kernel<<<div_up(nr, 2), n / 16, smem, s>>>(in, n, es, nr, nf, fstride, col_begin, tw,
                                                          dst);
  count_launch();
  CCFJ_LAUNCH_CHECK("hilbert_fft_kernel");
  return CCFJ_OK;
}

// Direct DFT for lengths that are not powers of two: one thread per
// (row, bin); the phase index k n mod N is exact in 64-bit integers.
__global__ void rdft_kernel(FftJob job) {
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int row = blockIdx.x;
  if (kk >= job.nbins) return;
  const long long k = (long long)kk * job.bin_stride;
  float2* out = job.out + (long long)row * job.nbins;
  const int N = job.npts;
  if (k > N / 2) {
    out[kk] = make_float2(0.f, 0.f);
    return;
  }
  const int i = row % job.ntr;
  const long long src_row = job.perm ? job.perm[i] : i;
  const float* x = job.u + src_row * job.u_ld;
  const bool taper = job.taper != nullptr;
  TaperSpec tp;
  if (taper) tp = job.taper[row];
  double re = 0, im = 0;
  long long p = 0;  // k n mod N
  for (int n = 0; n < N; ++n) {
    float v = x[n];
    if (taper) v *= taper_value(n, tp, N);
    float s, c;
    sincospif(-2.0f * (float)p / (float)N, &s, &c);
    re += (double)(v * c);
    im += (double)(v * s);
    p += k;
    if (p >= N) p -= N;
  }
  out[kk] = make_float2((float)re, (float)im);
}

int rfft_bins(const FftJob& job, int nrows_out, cudaStream_t s, Scratch& sc) {
  CCFJ_REQUIRE(job.npts >= 2, "rfft: npts=%d must be >= 2", job.npts);
  const bool pow2 = (job.npts & (job.npts - 1)) == 0 && job.npts <= 32768;
  if (pow2) {
    const int M = job.npts / 2;
    float2* tw = sc.get_n<float2>(M / 2 > 0 ? M / 2 : 1);
    if (!tw) return CCFJ_ERR_ALLOC;
    if (M >= 2) {
      fft_twiddle_kernel<<<div_up(M / 2, 256), 256, 0, s>>>(M, tw);
      count_launch();
      CCFJ_LAUNCH_CHECK("fft_twiddle_kernel");
    }
    FftJob j = job;
    j.log2n = 0;
    while ((1 << j.log2n) < job.npts) ++j.log2n;
    if (M >= kStockMinM && M <= kStockMaxM && (job.u_ld % 2) == 0 &&
        (reinterpret_cast<uintptr_t>(job.u) % 8) == 0) {
      const size_t smem = sizeof(float2) * (size_t)(M + M / 16);
      CCFJ_CUDA_TRY(cudaFuncSetAttribute(rfft_stockham_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      rfft_stockham_kernel<<<nrows_out, M / 16, smem, s>>>(j, tw);
      count_launch();
      CCFJ_LAUNCH_CHECK("rfft_stockham_kernel");
    } else {
      const size_t smem = sizeof(float2) * (size_t)M;
      CCFJ_CUDA_TRY(cudaFuncSetAttribute(rfft_pow2_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      rfft_pow2_kernel<<<nrows_out, kFftThreads, smem, s>>>(j, tw);
      count_launch();
      CCFJ_LAUNCH_CHECK("rfft_pow2_kernel");
    }
  } else {
    rdft_kernel<<<dim3(nrows_out, div_up(job.nbins, 128)), 128, 0, s>>>(job);
    count_launch();
    CCFJ_LAUNCH_CHECK("rdft_kernel");
  }
  return CCFJ_OK;
}

}  // namespace ccfj
