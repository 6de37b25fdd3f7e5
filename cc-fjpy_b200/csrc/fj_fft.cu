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
#include "ccfj_core.cuh"
#include "fj_fft.cuh"

namespace ccfj {

// Window value at sample t for the reference's `win`, given its integer
// n1, n2 and delta (computed on the host in float64 exactly as `win` does).
// Where both sine ramps cover t (delta > (n2-n1)/2, taper < 0) the later
// write of the reference's loop wins, i.e. the larger ramp index.
__device__ __forceinline__ float taper_value(int t, const TaperSpec& w) {
  if (t < w.n1 || t >= w.n2) return 0.0f;
  const int i = t - w.n1;
  const int j = w.n2 - 1 - t;
  int m;
  if (i < w.delta && j < w.delta)
    m = max(i, j);
  else if (i < w.delta)
    m = i;
  else if (j < w.delta)
    m = j;
  else
    return 1.0f;
  return sinpif(0.5f * (float)m / (float)w.delta);
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
      a *= taper_value(2 * m, tp);
      b *= taper_value(2 * m + 1, tp);
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
    if (taper) v *= taper_value(n, tp);
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
    const size_t smem = sizeof(float2) * (size_t)M;
    CCFJ_CUDA_TRY(cudaFuncSetAttribute(rfft_pow2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    rfft_pow2_kernel<<<nrows_out, kFftThreads, smem, s>>>(j, tw);
    count_launch();
    CCFJ_LAUNCH_CHECK("rfft_pow2_kernel");
  } else {
    rdft_kernel<<<dim3(nrows_out, div_up(job.nbins, 128)), 128, 0, s>>>(job);
    count_launch();
    CCFJ_LAUNCH_CHECK("rdft_kernel");
  }
  return CCFJ_OK;
}

}  // namespace ccfj
