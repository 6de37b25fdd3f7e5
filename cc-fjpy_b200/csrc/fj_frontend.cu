// Front ends that turn the caller's arrays into the F-J inputs on the device.
//
//   Hilbert transform along frequency (fj_noise func=1): the reference runs
//   scipy.fftpack.hilbert on every full row on the host
//   (src/ccfj-gpu.pyx:258-260). For a length-n row, scipy multiplies the
//   DFT coefficient k (numpy's forward convention, e^{-2 pi i k m / n}) by
//   +i sign(k), with the k = 0 term and, for even n, the Nyquist term set to
//   zero. Rows of 512..8192 (a power of two) columns take the FFT
//   (hilbert_rows_fft, fj_fft.cu); other lengths take the equivalent
//   circular convolution y[j] = sum_m h[m] x[(j - m) mod n] with
//       h[m] = -(2/n) sum_{k=1}^{K} sin(2 pi k m / n),   K = floor((n-1)/2)
//            = -(2/n) sin(K th/2) sin((K+1) th/2) / sin(th/2),  th = 2 pi m/n
//   (h[0] = 0), evaluated directly from a shared-memory copy of the row.
#include "ccfj_core.cuh"
#include "fj_frontend.cuh"

namespace ccfj {

// h[m] in FP64, rounded to FP32. sinpi keeps the arguments exact.
__global__ void hilbert_kernel_table(int n, float* __restrict__ h) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  if (m == 0) {
    h[0] = 0.0f;
    return;
  }
  const long long K = (n - 1) / 2;
  // th/2 = pi m / n; reduce the integer numerators mod 2n before scaling
  const long long twoN = 2LL * n;
  const double a = (double)((K * m) % twoN) / n;        // K th/2 / pi
  const double b = (double)(((K + 1) * m) % twoN) / n;  // (K+1) th/2 / pi
  const double c = (double)m / n;                       // th/2 / pi
  h[m] = (float)(-2.0 / n * sinpi(a) * sinpi(b) / sinpi(c));
}

constexpr int kHilR = 8;      // outputs per thread per pass
constexpr int kHilThreads = 256;
constexpr int kHilMaxN = 16384;  // 3 n floats of shared memory (192 KiB)

// One block per row (sorted order); shared memory holds the row twice
// (x2[t] = x[t mod n], so no index wraps) and the kernel table h. Thread
// tid sums outputs j = tid + 256 t: the x2 reads of a warp are consecutive
// words (no bank conflicts) and the h read is a broadcast.
__global__ void __launch_bounds__(kHilThreads) hilbert_rows_kernel(InDesc in, int n, int es, int nf,
                                                                  int fstride, int col_begin,
                                                                  const float* __restrict__ h,
                                                                  float* __restrict__ dst) {
  extern __shared__ float sm[];
  float* x2 = sm;          // [2n]
  float* hs = sm + 2 * n;  // [n]
  const int i = blockIdx.x;
  const long long row = in.perm ? in.perm[i] : i;
  const float* src = in.p + row * in.ld;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const float v = src[(long long)t * es];
    x2[t] = v;
    x2[t + n] = v;
    hs[t] = h[t];
  }
  __syncthreads();
  for (int j0 = 0; j0 < n; j0 += kHilThreads * kHilR) {
    float acc[kHilR];
#pragma unroll
    for (int t = 0; t < kHilR; ++t) acc[t] = 0.0f;
    const int jb = j0 + threadIdx.x + n;  // x2 index of output j at m = 0
    // outputs of this pass that exist (t with j0 + 256 t < n; uniform per CTA)
    const int tn = min(kHilR, (n - j0 + kHilThreads - 1) / kHilThreads);
    // y[j] = sum_m h[m] x2[j - m + n]; j - m + n stays in [1, 2n - 1]
    for (int m = 0; m < n; ++m) {
      const float hv = hs[m];
#pragma unroll
      for (int t = 0; t < kHilR; ++t) {
        const int idx = jb + t * kHilThreads - m;
        if (t < tn && idx < 2 * n) acc[t] = fmaf(hv, x2[idx], acc[t]);
      }
    }
    // keep only the columns the transform uses
#pragma unroll
    for (int t = 0; t < kHilR; ++t) {
      const int j = j0 + threadIdx.x + t * kHilThreads;
      const int col = j / fstride - col_begin;
      if (j < n && j % fstride == 0 && col >= 0 && col < nf) dst[(long long)i * nf + col] = acc[t];
    }
  }
}

int hilbert_rows(const InDesc& in, int n, int es, int nr, int nf, int fstride, int col_begin,
                 float* dst, cudaStream_t s, Scratch& sc) {
  if (hilbert_fft_supported(n))
    return hilbert_rows_fft(in, n, es, nr, nf, fstride, col_begin, dst, s, sc);
  if (n > kHilMaxN)
    return set_error(CCFJ_ERR_UNSUPPORTED,
                     "Hilbert transform rows longer than %d columns are not supported (got %d)",
                     kHilMaxN, n);
  float* h = sc.get_n<float>(n);
  if (!h) return CCFJ_ERR_ALLOC;
  hilbert_kernel_table<<<div_up(n, 256), 256, 0, s>>>(n, h);
  count_launch();
  CCFJ_LAUNCH_CHECK("hilbert_kernel_table");
  const size_t smem = sizeof(float) * 3 * (size_t)n;
  CCFJ_CUDA_TRY(cudaFuncSetAttribute(hilbert_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  hilbert_rows_kernel<<<nr, kHilThreads, smem, s>>>(in, n, es, nf, fstride, col_begin, h, dst);
  count_launch();
  CCFJ_LAUNCH_CHECK("hilbert_rows_kernel");
  return CCFJ_OK;
}

}  // namespace ccfj
