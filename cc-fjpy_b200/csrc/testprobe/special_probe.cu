// Test library (libccfj_b200_probe.so, not part of the product library):
// evaluates the special-function code of the transform kernels
// (fj_special.cuh, the same source the kernels include) on the host and on
// the device, so that unit tests can hold the approximations to
// high-precision values. Declared in include/ccfj_b200_probe.h.
#include <cuda_runtime.h>

#include "../../../include/ccfj_b200.h"
#include "../../../include/ccfj_b200_probe.h"
#include "../fj_cells.cuh"

namespace {

__host__ __device__ void special_values(int precision, double x, double* o) {
  // the phase in cycles as a double-float, as the kernels form it
  const double t = x / fjs::kTwoPi;
  if (precision == CCFJ_PREC_FP32) {
    const float p_hi = (float)t;
    const float p_lo = (float)(t - (double)p_hi);
    fjs::ZB<float> J, Y;
    fjs::eval_station_f32<true, true, true>((float)x, p_hi, p_lo, true, J, Y);
    o[0] = J.z0; o[1] = J.z1; o[2] = J.b; o[3] = Y.z0; o[4] = Y.z1; o[5] = Y.b;
  } else {
    fjs::ZB<double> J, Y;
    fjs::eval_station_f64<true, true, true>(x, t, J, Y);
    o[0] = J.z0; o[1] = J.z1; o[2] = J.b; o[3] = Y.z0; o[4] = Y.z1; o[5] = Y.b;
  }
}

__global__ void special_device_kernel(int precision, long long n, const double* __restrict__ x,
                                      double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) special_values(precision, x[i], out + 6 * i);
}

bool bad_args(int precision, long long n, const void* x, const void* out) {
  return n < 0 || (n > 0 && (!x || !out)) ||
         (precision != CCFJ_PREC_FP32 && precision != CCFJ_PREC_FP64);
}

}  // namespace

#if defined(FJS_HAVE_PAIRED)
// Station values y0 = J0 / M, y1 = J1 / M of two cells (f, c0) and (f, c1)
// at r (x >= 8 in both), by the scalar x >= 8 path of the transform kernels
// and by their paired (two cells per instruction) path.
__global__ void paired_probe_kernel(long long n, const float* __restrict__ in,
                                    float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float f = in[4 * i], c0 = in[4 * i + 1], c1 = in[4 * i + 2], r = in[4 * i + 3];
  ccfj::Cell<float> cl[2];
  cl[0].init(f, c0);
  cl[1].init(f, c1);
  cl[0].prepare_folded();
  cl[1].prepare_folded();
  const float rinv = 1.0f / r, sqrtr = sqrtf(r);
  float* o = out + 8 * i;
  for (int j = 0; j < 2; ++j) {
    fjs::ZB<float> J{}, Y{};
    cl[j].template eval_y<true, false, true, true>(r, rinv, sqrtr, J, Y);
    o[2 * j] = J.z0;
    o[2 * j + 1] = J.z1;
  }
  const fjs::PairPhase ph{make_float2(cl[0].q_hi, cl[1].q_hi), make_float2(-cl[0].q_hi, -cl[1].q_hi),
                          make_float2(cl[0].q_lo, cl[1].q_lo), make_float2(cl[0].s8, cl[1].s8)};
  fjs::ZB2 J2;
  fjs::eval_large_scaled_pair_j(ph, r, rinv, J2);
  o[4] = J2.z0.x;
  o[5] = J2.z1.x;
  o[6] = J2.z0.y;
  o[7] = J2.z1.y;
}
#endif

CCFJ_PROBE_API int ccfj_paired_probe(long long n, const float* in, float* out, void* stream) {
#if defined(FJS_HAVE_PAIRED)
  if (n < 0 || (n > 0 && (!in || !out))) return CCFJ_ERR_INVALID;
  if (n == 0) return CCFJ_OK;
  paired_probe_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, in, out);
  return cudaGetLastError() == cudaSuccess ? CCFJ_OK : CCFJ_ERR_CUDA;
#else
  (void)n; (void)in; (void)out; (void)stream;
  return CCFJ_ERR_UNSUPPORTED;
#endif
}

CCFJ_PROBE_API int ccfj_special_host(int precision, long long n, const double* x, double* out) {
  if (bad_args(precision, n, x, out)) return CCFJ_ERR_INVALID;
  for (long long i = 0; i < n; ++i) special_values(precision, x[i], out + 6 * i);
  return CCFJ_OK;
}

CCFJ_PROBE_API int ccfj_special_device(int precision, long long n, const double* x, double* out,
                                       void* stream) {
  if (bad_args(precision, n, x, out)) return CCFJ_ERR_INVALID;
  if (n == 0) return CCFJ_OK;
  special_device_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(precision,
                                                                                      n, x, out);
  return cudaGetLastError() == cudaSuccess ? CCFJ_OK : CCFJ_ERR_CUDA;
}
