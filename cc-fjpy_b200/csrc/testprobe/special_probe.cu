// Test library (libccfj_b200_probe.so, not part of the product library):
// evaluates the special-function code of the transform kernels
// (fj_special.cuh, the same source the kernels include) on the host and on
// the device, so that unit tests can hold the approximations to
// high-precision values. Declared in include/ccfj_b200_probe.h.
#include <cuda_runtime.h>

#include "../../../include/ccfj_b200.h"
#include "../../../include/ccfj_b200_probe.h"
#include "../fj_special.cuh"

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
