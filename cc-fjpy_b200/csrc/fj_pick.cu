// Dispersion-curve picking on an F-J spectrum (no counterpart in the
// reference, whose users pick the curves from the plotted spectrum): per
// frequency column of out[nc][nf], the velocity of the largest value within
// a velocity band, refined between the grid velocities by the vertex of the
// parabola through the maximum and its two neighbours.
//
// One thread per frequency walks the column (consecutive threads read
// consecutive frequencies of one velocity row: coalesced). The column's
// first largest value is taken (numpy's argmax order); a NaN anywhere in the
// band gives a NaN pick and amplitude, as a NaN column of the transform (f = 0)
// should.
#include <math.h>

#include "ccfj_core.cuh"

namespace ccfj {

__global__ void fj_pick_kernel(const float* __restrict__ spec, int nc, int nf,
                               const float* __restrict__ c, const float* __restrict__ cmin,
                               const float* __restrict__ cmax, float* __restrict__ cpick,
                               float* __restrict__ amp) {
  const int fi = blockIdx.x * blockDim.x + threadIdx.x;
  if (fi >= nf) return;
  const float lo = cmin ? cmin[fi] : -INFINITY;
  const float hi = cmax ? cmax[fi] : INFINITY;
  int best = -1;
  float bv = 0.0f;
  bool has_nan = false;
  for (int j = 0; j < nc; ++j) {
    const float cj = c[j];
    if (!(cj >= lo && cj <= hi)) continue;
    const float v = spec[(long long)j * nf + fi];
    if (isnan(v)) {
      has_nan = true;
      break;
    }
    if (best < 0 || v > bv) {
      best = j;
      bv = v;
    }
  }
  if (has_nan || best < 0) {
    cpick[fi] = __int_as_float(0x7fffffff);
    if (amp) amp[fi] = __int_as_float(0x7fffffff);
    return;
  }
  float cp = c[best], ap = bv;
  const bool in_lo = best > 0 && c[best - 1] >= lo && c[best - 1] <= hi;
  const bool in_hi = best + 1 < nc && c[best + 1] >= lo && c[best + 1] <= hi;
  if (in_lo && in_hi) {
    const float ym = spec[(long long)(best - 1) * nf + fi];
    const float yp = spec[(long long)(best + 1) * nf + fi];
    const float den = ym - 2.0f * bv + yp;
    if (den < 0.0f) {
      const float d = fminf(0.5f, fmaxf(-0.5f, 0.5f * (ym - yp) / den));
      cp = d >= 0.0f ? c[best] + d * (c[best + 1] - c[best]) : c[best] + d * (c[best] - c[best - 1]);
      ap = bv - 0.25f * (ym - yp) * d;
    }
  }
  cpick[fi] = cp;
  if (amp) amp[fi] = ap;
}

}  // namespace ccfj

CCFJ_API int ccfj_pick_v1(const float* spec, int nc, int nf, const float* c, const float* cmin,
                          const float* cmax, float* cpick, float* amp, int device_ptrs,
                          void* stream) {
  ccfj::clear_error();
  CCFJ_REQUIRE(nc >= 1 && nf >= 1, "ccfj_pick_v1: nc=%d nf=%d must be >= 1", nc, nf);
  CCFJ_REQUIRE(spec && c && cpick, "ccfj_pick_v1: NULL array");
  cudaStream_t s = (cudaStream_t)stream;
  if (device_ptrs) {
    ccfj::fj_pick_kernel<<<ccfj::div_up(nf, 128), 128, 0, s>>>(spec, nc, nf, c, cmin, cmax, cpick,
                                                               amp);
    ccfj::count_launch();
    CCFJ_LAUNCH_CHECK("fj_pick_kernel");
    return CCFJ_OK;
  }
  ccfj::Scratch sc(s);
  float* ds = sc.get_n<float>((size_t)nc * nf);
  float* dc = sc.get_n<float>(nc);
  float* dlo = cmin ? sc.get_n<float>(nf) : nullptr;
  float* dhi = cmax ? sc.get_n<float>(nf) : nullptr;
  float* dp = sc.get_n<float>(nf);
  float* da = amp ? sc.get_n<float>(nf) : nullptr;
  if (!ds || !dc || !dp || (cmin && !dlo) || (cmax && !dhi) || (amp && !da)) return CCFJ_ERR_ALLOC;
  CCFJ_CUDA_TRY(cudaMemcpyAsync(ds, spec, sizeof(float) * nc * nf, cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dc, c, sizeof(float) * nc, cudaMemcpyHostToDevice, s));
  if (dlo) CCFJ_CUDA_TRY(cudaMemcpyAsync(dlo, cmin, sizeof(float) * nf, cudaMemcpyHostToDevice, s));
  if (dhi) CCFJ_CUDA_TRY(cudaMemcpyAsync(dhi, cmax, sizeof(float) * nf, cudaMemcpyHostToDevice, s));
  ccfj::fj_pick_kernel<<<ccfj::div_up(nf, 128), 128, 0, s>>>(ds, nc, nf, dc, dlo, dhi, dp, da);
  ccfj::count_launch();
  CCFJ_LAUNCH_CHECK("fj_pick_kernel");
  CCFJ_CUDA_TRY(cudaMemcpyAsync(cpick, dp, sizeof(float) * nf, cudaMemcpyDeviceToHost, s));
  if (amp) CCFJ_CUDA_TRY(cudaMemcpyAsync(amp, da, sizeof(float) * nf, cudaMemcpyDeviceToHost, s));
  CCFJ_CUDA_TRY(cudaStreamSynchronize(s));
  return CCFJ_OK;
}
