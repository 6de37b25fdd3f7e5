// ccfj_fj_earthquake_v1: fj_earthquake and MWFJ from time-domain traces.
//
// Reference: src/ccfj-gpu.pyx:270-295 (fj_earthquake) and :297-313 (MWFJ).
// The reference re-sorts, re-FFTs and re-runs the whole transform (special
// functions included) once per window; here all windows' spectra come from
// one batched FFT launch and the transform of each window reuses the same
// station geometry on the device.
#include <vector>

#include "ccfj_core.cuh"
#include "fj_fft.cuh"
#include "fj_frontend.cuh"

namespace ccfj {

// spec row (w, i) <- TaperSpec of window w and trace row perm[i]
__global__ void taper_spec_kernel(const int* __restrict__ n1, const int* __restrict__ n2,
                                  const int* __restrict__ delta, const long long* __restrict__ perm,
                                  int nwin, int ntr, long long u_rows, TaperSpec* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int w = blockIdx.y;
  if (i >= ntr) return;
  const long long row = perm ? perm[i] : i;
  const long long src = (long long)w * u_rows + row;
  TaperSpec t;
  t.n1 = n1[src];
  t.n2 = n2[src];
  t.delta = delta[src];
  t.pad = 0;
  dst[(long long)w * ntr + i] = t;
}

static int eq_validate(const ccfj_eq_args* a) {
  CCFJ_REQUIRE(a != nullptr, "ccfj_fj_earthquake_v1: args is NULL");
  CCFJ_REQUIRE(a->struct_size == (int)sizeof(ccfj_eq_args),
               "ccfj_fj_earthquake_v1: struct_size %d != %d (header mismatch)", a->struct_size,
               (int)sizeof(ccfj_eq_args));
  CCFJ_REQUIRE(a->ntr >= 1 && a->nf >= 1 && a->nc >= 1 && a->npts >= 2,
               "ccfj_fj_earthquake_v1: ntr=%d nf=%d nc=%d npts=%d", a->ntr, a->nf, a->nc, a->npts);
  CCFJ_REQUIRE(a->itype == 0 || a->itype == 1, "ccfj_fj_earthquake_v1: itype must be 0 or 1");
  CCFJ_REQUIRE(a->func == 0 || a->func == 1, "ccfj_fj_earthquake_v1: func must be 0 or 1");
  CCFJ_REQUIRE(a->precision >= CCFJ_PREC_FP32 && a->precision <= CCFJ_PREC_FP64_PLAIN,
               "ccfj_fj_earthquake_v1: bad precision %d", a->precision);
  CCFJ_REQUIRE(a->fstride >= 1, "ccfj_fj_earthquake_v1: fstride must be >= 1");
  CCFJ_REQUIRE((long long)(a->nf - 1) * a->fstride <= a->npts / 2,
               "ccfj_fj_earthquake_v1: bin %lld beyond the last rfft bin %d",
               (long long)(a->nf - 1) * a->fstride, a->npts / 2);
  CCFJ_REQUIRE(a->u && a->r && a->f && a->c && a->out, "ccfj_fj_earthquake_v1: NULL array");
  CCFJ_REQUIRE(a->u_ld >= a->npts, "ccfj_fj_earthquake_v1: u_ld %lld < npts %d", a->u_ld, a->npts);
  CCFJ_REQUIRE(a->u_rows >= a->ntr, "ccfj_fj_earthquake_v1: u_rows %lld < ntr %d", a->u_rows,
               a->ntr);
  CCFJ_REQUIRE(a->out_f64 == 0 || a->out_f64 == 1, "ccfj_fj_earthquake_v1: out_f64 must be 0 or 1");
  CCFJ_REQUIRE(!(a->out_f64 && a->device_ptrs),
               "ccfj_fj_earthquake_v1: out_f64 needs host pointers (device_ptrs = 0)");
  CCFJ_REQUIRE(a->nwin >= 0, "ccfj_fj_earthquake_v1: nwin must be >= 0");
  CCFJ_REQUIRE(a->nwin == 0 || (a->win_n1 && a->win_n2 && a->win_delta),
               "ccfj_fj_earthquake_v1: nwin > 0 needs win_n1/win_n2/win_delta");
  // one FFT row (and CTA) per (window, trace)
  CCFJ_REQUIRE((long long)(a->nwin > 0 ? a->nwin : 1) * a->ntr <= 0x7fffffffLL,
               "ccfj_fj_earthquake_v1: nwin*ntr = %lld rows exceed 2^31-1",
               (long long)(a->nwin > 0 ? a->nwin : 1) * a->ntr);
  return CCFJ_OK;
}

// All pointers device pointers. call_err: a device word that receives this
// call's timeout flag of the tensor-core path (NULL: scratch of the call).
static int eq_device(const ccfj_eq_args& a, cudaStream_t s, unsigned int* call_err = nullptr) {
  Scratch sc(s);
  const int nw = a.nwin > 0 ? a.nwin : 1;
  const long long rows_out = (long long)nw * a.ntr;
  float2* spec = sc.get_n<float2>((size_t)rows_out * a.nf);
  if (!spec) return CCFJ_ERR_ALLOC;
  TaperSpec* taper = nullptr;
  if (a.nwin > 0) {
    taper = sc.get_n<TaperSpec>((size_t)rows_out);
    if (!taper) return CCFJ_ERR_ALLOC;
    taper_spec_kernel<<<dim3(div_up(a.ntr, 256), a.nwin), 256, 0, s>>>(
        a.win_n1, a.win_n2, a.win_delta, a.perm, a.nwin, a.ntr, a.u_rows, taper);
    count_launch();
    CCFJ_LAUNCH_CHECK("taper_spec_kernel");
  }
  FftJob job{};
  job.u = a.u;
  job.u_ld = a.u_ld;
  job.perm = a.perm;
  job.ntr = a.ntr;
  job.npts = a.npts;
  job.nbins = a.nf;
  job.bin_stride = a.fstride;
  job.taper = taper;
  job.out = spec;
  int st = rfft_bins(job, (int)rows_out, s, sc);
  if (st != CCFJ_OK) return st;

  // MWFJ: all windows share the pairs, so their transforms share the
  // interval moments (one pass over the geometry for a tile of windows).
  if (a.nwin > 0 && a.precision == CCFJ_PREC_FP32) {
    // tensor cores when the window dimension makes the contraction dense
    const bool tc_ok = a.itype == 1 && a.func == 0 && a.ntr >= 2 && a.nwin <= 128;
    const int path = g_mwfj_path.load(std::memory_order_relaxed);
    const bool use_tc = tc_ok && (path >= 2 || (path == 0 && a.nwin >= 8));
    if (use_tc) return mwfj_tensor(a, spec, s, sc, call_err, path != 3);
    return mwfj_cuda_core(a, spec, s, sc);
  }

  // One transform per window over its [ntr][nf] complex spectra: input 0 is
  // the real part, input 1 the imaginary part (element stride 2).
  for (int w = 0; w < nw; ++w) {
    ccfj_fj_args d{};
    d.struct_size = sizeof(d);
    d.nr = a.ntr;
    d.nf = a.nf;
    d.nc = a.nc;
    d.itype = a.itype;
    d.mode = a.func == 0 ? CCFJ_MODE_ABS_J : CCFJ_MODE_ABS_H;
    d.precision = a.precision;
    d.normalize = a.normalize;
    d.device_ptrs = 1;
    const float* base = reinterpret_cast<const float*>(spec + (size_t)w * a.ntr * a.nf);
    d.u[0] = base;
    d.u[1] = base + 1;
    d.u_ld = 2LL * a.nf;
    d.u_rows = a.ntr;
    d.u_es = 2;
    d.u_ncols = a.nf;
    d.fstride = 1;
    d.r = a.r;
    d.f = a.f;
    d.c = a.c;
    d.out = a.out + (size_t)w * a.nc * a.nf;
    d.tau = a.tau;
    st = fj_device(d, s);
    if (st != CCFJ_OK) return st;
  }
  return CCFJ_OK;
}

static int eq_host(const ccfj_eq_args& a, cudaStream_t s) {
  if (a.perm)
    for (int i = 0; i < a.ntr; ++i)
      CCFJ_REQUIRE(a.perm[i] >= 0 && a.perm[i] < a.u_rows,
                   "ccfj_fj_earthquake_v1: perm[%d]=%lld out of range", i, a.perm[i]);
  Scratch sc(s);
  ccfj_eq_args d = a;
  d.device_ptrs = 1;
  d.out_f64 = 0;
  const int nw = a.nwin > 0 ? a.nwin : 1;
  const size_t ubytes = sizeof(float) * ((size_t)(a.u_rows - 1) * a.u_ld + a.npts);
  float* du = static_cast<float*>(sc.get(ubytes));
  float* dr = sc.get_n<float>(a.ntr);
  float* df = sc.get_n<float>(a.nf);
  float* dc = sc.get_n<float>(a.nc);
  float* dout = sc.get_n<float>((size_t)nw * a.nc * a.nf);
  unsigned int* derr = sc.get_n<unsigned int>(1);
  if (!du || !dr || !df || !dc || !dout || !derr) return CCFJ_ERR_ALLOC;
  CCFJ_CUDA_TRY(cudaMemsetAsync(derr, 0, sizeof(unsigned int), s));
  int cst = copy_from_host(du, a.u, ubytes, s);
  if (cst != CCFJ_OK) return cst;
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dr, a.r, sizeof(float) * a.ntr, cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(df, a.f, sizeof(float) * a.nf, cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dc, a.c, sizeof(float) * a.nc, cudaMemcpyHostToDevice, s));
  if (a.perm) {
    long long* dp = sc.get_n<long long>(a.ntr);
    if (!dp) return CCFJ_ERR_ALLOC;
    CCFJ_CUDA_TRY(cudaMemcpyAsync(dp, a.perm, sizeof(long long) * a.ntr, cudaMemcpyHostToDevice, s));
    d.perm = dp;
  }
  if (a.nwin > 0) {
    const size_t nwb = sizeof(int) * (size_t)a.nwin * a.u_rows;
    int* w1 = static_cast<int*>(sc.get(nwb));
    int* w2 = static_cast<int*>(sc.get(nwb));
    int* wd = static_cast<int*>(sc.get(nwb));
    if (!w1 || !w2 || !wd) return CCFJ_ERR_ALLOC;
    CCFJ_CUDA_TRY(cudaMemcpyAsync(w1, a.win_n1, nwb, cudaMemcpyHostToDevice, s));
    CCFJ_CUDA_TRY(cudaMemcpyAsync(w2, a.win_n2, nwb, cudaMemcpyHostToDevice, s));
    CCFJ_CUDA_TRY(cudaMemcpyAsync(wd, a.win_delta, nwb, cudaMemcpyHostToDevice, s));
    d.win_n1 = w1;
    d.win_n2 = w2;
    d.win_delta = wd;
  }
  d.u = du;
  d.r = dr;
  d.f = df;
  d.c = dc;
  d.out = dout;
  int st = eq_device(d, s, derr);
  if (st != CCFJ_OK) return st;
  const size_t nout = (size_t)nw * a.nc * a.nf;
  st = a.out_f64 ? copy_to_host(a.out, dout, nout, 1, s)
                 : copy_to_host(a.out, dout, sizeof(float) * nout, 0, s);
  if (st != CCFJ_OK) return st;
  bool failed = false;
  st = mw_tc_call_error(derr, s, &failed);
  if (st != CCFJ_OK) return st;
  if (failed)
    return set_error(CCFJ_ERR_TIMEOUT, "ccfj_fj_earthquake_v1: a bounded device wait ran out");
  return CCFJ_OK;
}

std::atomic<int> g_mwfj_path{0};

}  // namespace ccfj

CCFJ_API int ccfj_set_mwfj_path(int path) {
  if (path < 0 || path > 3)
    return ccfj::set_error(CCFJ_ERR_INVALID, "ccfj_set_mwfj_path: path must be 0, 1, 2 or 3");
  ccfj::g_mwfj_path.store(path, std::memory_order_relaxed);
  return CCFJ_OK;
}

CCFJ_API int ccfj_device_status(void* stream) {
  ccfj::clear_error();
  bool failed = false;
  const int st = ccfj::mw_tc_sticky_error((cudaStream_t)stream, &failed);
  if (st != CCFJ_OK) return st;
  if (failed) return ccfj::set_error(CCFJ_ERR_TIMEOUT, "a bounded device wait ran out");
  return CCFJ_OK;
}

CCFJ_API int ccfj_fj_earthquake_v1(const ccfj_eq_args* args, void* stream) {
  ccfj::clear_error();
  int st = ccfj::eq_validate(args);
  if (st != CCFJ_OK) return st;
  if (args->device_ptrs) return ccfj::eq_device(*args, (cudaStream_t)stream);
  return ccfj::eq_host(*args, (cudaStream_t)stream);
}
