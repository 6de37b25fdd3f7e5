// Ragged batch: many data sets (subarrays) of uneven pair counts that share
// the frequency and velocity grids, transformed in one persistent launch.
//
// The reference has no batch entry; a user calls fj_noise once per subarray
// (src/ccfj-gpu.pyx:241-268), and each call pays its own allocation, copies
// and launch. Here the pairs of all sets are concatenated (CSR offsets), the
// preparation runs once over all of them, and one persistent kernel with
// one CTA per resident slot pulls work items -- (set, 32 frequencies, 8*CPT
// velocities) -- from a global atomic counter, largest sets first (a
// longest-processing-time order, so the uneven costs even out at the end).
// The counter is only incremented: no thread ever waits on another.
//
// With use_graph, the whole sequence (counter reset, preparation, Hilbert
// transform, persistent kernel, normalisation, and its stream-ordered
// scratch allocations) is captured once per argument set into a CUDA graph
// and replayed on later calls.
#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "batch_plan.h"
#include "fj_cells.cuh"

namespace ccfj {

namespace {

__device__ __forceinline__ int set_of(const long long* __restrict__ off, int nsets, long long i) {
  int lo = 0, hi = nsets;  // off[lo] <= i < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= i)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__global__ void batch_prep_geom_kernel(const float* __restrict__ rs,
                                       const long long* __restrict__ off, int nsets,
                                       long long total, float* __restrict__ drs,
                                       float* __restrict__ wtr, float4* __restrict__ geo) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == total) drs[total] = 0.0f;  // padding read by the one-station lookahead
  if (i >= total) return;
  const int b = set_of(off, nsets, i);
  const long long s = off[b], e = off[b + 1];
  const float r = rs[i];
  const float dl = i > s ? r - rs[i - 1] : 0.0f;
  const float dr = i + 1 < e ? rs[i + 1] - r : 0.0f;
  drs[i] = dl;
  if (geo) geo[i] = station_geometry(r, dr);
  const float w0 = i > s ? fmaxf(dl, 0.1f) : 0.0f;
  const float w1 = i + 1 < e ? fmaxf(dr, 0.1f) : 0.0f;
  wtr[i] = (w0 + w1) * 0.5f * r;
}

// As fj_prep_coef_kernel (itype 1) and fj_prep_u_kernel (itype 0), with
// each set's first and last pair closing its interval chain.
__global__ void batch_prep_u_kernel(InDesc in, const long long* __restrict__ off, int nsets,
                                    long long total, int nf, const float* __restrict__ rs,
                                    const float* __restrict__ drs, const float* __restrict__ wtr,
                                    const float4* __restrict__ geo,
                                    const float* __restrict__ thr, int itype,
                                    void* __restrict__ dst) {
  // rows on grid x (up to 2^31 - 1 blocks), frequencies on grid y
  const int fi = blockIdx.y * blockDim.x + threadIdx.x;
  const long long i = (long long)blockIdx.x * blockDim.y + threadIdx.y;
  if (fi >= nf || i >= total) return;
  const long long col = (long long)fi * in.cs;
  const float g = in.p[(in.perm ? in.perm[i] : i) * in.ld + col];
  if (itype == 1) {
    const int b = set_of(off, nsets, i);
    const bool hl = i > off[b], hr = i + 1 < off[b + 1];
    const float gl = hl ? in.p[(in.perm ? in.perm[i - 1] : i - 1) * in.ld + col] : 0.0f;
    const float gr = hr ? in.p[(in.perm ? in.perm[i + 1] : i + 1) * in.ld + col] : 0.0f;
    static_cast<StationCoef<float>*>(dst)[i * nf + fi] =
        station_coef<float>(g, gl, gr, hl, hr, rs[i], hl ? rs[i - 1] : 0.0f, drs[i],
                            hr ? drs[i + 1] : 0.0f, geo[i].w, thr[fi]);
  } else {
    static_cast<float*>(dst)[i * nf + fi] = g * wtr[i] / geo[i].w;
  }
}

// Sets ordered by pair count, largest first (one CTA; nsets <= 4096).
constexpr int kSortMax = 4096;
__global__ void batch_order_kernel(const long long* __restrict__ off, int nsets,
                                   int* __restrict__ order) {
  __shared__ long long key[kSortMax];
  __shared__ int val[kSortMax];
  int n2 = 1;
  while (n2 < nsets) n2 <<= 1;
  for (int t = threadIdx.x; t < n2; t += blockDim.x) {
    key[t] = t < nsets ? -(off[t + 1] - off[t]) : LLONG_MAX;  // ascending key = descending size
    val[t] = t;
  }
  __syncthreads();
  for (int k = 2; k <= n2; k <<= 1) {       // bitonic sort of (key, val)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < n2; t += blockDim.x) {
        const int p = t ^ j;
        if (p > t) {
          const bool up = (t & k) == 0;
          const bool gt = key[t] > key[p] || (key[t] == key[p] && val[t] > val[p]);
          if (gt == up) {
            const long long tk = key[t];
            key[t] = key[p];
            key[p] = tk;
            const int tv = val[t];
            val[t] = val[p];
            val[p] = tv;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < nsets; t += blockDim.x) order[t] = val[t];
}

__global__ void batch_identity_order_kernel(int nsets, int* __restrict__ order) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nsets) order[t] = t;
}

struct BatchDev {
  FjDev base;                 // shared arrays for all sets; nr unused
  const long long* off;
  const int* order;
  int nsets;
  int ftiles, ctiles;
  long long items;
  unsigned long long* counter;
};

template <int MODE, int ITYPE, int CPT>
__global__ void __launch_bounds__(256, fj_min_blocks<float>()) fj_batch_persistent_kernel(BatchDev bd) {
  __shared__ long long item_s;
  for (;;) {
    if (threadIdx.x == 0 && threadIdx.y == 0) item_s = (long long)atomicAdd(bd.counter, 1ULL);
    __syncthreads();
    const long long item = item_s;
    __syncthreads();  // all threads hold `item` before thread 0 may overwrite item_s
    if (item >= bd.items) break;
    const long long per_set = (long long)bd.ftiles * bd.ctiles;
    const int b = bd.order[item / per_set];
    const int rem = (int)(item % per_set);
    const long long o = bd.off[b];
    FjDev a = bd.base;
    a.nr = (int)(bd.off[b + 1] - o);
    a.i_lo = 0;  // the whole set
    a.i_hi = a.nr;
    a.rs += o;
    a.drs += o;
    a.geo += o;
    constexpr long long esz = ITYPE == 1 ? sizeof(StationCoef<float>) : sizeof(float);
    a.gb[0] = static_cast<const char*>(bd.base.gb[0]) + o * a.nf * esz;
    if (ModeTraits<MODE>::NIN > 1) a.gb[1] = static_cast<const char*>(bd.base.gb[1]) + o * a.nf * esz;
    a.out += (long long)b * a.nc * a.nf;
    // velocity tiles fastest: the items of one frequency tile run side by
    // side and share its station coefficients in L2
    const int fi = (rem / bd.ctiles) * 32 + threadIdx.x;
    const int c0 = ((rem % bd.ctiles) * 8 + threadIdx.y) * CPT;
    fj_cells<MODE, ITYPE, float, CPT>(a, fi, c0);
  }
}

// Per (set, frequency) column normalisation (builtin-max semantics, as
// fj_normalize_kernel), set = blockIdx.y.
__global__ void batch_normalize_kernel(float* __restrict__ out, int nc, int nf) {
  __shared__ float red[8][33];
  __shared__ float colmax[32];
  float* o = out + (long long)blockIdx.y * nc * nf;
  const int fi = blockIdx.x * 32 + threadIdx.x;
  // two running maxima and eight loads in flight per thread (the maximum
  // does not depend on the order)
  float m = -INFINITY, m2 = -INFINITY;
  if (fi < nf) {
#pragma unroll 8
    for (int c = threadIdx.y; c < nc; c += 2 * blockDim.y) {
      m = fmaxf(m, fabsf(o[(long long)c * nf + fi]));
      if (c + (int)blockDim.y < nc) m2 = fmaxf(m2, fabsf(o[(long long)(c + blockDim.y) * nf + fi]));
    }
  }
  m = fmaxf(m, m2);
  red[threadIdx.y][threadIdx.x] = m;
  __syncthreads();
  if (threadIdx.y == 0) {
    for (int y = 1; y < (int)blockDim.y; ++y) m = fmaxf(m, red[y][threadIdx.x]);
    if (fi < nf) {
      const float first = fabsf(o[fi]);
      colmax[threadIdx.x] = isnan(first) ? first : m;
    }
  }
  __syncthreads();
  if (fi < nf) {
    const float dv = colmax[threadIdx.x];
#pragma unroll 8
    for (int c = threadIdx.y; c < nc; c += blockDim.y) {
      const long long k = (long long)c * nf + fi;
      o[k] = o[k] / dv;
    }
  }
}

int nin_of_mode(int mode) { return (mode == CCFJ_MODE_J || mode == CCFJ_MODE_Y) ? 1 : 2; }

template <int MODE, int CPT>
void launch_batch_cpt(int itype, const BatchDev& bd, int grid, cudaStream_t s) {
  if (itype == 1)
    fj_batch_persistent_kernel<MODE, 1, CPT><<<grid, dim3(32, 8), 0, s>>>(bd);
  else
    fj_batch_persistent_kernel<MODE, 0, CPT><<<grid, dim3(32, 8), 0, s>>>(bd);
}

template <int MODE>
int launch_batch(int itype, int cpt, BatchDev bd, cudaStream_t s) {
  int dev = 0, sms = 0, per_sm = 0;
  CCFJ_CUDA_TRY(cudaGetDevice(&dev));
  CCFJ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const void* fn = nullptr;
#define CCFJ_PICK(C)                                                                           \
  fn = itype == 1 ? (const void*)fj_batch_persistent_kernel<MODE, 1, C>                        \
                  : (const void*)fj_batch_persistent_kernel<MODE, 0, C>
  if (cpt == 1)
    CCFJ_PICK(1);
  else if (cpt == 4)
    CCFJ_PICK(4);
  else
    CCFJ_PICK(2);
#undef CCFJ_PICK
  CCFJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0));
  const long long slots = (long long)sms * (per_sm > 0 ? per_sm : 1);
  const int grid = (int)(bd.items < slots ? bd.items : slots);
  if (cpt == 1)
    launch_batch_cpt<MODE, 1>(itype, bd, grid, s);
  else if (cpt == 4)
    launch_batch_cpt<MODE, 4>(itype, bd, grid, s);
  else
    launch_batch_cpt<MODE, 2>(itype, bd, grid, s);
  return CCFJ_OK;
}

int batch_validate(const ccfj_batch_args* a) {
  CCFJ_REQUIRE(a != nullptr, "ccfj_fj_batch_v1: args is NULL");
  CCFJ_REQUIRE(a->struct_size == (int)sizeof(ccfj_batch_args),
               "ccfj_fj_batch_v1: struct_size %d != %d (header mismatch)", a->struct_size,
               (int)sizeof(ccfj_batch_args));
  CCFJ_REQUIRE(a->nsets >= 1 && a->nf >= 1 && a->nc >= 1,
               "ccfj_fj_batch_v1: nsets=%d nf=%d nc=%d must be >= 1", a->nsets, a->nf, a->nc);
  CCFJ_REQUIRE(a->nsets <= 65535, "ccfj_fj_batch_v1: nsets=%d > 65535", a->nsets);
  CCFJ_REQUIRE(a->itype == 0 || a->itype == 1, "ccfj_fj_batch_v1: itype must be 0 or 1");
  CCFJ_REQUIRE(a->mode >= CCFJ_MODE_J && a->mode <= CCFJ_MODE_ABS_H, "ccfj_fj_batch_v1: bad mode");
  CCFJ_REQUIRE(a->precision == CCFJ_PREC_FP32, "ccfj_fj_batch_v1: only CCFJ_PREC_FP32");
  CCFJ_REQUIRE(a->variant == 0 || a->variant == 1 || a->variant == 2 || a->variant == 4,
               "ccfj_fj_batch_v1: variant must be 0, 1, 2 or 4");
  CCFJ_REQUIRE(a->offsets && a->r && a->f && a->c && a->out && a->u[0],
               "ccfj_fj_batch_v1: NULL array");
  CCFJ_REQUIRE(a->fstride >= 1 && a->u_es >= 1 && a->u_ld >= 1, "ccfj_fj_batch_v1: bad layout");
  CCFJ_REQUIRE(a->u_ncols >= 1 && (a->u_ncols + a->fstride - 1) / a->fstride == a->nf,
               "ccfj_fj_batch_v1: %d columns with fstride %d do not give nf=%d", a->u_ncols,
               a->fstride, a->nf);
  CCFJ_REQUIRE(a->u_ld >= (long long)(a->u_ncols - 1) * a->u_es + 1, "ccfj_fj_batch_v1: u_ld too small");
  if (a->hilbert)
    CCFJ_REQUIRE(a->mode == CCFJ_MODE_J_MINUS_Y && a->u[1] == nullptr,
                 "ccfj_fj_batch_v1: hilbert=1 needs mode J_MINUS_Y and u[1] == NULL");
  else
    CCFJ_REQUIRE(nin_of_mode(a->mode) == 1 || a->u[1], "ccfj_fj_batch_v1: mode needs two inputs");
  return CCFJ_OK;
}

// Velocities per thread of the persistent kernel per batch class (mode,
// itype and the powers of two of the total pairs, sets, nf and nc), as
// recorded by ccfj_autotune_batch_v1; variant 0 uses it, else the untuned
// per-mode default.

long long batch_tune_key(const ccfj_batch_args& a, long long total) {
  auto lg = [](long long v) {
    int b = 0;
    while ((1LL << (b + 1)) <= v) ++b;
    return (long long)b;
  };
  return (((((long long)a.mode * 2 + a.itype) * 64 + lg(total)) * 64 + lg(a.nsets)) * 64 +
          lg(a.nf)) * 64 + lg(a.nc);
}

int batch_variant(const ccfj_batch_args& a, long long total) {
  if (a.variant > 0) return a.variant;
  int choice = 0;
  return tune_lookup("batch", batch_tune_key(a, total), &choice) ? choice
                                                                  : default_cpt_for(a.mode, a.itype);
}

// The device sequence of one batch (all pointers device pointers;
// `total` = offsets[nsets], known to the caller).
int batch_device(const ccfj_batch_args& a, long long total, cudaStream_t s) {
  Scratch sc(s);
  const int nin = nin_of_mode(a.mode);
  float* drs = sc.get_n<float>(total + 1);
  float* wtr = sc.get_n<float>(total);
  float4* geo = sc.get_n<float4>(total);
  int* order = sc.get_n<int>(a.nsets);
  unsigned long long* counter = sc.get_n<unsigned long long>(1);
  if (!drs || !wtr || !order || !counter || !geo) return CCFJ_ERR_ALLOC;
  CCFJ_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
  if (a.nsets <= kSortMax)
    batch_order_kernel<<<1, 1024, 0, s>>>(a.offsets, a.nsets, order);
  else
    batch_identity_order_kernel<<<div_up(a.nsets, 256), 256, 0, s>>>(a.nsets, order);
  count_launch();
  CCFJ_LAUNCH_CHECK("batch_order_kernel");
  batch_prep_geom_kernel<<<div_up(total + 1, 256), 256, 0, s>>>(a.r, a.offsets, a.nsets, total, drs,
                                                             wtr, geo);
  count_launch();
  CCFJ_LAUNCH_CHECK("batch_prep_geom_kernel");

  InDesc in[2];
  for (int j = 0; j < 2; ++j) in[j] = InDesc{a.u[j], a.u_ld, (long long)a.u_es * a.fstride, a.perm};
  if (a.hilbert) {
    float* hb = sc.get_n<float>((size_t)total * a.nf);
    if (!hb) return CCFJ_ERR_ALLOC;
    CCFJ_REQUIRE(total <= INT_MAX, "ccfj_fj_batch_v1: too many pairs for the Hilbert transform");
    const int st = hilbert_rows(InDesc{a.u[0], a.u_ld, a.u_es, a.perm}, a.u_ncols, a.u_es,
                                (int)total, a.nf, a.fstride, 0, hb, s, sc);
    if (st != CCFJ_OK) return st;
    in[1] = InDesc{hb, a.nf, 1, nullptr};
  }
  BatchDev bd{};
  const float tau = a.tau > 0 ? a.tau : kDefaultTau32;
  float* kb = nullptr;
  if (a.itype == 1) {
    kb = sc.get_n<float>(a.nf);
    if (!kb) return CCFJ_ERR_ALLOC;
    fj_kbounds_kernel<float><<<div_up(a.nf, 8), dim3(32, 8), 0, s>>>(a.f, a.c, a.nf, a.nc, tau, kb);
    count_launch();
    CCFJ_LAUNCH_CHECK("fj_kbounds_kernel");
  }
  const size_t esz = a.itype == 1 ? sizeof(StationCoef<float>) : 4;
  for (int j = 0; j < nin; ++j) {
    void* g = sc.get((size_t)total * a.nf * esz);
    if (!g) return CCFJ_ERR_ALLOC;
    batch_prep_u_kernel<<<dim3(div_up(total, 8), div_up(a.nf, 32)), dim3(32, 8), 0, s>>>(
        in[j], a.offsets, a.nsets, total, a.nf, a.r, drs, wtr, geo, kb, a.itype, g);
    count_launch();
    CCFJ_LAUNCH_CHECK("batch_prep_u_kernel");
    bd.base.gb[j] = g;
  }
  bd.base.kb = kb;
  bd.base.geo = geo;
  bd.base.rs = a.r;
  bd.base.drs = drs;
  bd.base.f = a.f;
  bd.base.c = a.c;
  bd.base.out = a.out;
  bd.base.nf = a.nf;
  bd.base.nc = a.nc;
  bd.base.tau = tau;
  bd.off = a.offsets;
  bd.order = order;
  bd.nsets = a.nsets;
  const int cpt = batch_variant(a, total);
  bd.ftiles = div_up(a.nf, 32);
  bd.ctiles = div_up(a.nc, 8 * cpt);
  bd.items = (long long)a.nsets * bd.ftiles * bd.ctiles;
  bd.counter = counter;
  int st = CCFJ_OK;
  switch (a.mode) {
    case CCFJ_MODE_J: st = launch_batch<CCFJ_MODE_J>(a.itype, cpt, bd, s); break;
    case CCFJ_MODE_Y: st = launch_batch<CCFJ_MODE_Y>(a.itype, cpt, bd, s); break;
    case CCFJ_MODE_J_MINUS_Y: st = launch_batch<CCFJ_MODE_J_MINUS_Y>(a.itype, cpt, bd, s); break;
    case CCFJ_MODE_ABS_J: st = launch_batch<CCFJ_MODE_ABS_J>(a.itype, cpt, bd, s); break;
    default: st = launch_batch<CCFJ_MODE_ABS_H>(a.itype, cpt, bd, s); break;
  }
  if (st != CCFJ_OK) return st;
  count_launch();
  CCFJ_LAUNCH_CHECK("fj_batch_persistent_kernel");
  if (a.normalize) {
    batch_normalize_kernel<<<dim3(div_up(a.nf, 32), a.nsets), dim3(32, 8), 0, s>>>(a.out, a.nc,
                                                                                   a.nf);
    count_launch();
    CCFJ_LAUNCH_CHECK("batch_normalize_kernel");
  }
  return CCFJ_OK;
}

// ---------------------------------------------------------- graph cache
// At most kMaxGraphs instantiated graphs are kept (each may hold the device
// memory of its captured scratch allocations); capturing one more destroys
// the least recently launched (a graph still running is freed when it ends).
constexpr size_t kMaxGraphs = 16;
struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
  unsigned long long last_use = 0;
};
std::mutex g_graph_mu;
std::map<std::string, GraphEntry> g_graphs;
unsigned long long g_graph_clock = 0;
cudaStream_t g_capture_stream[64] = {};
// per device: stream 0 -> library stream, library stream -> stream 0
// (used under g_graph_mu)
cudaEvent_t g_order_event[64][2] = {};

template <typename T>
void key_put(std::string& k, const T& v) {
  k.append(reinterpret_cast<const char*>(&v), sizeof(v));
}

// Every field of the arguments (not the struct's bytes: its padding is not
// ours to read), the total pair count and the device.
std::string graph_key(const ccfj_batch_args& a, long long total) {
  std::string k;
  k.reserve(192);
  key_put(k, a.struct_size);
  key_put(k, a.nsets);
  key_put(k, a.nf);
  key_put(k, a.nc);
  key_put(k, a.itype);
  key_put(k, a.mode);
  key_put(k, a.precision);
  key_put(k, a.normalize);
  key_put(k, a.device_ptrs);
  key_put(k, a.hilbert);
  key_put(k, a.use_graph);
  key_put(k, a.variant);
  key_put(k, a.offsets);
  key_put(k, a.total_pairs);
  key_put(k, a.r);
  key_put(k, a.u[0]);
  key_put(k, a.u[1]);
  key_put(k, a.u_ld);
  key_put(k, a.u_rows);
  key_put(k, a.u_es);
  key_put(k, a.u_ncols);
  key_put(k, a.fstride);
  key_put(k, a.perm);
  key_put(k, a.f);
  key_put(k, a.c);
  key_put(k, a.out);
  key_put(k, a.tau);
  key_put(k, total);
  key_put(k, batch_variant(a, total));  // a tuning recorded later gives a new graph
  int dev = 0;
  cudaGetDevice(&dev);
  key_put(k, dev);
  return k;
}

void evict_oldest_graph() {
  auto oldest = g_graphs.begin();
  for (auto it = g_graphs.begin(); it != g_graphs.end(); ++it)
    if (it->second.last_use < oldest->second.last_use) oldest = it;
  if (oldest->second.exec) cudaGraphExecDestroy(oldest->second.exec);
  g_graphs.erase(oldest);
}

int batch_device_graph(const ccfj_batch_args& a, long long total, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (s) CCFJ_CUDA_TRY(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) return batch_device(a, total, s);  // caller's capture
  const std::string key = graph_key(a, total);
  std::lock_guard<std::mutex> lk(g_graph_mu);
  auto it = g_graphs.find(key);
  if (it == g_graphs.end()) {
    int dev = 0;
    CCFJ_CUDA_TRY(cudaGetDevice(&dev));
    CCFJ_REQUIRE(dev >= 0 && dev < 64, "ccfj_fj_batch_v1: device ordinal %d", dev);
    cudaStream_t cap = s;
    if (!cap) {  // the legacy default stream cannot be captured
      if (!g_capture_stream[dev])
        CCFJ_CUDA_TRY(cudaStreamCreateWithFlags(&g_capture_stream[dev], cudaStreamNonBlocking));
      cap = g_capture_stream[dev];
    }
    cudaGraph_t graph = nullptr;
    CCFJ_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    const int st = batch_device(a, total, cap);
    const cudaError_t e = cudaStreamEndCapture(cap, &graph);
    if (st != CCFJ_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (e != cudaSuccess)
      return set_error(CCFJ_ERR_CUDA, "ccfj_fj_batch_v1: graph capture failed: %s",
                       cudaGetErrorString(e));
    GraphEntry ge;
    const cudaError_t ei = cudaGraphInstantiate(&ge.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess)
      return set_error(CCFJ_ERR_CUDA, "ccfj_fj_batch_v1: graph instantiation failed: %s",
                       cudaGetErrorString(ei));
    if (g_graphs.size() >= kMaxGraphs) evict_oldest_graph();
    it = g_graphs.emplace(key, ge).first;
  }
  it->second.last_use = ++g_graph_clock;
  if (s) {
    CCFJ_CUDA_TRY(cudaGraphLaunch(it->second.exec, s));
  } else {
    // The legacy default stream cannot launch a captured graph's work in
    // order by itself, and the library stream is non-blocking: order the
    // launch after the caller's earlier default-stream work, and the
    // caller's later default-stream work after the launch, with events (no
    // host synchronisation), as a kernel launched on stream 0 would be.
    int dev = 0;
    CCFJ_CUDA_TRY(cudaGetDevice(&dev));
    cudaStream_t cap = g_capture_stream[dev];
    if (!g_order_event[dev][0]) {
      CCFJ_CUDA_TRY(cudaEventCreateWithFlags(&g_order_event[dev][0], cudaEventDisableTiming));
      CCFJ_CUDA_TRY(cudaEventCreateWithFlags(&g_order_event[dev][1], cudaEventDisableTiming));
    }
    CCFJ_CUDA_TRY(cudaEventRecord(g_order_event[dev][0], 0));
    CCFJ_CUDA_TRY(cudaStreamWaitEvent(cap, g_order_event[dev][0], 0));
    CCFJ_CUDA_TRY(cudaGraphLaunch(it->second.exec, cap));
    CCFJ_CUDA_TRY(cudaEventRecord(g_order_event[dev][1], cap));
    CCFJ_CUDA_TRY(cudaStreamWaitEvent(0, g_order_event[dev][1], 0));
  }
  count_launch();
  return CCFJ_OK;
}

int batch_run_device(const ccfj_batch_args& a, long long total, cudaStream_t s) {
  if (a.use_graph && !allocator_hooked()) return batch_device_graph(a, total, s);
  return batch_device(a, total, s);
}

// ------------------------------------------------- host-memory batches
// Large host batches run in groups of sets (batch_plan.h).
std::vector<SetGroup> plan_groups(const ccfj_batch_args& a, long long total, int nin,
                                  size_t ubytes) {
  return plan_set_groups(a.offsets, a.nsets, a.perm, total, nin, ubytes);
}

// The copy stream of a pipelined batch and its events; waits for every copy
// before anything it wrote into is freed (it is declared after the call's
// Scratch, so it goes first).
struct CopyLane {
  cudaStream_t cs = nullptr;
  std::vector<cudaEvent_t> ev;
  ~CopyLane() {
    if (cs) {
      cudaStreamSynchronize(cs);
      cudaStreamDestroy(cs);
    }
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
};

int batch_host(const ccfj_batch_args& a, cudaStream_t s) {
  const long long* off = a.offsets;
  CCFJ_REQUIRE(off[0] == 0, "ccfj_fj_batch_v1: offsets[0] must be 0");
  for (int b = 0; b < a.nsets; ++b)
    CCFJ_REQUIRE(off[b + 1] > off[b], "ccfj_fj_batch_v1: set %d is empty or offsets decrease", b);
  const long long total = off[a.nsets];
  CCFJ_REQUIRE(a.total_pairs == 0 || a.total_pairs == total,
               "ccfj_fj_batch_v1: total_pairs %lld != offsets[nsets] %lld", a.total_pairs, total);
  CCFJ_REQUIRE(a.u_rows >= total || a.perm, "ccfj_fj_batch_v1: u_rows < total pairs");
  if (a.perm)
    for (long long i = 0; i < total; ++i)
      CCFJ_REQUIRE(a.perm[i] >= 0 && a.perm[i] < a.u_rows, "ccfj_fj_batch_v1: perm[%lld] out of range",
                   i);
  const int nin = a.hilbert ? 1 : nin_of_mode(a.mode);
  const long long span = (a.u_rows - 1) * a.u_ld + (long long)(a.u_ncols - 1) * a.u_es + 1;
  const float* lo = a.u[0];
  const float* hi = a.u[0] + span;
  if (nin == 2) {
    lo = std::min(lo, a.u[1]);
    hi = std::max(hi, a.u[1] + span);
  }
  CCFJ_REQUIRE(nin == 1 || (size_t)(hi - lo) <= (size_t)(2 * span + 16),
               "ccfj_fj_batch_v1: host mode needs both inputs in one array (real/imaginary parts)");
  const size_t ubytes = sizeof(float) * (size_t)(hi - lo);
  const std::vector<SetGroup> groups = plan_groups(a, total, nin, ubytes);
  const int ng = (int)groups.size();
  Scratch sc(s);
  float* du = sc.get_n<float>(hi - lo);
  // the batch's offsets, then (pipelined) each group's rebased offsets
  long long* doff = sc.get_n<long long>(a.nsets + 1 + (ng > 0 ? a.nsets + ng : 0));
  float* dr = sc.get_n<float>(total);
  float* df = sc.get_n<float>(a.nf);
  float* dc = sc.get_n<float>(a.nc);
  float* dout = sc.get_n<float>((size_t)a.nsets * a.nc * a.nf);
  long long* dp = a.perm ? sc.get_n<long long>(total) : nullptr;
  if (!du || !doff || !dr || !df || !dc || !dout || (a.perm && !dp)) return CCFJ_ERR_ALLOC;
  if (ng == 0) {
    const int cst = copy_from_host(du, lo, ubytes, s);
    if (cst != CCFJ_OK) return cst;
  }
  CCFJ_CUDA_TRY(cudaMemcpyAsync(doff, off, sizeof(long long) * (a.nsets + 1), cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dr, a.r, sizeof(float) * total, cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(df, a.f, sizeof(float) * a.nf, cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dc, a.c, sizeof(float) * a.nc, cudaMemcpyHostToDevice, s));
  if (dp) CCFJ_CUDA_TRY(cudaMemcpyAsync(dp, a.perm, sizeof(long long) * total, cudaMemcpyHostToDevice, s));
  ccfj_batch_args d = a;
  d.device_ptrs = 1;
  d.use_graph = 0;  // per-call buffers: nothing to replay
  for (int j = 0; j < nin; ++j) d.u[j] = du + (a.u[j] - lo);
  d.offsets = doff;
  d.r = dr;
  d.f = df;
  d.c = dc;
  d.out = dout;
  d.perm = dp;
  const size_t out_bytes = sizeof(float) * a.nsets * a.nc * a.nf;
  if (ng == 0) {
    const int st = batch_device(d, total, s);
    if (st != CCFJ_OK) return st;
    return copy_to_host(a.out, dout, out_bytes, 0, s);
  }

  // Pipelined: each group's offsets rebased to its first pair (one copy for
  // all groups, after the whole batch's), its rows of u on the copy stream.
  std::vector<long long> goff;
  goff.reserve(a.nsets + ng);
  for (const SetGroup& g : groups)
    for (int b = g.b0; b <= g.b1; ++b) goff.push_back(off[b] - off[g.b0]);
  long long* dgoff = doff + a.nsets + 1;
  CCFJ_CUDA_TRY(cudaMemcpyAsync(dgoff, goff.data(), sizeof(long long) * goff.size(),
                                cudaMemcpyHostToDevice, s));
  // goff may go, and the scratch allocated on s may be used on the copy stream
  CCFJ_CUDA_TRY(cudaStreamSynchronize(s));
  CopyLane lane;
  CCFJ_CUDA_TRY(cudaStreamCreateWithFlags(&lane.cs, cudaStreamNonBlocking));
  lane.ev.assign(ng, nullptr);
  for (cudaEvent_t& e : lane.ev) CCFJ_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  auto copy_group = [&](int g) -> int {
    const long long f0 = groups[g].row_lo * a.u_ld;
    const long long f1 = groups[g].row_hi * a.u_ld + (long long)(a.u_ncols - 1) * a.u_es + 1;
    CCFJ_CUDA_TRY(cudaMemcpyAsync(du + f0, lo + f0, sizeof(float) * (f1 - f0),
                                  cudaMemcpyHostToDevice, lane.cs));
    CCFJ_CUDA_TRY(cudaEventRecord(lane.ev[g], lane.cs));
    return CCFJ_OK;
  };
  int st = copy_group(0);
  if (st != CCFJ_OK) return st;
  const int variant = batch_variant(a, total);  // the whole batch's choice for every group
  long long slot = 0;
  for (int g = 0; g < ng; ++g) {
    const SetGroup& G = groups[g];
    ccfj_batch_args dg = d;
    dg.nsets = G.b1 - G.b0;
    dg.offsets = dgoff + slot;
    slot += dg.nsets + 1;
    dg.total_pairs = off[G.b1] - off[G.b0];
    dg.r = dr + off[G.b0];
    dg.perm = dp ? dp + off[G.b0] : nullptr;
    if (!dp) dg.u[0] = d.u[0] + off[G.b0] * a.u_ld;  // rows are pair indices
    dg.out = dout + (size_t)G.b0 * a.nc * a.nf;
    dg.variant = variant;
    CCFJ_CUDA_TRY(cudaStreamWaitEvent(s, lane.ev[g], 0));
    st = batch_device(dg, dg.total_pairs, s);
    if (st != CCFJ_OK) return st;
    if (g + 1 < ng && (st = copy_group(g + 1)) != CCFJ_OK) return st;
  }
  return copy_to_host(a.out, dout, out_bytes, 0, s);
}

}  // namespace

int normalize_sets(float* out, int nsets, int nc, int nf, cudaStream_t s) {
  CCFJ_REQUIRE(nsets <= 65535, "normalisation of %d sets (> 65535)", nsets);
  batch_normalize_kernel<<<dim3(div_up(nf, 32), nsets), dim3(32, 8), 0, s>>>(out, nc, nf);
  count_launch();
  CCFJ_LAUNCH_CHECK("batch_normalize_kernel");
  return CCFJ_OK;
}

}  // namespace ccfj

CCFJ_API int ccfj_fj_batch_v1(const ccfj_batch_args* args, void* stream) {
  ccfj::clear_error();
  int st = ccfj::batch_validate(args);
  if (st != CCFJ_OK) return st;
  if (!args->device_ptrs) return ccfj::batch_host(*args, (cudaStream_t)stream);
  CCFJ_REQUIRE(args->total_pairs >= args->nsets,
               "ccfj_fj_batch_v1: device mode needs total_pairs (= offsets[nsets])");
  return ccfj::batch_run_device(*args, args->total_pairs, (cudaStream_t)stream);
}

CCFJ_API int ccfj_autotune_batch_v1(const ccfj_batch_args* args, void* stream, int* best_variant,
                                    float* best_ms) {
  ccfj::clear_error();
  int st = ccfj::batch_validate(args);
  if (st != CCFJ_OK) return st;
  CCFJ_REQUIRE(args->device_ptrs, "ccfj_autotune_batch_v1: needs device pointers");
  CCFJ_REQUIRE(args->total_pairs >= args->nsets,
               "ccfj_autotune_batch_v1: needs total_pairs (= offsets[nsets])");
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return ccfj::set_error(CCFJ_ERR_CUDA, "ccfj_autotune_batch_v1: cudaEventCreate failed: %s",
                           cudaGetErrorString(cudaGetLastError()));
  }
  const int cands[3] = {1, 2, 4};
  int best = 0;
  float best_t = 1e30f;
  for (int c : cands) {
    ccfj_batch_args d = *args;
    d.variant = c;
    d.use_graph = 0;
    float t = 1e30f;
    for (int rep = 0; rep < 3 && st == CCFJ_OK; ++rep) {
      cudaEventRecord(e0, s);
      st = ccfj::batch_device(d, args->total_pairs, s);
      cudaEventRecord(e1, s);
      const cudaError_t e = cudaEventSynchronize(e1);
      if (st == CCFJ_OK && e != cudaSuccess)
        st = ccfj::set_error(CCFJ_ERR_CUDA, "ccfj_autotune_batch_v1: %s", cudaGetErrorString(e));
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) t = std::min(t, ms);  // the first run is a warm-up
    }
    if (st != CCFJ_OK) break;
    if (t < best_t) {
      best_t = t;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != CCFJ_OK) return st;
  st = ccfj::tune_record("batch", ccfj::batch_tune_key(*args, args->total_pairs), best, best_t);
  if (best_variant) *best_variant = best;
  if (best_ms) *best_ms = best_t;
  return st;
}

CCFJ_API int ccfj_batch_graph_cache_clear(void) {
  std::lock_guard<std::mutex> lk(ccfj::g_graph_mu);
  for (auto& kv : ccfj::g_graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  ccfj::g_graphs.clear();
  return CCFJ_OK;
}
