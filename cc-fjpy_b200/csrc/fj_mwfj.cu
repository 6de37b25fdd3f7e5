// MWFJ with the station geometry shared by all windows.
//
// The reference (src/ccfj-gpu.pyx:297-313) calls fj_earthquake once per
// window, re-sorting, re-FFTing and re-evaluating every special function for
// every window. All windows of one call share the pairs and their
// distances, so here the per-(f, c, interval) moments I0, I1 -- the
// expensive part -- are computed once per window tile and contracted with
// the interval data of every window in it:
//
//   out_w(c, f) = | sum_i [g_{i-1,w} I0_i + b_{i,w} I1_i / k] (Re)
//                 + i sum_i [...] (Im) | / k^2
//
// i.e. a contraction over K = 2 (nr - 1) of the per-(c, f) moment vector with
// the per-f matrix [g, b] x (Re, Im of every window). This file is the
// CUDA-core form: each thread keeps the accumulators of NWT windows (both
// parts) of one (f, c) cell, so a station's special functions are shared by
// NWT windows; the window tiles are the grid's z dimension. A warp spans 32
// velocities of one frequency, so the window data of a station is one
// warp-uniform 16*NWT-byte segment (broadcast loads), prefetched a few
// stations ahead.
#include "fj_cells.cuh"
#include "fj_fft.cuh"

namespace ccfj {

struct MwDev {
  const float* rs;
  const float* drs;
  const void* gb;  // [nr][nf][2 nwin]: float2 (g_{i-1}, b_i) for itype 1, float g*w for itype 0
  const float* f;
  const float* c;
  float* out;  // [nwin][nc][nf]
  int nr, nf, nc, nwin;
  float tau;
};

// Interval data of every window from the FFT output spec[w][i][f] (complex):
// dst[(i nf + f) 2 nwin + 2 w + part], part 0 = real, 1 = imaginary. A block
// stages a 32-frequency x 8-window tile in shared memory so that both the
// reads (along f) and the writes (along w) are contiguous.
__global__ void mw_prep_kernel(const float2* __restrict__ spec, int ntr, int nf, int nwin,
                               const float* __restrict__ drs, const float* __restrict__ wtr,
                               int itype, void* __restrict__ dst) {
  __shared__ float2 cur[8][33];
  __shared__ float2 prv[8][33];
  const int i = blockIdx.x;
  const int f0 = blockIdx.y * 32;
  const int w0 = blockIdx.z * 8;
  const int w = w0 + threadIdx.y;
  const int fi = f0 + threadIdx.x;
  if (w < nwin && fi < nf) {
    cur[threadIdx.y][threadIdx.x] = spec[((long long)w * ntr + i) * nf + fi];
    prv[threadIdx.y][threadIdx.x] =
        i > 0 ? spec[((long long)w * ntr + i - 1) * nf + fi] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float dr0 = i > 0 ? fmaxf(drs[i], 0.1f) : 1.0f;
  const float wt = wtr[i];
  const int nw2 = 2 * nwin;
  // 32 f x 8 w x 2 parts = 512 outputs, two per thread, part fastest
  for (int t = threadIdx.y * 32 + threadIdx.x; t < 512; t += 256) {
    const int p = t & 1;
    const int wl = (t >> 1) & 7;
    const int fl = t >> 4;
    if (w0 + wl >= nwin || f0 + fl >= nf) continue;
    const float g = p ? cur[wl][fl].y : cur[wl][fl].x;
    const long long o = ((long long)i * nf + f0 + fl) * nw2 + 2 * (w0 + wl) + p;
    if (itype == 1) {
      const float gp = p ? prv[wl][fl].y : prv[wl][fl].x;
      static_cast<float2*>(dst)[o] = i > 0 ? make_float2(gp, (g - gp) / dr0) : make_float2(0.f, 0.f);
    } else {
      static_cast<float*>(dst)[o] = g * wt;
    }
  }
}

constexpr int kMwPrefetch = 4;  // stations ahead

template <int FUNC, int ITYPE, int NWT>
__global__ void __launch_bounds__(256) fj_mw_kernel(MwDev a) {
  constexpr bool WJ = true, WY = FUNC == 1;
  const int ci = blockIdx.x * 32 + threadIdx.x;
  const int fi = blockIdx.y * 8 + threadIdx.y;
  const int w0 = blockIdx.z * NWT;
  if (fi >= a.nf || ci >= a.nc) return;
  Cell<float> cell;
  cell.init(a.f[fi], a.c[ci]);
  const int nw2 = 2 * a.nwin;
  // clamp the window index of a partial last tile (results not stored)
  int wsel[NWT];
#pragma unroll
  for (int w = 0; w < NWT; ++w) wsel[w] = min(w0 + w, a.nwin - 1);
  float tot[NWT][2], acc[NWT][2];
#pragma unroll
  for (int w = 0; w < NWT; ++w) tot[w][0] = tot[w][1] = 0.f;
  ZB<float> Jz{}, Yz{};
  if (ITYPE == 1) {
    const float tau = a.tau;
    Station<float> sJp, sYp;
    float xp = cell.k * __ldg(a.rs);
    float dr_next = __ldg(a.drs + 1);  // drs has nr + 1 entries, the last 0
    cell.eval<WJ, WY, true>(__ldg(a.rs), xp, closed_form<float, WY>(cell.k * dr_next, xp, tau),
                            Jz, Yz);
    sJp = fjs::make_station(xp, Jz);
    if (WY) sYp = fjs::make_station(xp, Yz);
    bool lnJ = closed_form<float, false>(cell.k * dr_next, xp, tau);
    bool lnY = closed_form<float, true>(cell.k * dr_next, xp, tau);
    for (int i0 = 1; i0 < a.nr; i0 += kChunk) {
      const int i1 = min(a.nr, i0 + kChunk);
#pragma unroll
      for (int w = 0; w < NWT; ++w) acc[w][0] = acc[w][1] = 0.f;
      for (int i = i0; i < i1; ++i) {
        const float r = __ldg(a.rs + i);
        const float dr = dr_next;
        dr_next = __ldg(a.drs + i + 1);
        const float x = cell.k * r;
        const float dx = cell.k * dr;
        const bool lcJ = lnJ, lcY = lnY;
        const float dxn = cell.k * dr_next;
        lnJ = closed_form<float, false>(dxn, x, tau);
        if (WY) lnY = closed_form<float, true>(dxn, x, tau);
        cell.eval<WJ, WY, true>(r, x, WY ? (lcY || lnY) : (lcJ || lnJ), Jz, Yz);
        float I0J, I1J, I0Y = 0.f, I1Y = 0.f;
        const Station<float> sJ = fjs::make_station(x, Jz);
        fjs::interval_moments<float>(sJp, sJ, dx, lcJ, I0J, I1J);
        sJp = sJ;
        if (WY) {
          const Station<float> sY = fjs::make_station(x, Yz);
          fjs::interval_moments<float>(sYp, sY, dx, lcY, I0Y, I1Y);
          sYp = sY;
        }
        I1J *= cell.inv_k;
        I1Y *= cell.inv_k;
        const float2* g = static_cast<const float2*>(a.gb) + ((long long)i * a.nf + fi) * nw2;
        if (i + kMwPrefetch < a.nr)
          asm volatile("prefetch.global.L1 [%0];" ::"l"(g + (long long)kMwPrefetch * a.nf * nw2 +
                                                        2 * w0));
#pragma unroll
        for (int w = 0; w < NWT; ++w) {
          const float4 v = __ldg(reinterpret_cast<const float4*>(g + 2 * wsel[w]));
          // v = (g_re, b_re, g_im, b_im)
          const float jr = fmaf(v.x, I0J, v.y * I1J), ji = fmaf(v.z, I0J, v.w * I1J);
          if (FUNC == 0) {
            acc[w][0] += jr;
            acc[w][1] += ji;
          } else {
            const float yr = fmaf(v.x, I0Y, v.y * I1Y), yi = fmaf(v.z, I0Y, v.w * I1Y);
            acc[w][0] += jr - yi;
            acc[w][1] += ji + yr;
          }
        }
        xp = x;
      }
#pragma unroll
      for (int w = 0; w < NWT; ++w) {
        tot[w][0] += acc[w][0];
        tot[w][1] += acc[w][1];
      }
    }
#pragma unroll
    for (int w = 0; w < NWT; ++w) {
      tot[w][0] *= cell.inv_k2;
      tot[w][1] *= cell.inv_k2;
    }
  } else {
    for (int i0 = 0; i0 < a.nr; i0 += kChunk) {
      const int i1 = min(a.nr, i0 + kChunk);
#pragma unroll
      for (int w = 0; w < NWT; ++w) acc[w][0] = acc[w][1] = 0.f;
      for (int i = i0; i < i1; ++i) {
        const float r = __ldg(a.rs + i);
        cell.eval<WJ, WY, false>(r, cell.k * r, false, Jz, Yz);
        const float* g = static_cast<const float*>(a.gb) + ((long long)i * a.nf + fi) * nw2;
#pragma unroll
        for (int w = 0; w < NWT; ++w) {
          const float2 v = __ldg(reinterpret_cast<const float2*>(g + 2 * wsel[w]));
          if (FUNC == 0) {
            acc[w][0] = fmaf(v.x, Jz.z0, acc[w][0]);
            acc[w][1] = fmaf(v.y, Jz.z0, acc[w][1]);
          } else {
            acc[w][0] += v.x * Jz.z0 - v.y * Yz.z0;
            acc[w][1] += v.y * Jz.z0 + v.x * Yz.z0;
          }
        }
      }
#pragma unroll
      for (int w = 0; w < NWT; ++w) {
        tot[w][0] += acc[w][0];
        tot[w][1] += acc[w][1];
      }
    }
  }
#pragma unroll
  for (int w = 0; w < NWT; ++w) {
    if (w0 + w >= a.nwin) break;
    const float re = tot[w][0], im = tot[w][1];
    a.out[((long long)(w0 + w) * a.nc + ci) * a.nf + fi] = sqrtf(re * re + im * im);
  }
}

template <int FUNC, int ITYPE>
void launch_mw(const MwDev& d, int nwt, cudaStream_t s) {
  const dim3 block(32, 8);  // 32 velocities x 8 frequencies
  const dim3 grid(div_up(d.nc, 32), div_up(d.nf, 8), div_up(d.nwin, nwt));
  if (nwt == 1)
    fj_mw_kernel<FUNC, ITYPE, 1><<<grid, block, 0, s>>>(d);
  else if (nwt == 2)
    fj_mw_kernel<FUNC, ITYPE, 2><<<grid, block, 0, s>>>(d);
  else if (nwt == 4)
    fj_mw_kernel<FUNC, ITYPE, 4><<<grid, block, 0, s>>>(d);
  else
    fj_mw_kernel<FUNC, ITYPE, 8><<<grid, block, 0, s>>>(d);
}

// All windows' spectra in `spec` ([nwin][ntr][nf] complex, sorted traces),
// distances `rs` sorted. Writes out [nwin][nc][nf] (normalised if asked).
int mwfj_cuda_core(const ccfj_eq_args& a, const float2* spec, cudaStream_t s, Scratch& sc) {
  const int nr = a.ntr, nf = a.nf, nwin = a.nwin;
  float* drs = sc.get_n<float>(nr + 1);
  float* wtr = sc.get_n<float>(nr);
  if (!drs || !wtr) return CCFJ_ERR_ALLOC;
  fj_prep_geom_kernel_shared(a.r, nr, drs, wtr, s);
  count_launch();
  CCFJ_LAUNCH_CHECK("fj_prep_geom_kernel");
  const size_t esz = a.itype == 1 ? 8 : 4;
  void* gb = sc.get((size_t)nr * nf * 2 * nwin * esz);
  if (!gb) return CCFJ_ERR_ALLOC;
  mw_prep_kernel<<<dim3(nr, div_up(nf, 32), div_up(nwin, 8)), dim3(32, 8), 0, s>>>(
      spec, nr, nf, nwin, drs, wtr, a.itype, gb);
  count_launch();
  CCFJ_LAUNCH_CHECK("mw_prep_kernel");
  MwDev d{};
  d.rs = a.r;
  d.drs = drs;
  d.gb = gb;
  d.f = a.f;
  d.c = a.c;
  d.out = a.out;
  d.nr = nr;
  d.nf = nf;
  d.nc = a.nc;
  d.nwin = nwin;
  d.tau = a.tau > 0 ? a.tau : kDefaultTau32;
  const int nwt = nwin >= 8 ? 8 : nwin >= 4 ? 4 : nwin >= 2 ? 2 : 1;
  prof_begin(s);
  if (a.func == 0) {
    if (a.itype == 1)
      launch_mw<0, 1>(d, nwt, s);
    else
      launch_mw<0, 0>(d, nwt, s);
  } else {
    if (a.itype == 1)
      launch_mw<1, 1>(d, nwt, s);
    else
      launch_mw<1, 0>(d, nwt, s);
  }
  prof_end(s);
  count_launch();
  CCFJ_LAUNCH_CHECK("fj_mw_kernel");
  if (a.normalize) return normalize_sets(a.out, nwin, a.nc, nf, s);
  return CCFJ_OK;
}

}  // namespace ccfj
