// Host replay of the cross-correlation kernels (cc-fjpy_b200/csrc/xcorr.cu)
// for the CPU tests: the same plan (cc_plan.h) and the same per-thread
// arithmetic (cc_core.cuh), driven in the kernels' loop structure -- per
// Stockham pass every butterfly's loads before any store (the in-place
// pass), per station tile the same 4-shift staging with zero fill, the
// same epilogue. Test infrastructure only: built by tests/test_cc_emul.py
// with the host C++ compiler, never part of the library.
#include <math.h>
#include <string.h>

#include <string>
#include <vector>

#include "cc_plan.h"

using namespace ccfj::xc;

static std::string g_err;

extern "C" const char* cc_emul_error() { return g_err.c_str(); }

static void twiddle(std::vector<Cpx>& out, int n, int count) {
  out.resize(count);
  for (int u = 0; u < count; ++u) {
    const double a = -2.0 * M_PI * (double)u / (double)n;
    out[u] = cpx((float)cos(a), (float)sin(a));
  }
}

template <int R>
static void pass(std::vector<Cpx>& s, int M, int Ns, const Cpx* tw) {
  const int nb = M / R;
  std::vector<Cpx> v((size_t)nb * R);
  for (int t = 0; t < nb; ++t) bf_load<R>(s.data(), M, t, &v[(size_t)t * R]);
  for (int t = 0; t < nb; ++t) bf_finish<R>(s.data(), M, Ns, tw, t, &v[(size_t)t * R]);
}

// xc_spectra_kernel / xc_spectra_direct_kernel for every kept window
static void spectra(const Plan& p, const ccfj_cc_args& a, const float* data, std::vector<Cpx>& X) {
  X.assign((size_t)p.nshifts * a.nsta * p.ldj, cpx(0.f, 0.f));
  std::vector<Cpx> tw, twh;
  if (p.stockham) {
    twiddle(tw, p.M, p.M);
    twiddle(twh, 2 * p.M, p.M + 1);
  } else {
    twiddle(tw, p.F, p.F);
  }
  std::vector<Cpx> s;
  for (const Window& w : p.windows) {
    const float* x = data + (long long)w.i * a.npts + (long long)w.k * a.steplen;
    Cpx* out = X.data() + ((long long)w.k * a.nsta + w.i) * p.ldj;
    if (p.stockham) {
      s.resize(p.M);
      for (int m = 0; m < p.M; ++m) {
        float u = x[2 * m], v = x[2 * m + 1];
        if (a.onebit) {
          u = onebit(u);
          v = onebit(v);
        }
        s[m] = cpx(u, v);
      }
      int Ns = 1;
      for (int q = 0; q < p.npass; ++q) {
        const int R = p.radix[q];
        switch (R) {
          case 8: pass<8>(s, p.M, Ns, tw.data()); break;
          case 4: pass<4>(s, p.M, Ns, tw.data()); break;
          case 2: pass<2>(s, p.M, Ns, tw.data()); break;
          case 3: pass<3>(s, p.M, Ns, tw.data()); break;
          default: pass<5>(s, p.M, Ns, tw.data()); break;
        }
        Ns *= R;
      }
      for (int q = 0; q < a.nf; ++q) {
        const int k = q * a.fstride;
        Cpx v = real_bin(s.data(), p.M, k, twh[k]);
        if (a.whiten) v = whiten(v);
        out[q] = v;
      }
    } else {
      for (int q = 0; q < a.nf; ++q) {
        const long long k = (long long)q * a.fstride;
        double re = 0.0, im = 0.0;
        long long ph = 0;
        for (int n = 0; n < p.F; ++n) {
          float v = x[n];
          if (a.onebit) v = onebit(v);
          re += (double)v * (double)tw[ph].re;
          im += (double)v * (double)tw[ph].im;
          ph += k;
          if (ph >= p.F) ph -= p.F;
        }
        Cpx v = cpx((float)re, (float)im);
        if (a.whiten) v = whiten(v);
        out[q] = v;
      }
    }
  }
}

// xc_gram_kernel for every tile and frequency block
static void gram(const Plan& p, const ccfj_cc_args& a, const std::vector<Cpx>& X, float* out_re,
                 float* out_im, long long out_ld, int out_es) {
  constexpr int W = kGramThreads / 32;
  std::vector<Cpx> xs((size_t)kShiftChunk * 2 * kTile * kLanes);
  std::vector<Cpx> acc((size_t)W * kLanes * kRowsPerWarp * kTile);
  for (const Tile& t : p.tiles) {
    for (int j0 = 0; j0 < a.nf; j0 += kLanes) {
      for (Cpx& c : acc) c = cpx(0.f, 0.f);
      for (int kc = t.k0; kc <= t.k1; kc += kShiftChunk) {
        for (int e = 0; e < kShiftChunk * 2 * kTile * kLanes; ++e) {
          const int l = e % kLanes;
          const int row = (e / kLanes) % kTile;
          const int side = (e / (kLanes * kTile)) % 2;
          const int kk = e / (2 * kTile * kLanes);
          const int k = kc + kk;
          const int st = (side ? t.b0 : t.a0) + row;
          Cpx v = cpx(0.f, 0.f);
          if (k <= t.k1 && st < a.nsta) v = X[((long long)k * a.nsta + st) * p.ldj + j0 + l];
          xs[(((size_t)kk * 2 + side) * kTile + row) * kLanes + l] = v;
        }
        for (int kk = 0; kk < kShiftChunk; ++kk)
          for (int w = 0; w < W; ++w)
            for (int lane = 0; lane < kLanes; ++lane) {
              Cpx(&ac)[kRowsPerWarp][kTile] = *reinterpret_cast<Cpx(*)[kRowsPerWarp][kTile]>(
                  &acc[((size_t)w * kLanes + lane) * kRowsPerWarp * kTile]);
              gram_step(&xs[((size_t)kk * 2 + 0) * kTile * kLanes],
                        &xs[((size_t)kk * 2 + 1) * kTile * kLanes], w, lane, ac);
            }
      }
      for (int w = 0; w < W; ++w)
        for (int lane = 0; lane < kLanes; ++lane) {
          const int j = j0 + lane;
          if (j >= a.nf) continue;
          for (int ra = 0; ra < kRowsPerWarp; ++ra) {
            const int s0 = t.a0 + w * kRowsPerWarp + ra;
            if (s0 >= a.nsta) continue;
            for (int b = 0; b < kTile; ++b) {
              const int s1 = t.b0 + b;
              if (s1 >= a.nsta) continue;
              int q = p.pmap[(size_t)s0 * a.nsta + s1];
              if (q < 0) continue;
              const int cnt = pair_count(p.lo[s0], p.hi[s0], p.lo[s1], p.hi[s1]);
              if (cnt == 0) continue;
              const Cpx sum = acc[(((size_t)w * kLanes + lane) * kRowsPerWarp + ra) * kTile + b];
              for (; q >= 0; q = p.pnext[q]) {
                float* re = out_re + (long long)q * out_ld + (long long)j * out_es;
                float* im = out_im + (long long)q * out_ld + (long long)j * out_es;
                const Cpx init = a.accumulate ? cpx(*re, *im) : cpx(0.f, 0.f);
                const Cpx v = pair_value(init, sum, cnt);
                *re = v.re;
                *im = v.im;
              }
            }
          }
        }
    }
  }
}

// The host-memory path of ccfj_cc_v1, replayed: returns its status.
extern "C" int cc_emul_v1(const ccfj_cc_args* args) {
  g_err.clear();
  const ccfj_cc_args& a = *args;
  if (a.struct_size != (int)sizeof(ccfj_cc_args)) {
    g_err = "struct_size";
    return CCFJ_ERR_INVALID;
  }
  if (!a.data) {
    g_err = "data is NULL";
    return CCFJ_ERR_INVALID;
  }
  Plan p;
  const int st = make_plan(a, &p, &g_err);
  if (st != CCFJ_OK) return st;
  const long long nout = (long long)a.npairs * a.nf;
  const long long nrec = (long long)a.nsta * a.npts;
  if (a.onebit)
    for (long long n = 0; n < nrec; ++n) a.data[n] = onebit(a.data[n]);
  float* re = a.out_re;
  float* im = a.out_layout == 1 ? (a.out_re ? a.out_re + 1 : nullptr) : a.out_im;
  if (nout > 0 && !a.accumulate) {
    if (a.out_layout == 1) {
      memset(re, 0, 2 * nout * sizeof(float));
    } else {
      memset(re, 0, nout * sizeof(float));
      memset(im, 0, nout * sizeof(float));
    }
  }
  if (nout > 0 && !p.tiles.empty()) {
    std::vector<Cpx> X;
    spectra(p, a, a.data, X);
    gram(p, a, X, re, im, a.out_layout == 1 ? 2LL * a.nf : a.nf, a.out_layout == 1 ? 2 : 1);
  }
  return CCFJ_OK;
}

// The window spectra X [nshifts][nsta][ldj] of a call (complex float pairs);
// *ldj and *nshifts receive the layout. out may be NULL to query sizes.
extern "C" int cc_emul_spectra(const ccfj_cc_args* args, float* out, int* ldj,
                               long long* nshifts, int* stockham) {
  g_err.clear();
  Plan p;
  const int st = make_plan(*args, &p, &g_err);
  if (st != CCFJ_OK) return st;
  *ldj = p.ldj;
  *nshifts = p.nshifts;
  *stockham = p.stockham ? 1 : 0;
  if (out) {
    std::vector<Cpx> X;
    spectra(p, *args, args->data, X);
    memcpy(out, X.data(), X.size() * sizeof(Cpx));
  }
  return CCFJ_OK;
}

extern "C" void cc_emul_shift_range(long long nshifts, long long steplen, long long fftlen,
                                    long long start, long long end, long long* lo,
                                    long long* hi) {
  shift_range(nshifts, steplen, fftlen, start, end, lo, hi);
}

extern "C" int cc_emul_fft_plan(int M, int* radix) { return fft_plan(M, radix); }
