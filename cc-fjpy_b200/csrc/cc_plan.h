// Host-side plan of one cross-correlation call (xcorr.cu): argument checks,
// the shift count, each station's kept shifts, the list of windows to
// transform, the FFT plan, and the station tiles and pair lookup of the pair
// products. Plain C++ (no CUDA), shared by the device driver and the
// host-side checks of the tests.
//
// Reference behaviour that the checks turn into errors instead of
// reproducing (src/CrossCorr.cpp):
// * bins j*fstride past fftlen/2, which the reference reads from FFTW output
//   memory that the transform never wrote (:97-115);
// * steplen <= 0 with fftlen < npts, where the reference divides by it (:52);
// * pair indices outside [0, nsta), read out of bounds (:120-127).
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/ccfj_b200.h"
#include "cc_core.cuh"

namespace ccfj {
namespace xc {

// Largest half length the shared-memory FFT handles (M complex points in
// one CTA: 64 KiB, with each thread holding at most M / 512 points of a
// pass in registers); longer or odd windows, or lengths with a prime factor
// above 5, take the direct transform of the requested bins.
constexpr int kMaxM = 8192;
constexpr int kFftThreads = 512;
// Shifts staged per step of the pair-product kernel
constexpr int kShiftChunk = 4;
// Largest station count (the pair lookup is nsta x nsta)
constexpr int kMaxStations = 16384;

struct Window {
  int k, i;  // shift, station
};

struct Tile {
  int a0, b0;  // first station of the a rows and of the b columns
  int k0, k1;  // shifts that can contribute (inclusive; k1 < k0: none)
  int pad;
};

struct Plan {
  int F = 0;               // samples per window (fftlen clamped to npts)
  long long nshifts = 0;   // windows per station
  bool stockham = false;   // shared-memory FFT (else direct transform)
  int M = 0;               // F / 2 for the shared-memory FFT
  int npass = 0;
  int radix[kMaxPasses] = {};
  int ldj = 0;             // row length of the spectra (nf rounded up to 32)
  std::vector<int> lo, hi; // [nsta] kept shifts lo..hi
  std::vector<Window> windows;  // kept (shift, station) windows, station-major
  std::vector<Tile> tiles;      // station tiles holding at least one pair
  std::vector<int> pmap;        // [nsta * nsta]: first pair (a, b), or -1
  std::vector<int> pnext;       // [npairs]: next pair with the same (a, b), or -1
};

inline int plan_fail(std::string* err, const std::string& msg) {
  if (err) *err = msg;
  return CCFJ_ERR_INVALID;
}

// Fills *p for the arguments (host pointers for pairs and startend).
inline int make_plan(const ccfj_cc_args& a, Plan* p, std::string* err) {
  if (a.nsta < 1 || a.nsta > kMaxStations)
    return plan_fail(err, "nsta=" + std::to_string(a.nsta) + " must be in 1.." +
                              std::to_string(kMaxStations));
  if (a.npts < 1) return plan_fail(err, "npts=" + std::to_string(a.npts) + " must be >= 1");
  if (a.nf < 0 || a.npairs < 0) return plan_fail(err, "nf and npairs must be >= 0");
  if (a.fstride < 1) return plan_fail(err, "fstride=" + std::to_string(a.fstride) + " must be >= 1");
  if (a.fftlen < 1) return plan_fail(err, "fftlen=" + std::to_string(a.fftlen) + " must be >= 1");
  if (!a.startend) return plan_fail(err, "startend is NULL");
  if (a.npairs > 0 && !a.pairs) return plan_fail(err, "pairs is NULL");
  if (a.out_layout != 0 && a.out_layout != 1)
    return plan_fail(err, "out_layout=" + std::to_string(a.out_layout) + " must be 0 or 1");
  const long long npts = a.npts;
  if (a.fftlen >= a.npts) {
    p->F = a.npts;
    p->nshifts = 1;
  } else {
    if (a.steplen <= 0)
      return plan_fail(err, "steplen=" + std::to_string(a.steplen) +
                                " must be > 0 when fftlen < npts (overlaprate < 1)");
    p->F = a.fftlen;
    p->nshifts = 1 + (npts - a.fftlen) / a.steplen;
  }
  if (a.nf > 0 && (long long)(a.nf - 1) * a.fstride > p->F / 2)
    return plan_fail(err, "bin (nf-1)*fstride=" + std::to_string((long long)(a.nf - 1) * a.fstride) +
                              " is past the last real-FFT bin " + std::to_string(p->F / 2) +
                              " of a " + std::to_string(p->F) + "-sample window");
  if (p->nshifts > (1LL << 30)) return plan_fail(err, "too many shifts");
  p->stockham = false;
  if (p->F % 2 == 0 && p->F / 2 <= kMaxM) {
    p->M = p->F / 2;
    p->npass = fft_plan(p->M, p->radix);
    p->stockham = p->npass > 0;
  }
  p->ldj = ((a.nf > 0 ? a.nf : 1) + kLanes - 1) / kLanes * kLanes;

  const int nsta = a.nsta;
  p->lo.assign(nsta, 0);
  p->hi.assign(nsta, -1);
  p->windows.clear();
  for (int i = 0; i < nsta; ++i) {
    long long lo, hi;
    shift_range(p->nshifts, a.steplen, p->F, a.startend[2 * i], a.startend[2 * i + 1], &lo, &hi);
    if (hi >= lo) {
      p->lo[i] = (int)lo;
      p->hi[i] = (int)hi;
      for (long long k = lo; k <= hi; ++k) p->windows.push_back(Window{(int)k, i});
    }
  }

  p->pmap.assign((size_t)nsta * nsta, -1);
  p->pnext.assign(a.npairs, -1);
  const int ntile = (nsta + kTile - 1) / kTile;
  std::vector<char> used((size_t)ntile * ntile, 0);
  for (int q = 0; q < a.npairs; ++q) {
    const int s0 = a.pairs[2 * q], s1 = a.pairs[2 * q + 1];
    if (s0 < 0 || s0 >= nsta || s1 < 0 || s1 >= nsta)
      return plan_fail(err, "pair " + std::to_string(q) + " = (" + std::to_string(s0) + ", " +
                                std::to_string(s1) + ") has a station outside 0.." +
                                std::to_string(nsta - 1));
    const size_t key = (size_t)s0 * nsta + s1;
    p->pnext[q] = p->pmap[key];
    p->pmap[key] = q;
    used[(size_t)(s0 / kTile) * ntile + s1 / kTile] = 1;
  }
  p->tiles.clear();
  for (int ta = 0; ta < ntile; ++ta)
    for (int tb = 0; tb < ntile; ++tb) {
      if (!used[(size_t)ta * ntile + tb]) continue;
      // shifts where some a row and some b column are both nonzero
      int alo = 1 << 30, ahi = -1, blo = 1 << 30, bhi = -1;
      for (int s = ta * kTile; s < nsta && s < (ta + 1) * kTile; ++s)
        if (p->hi[s] >= p->lo[s]) {
          alo = alo < p->lo[s] ? alo : p->lo[s];
          ahi = ahi > p->hi[s] ? ahi : p->hi[s];
        }
      for (int s = tb * kTile; s < nsta && s < (tb + 1) * kTile; ++s)
        if (p->hi[s] >= p->lo[s]) {
          blo = blo < p->lo[s] ? blo : p->lo[s];
          bhi = bhi > p->hi[s] ? bhi : p->hi[s];
        }
      const int k0 = alo > blo ? alo : blo, k1 = ahi < bhi ? ahi : bhi;
      if (k1 >= k0) p->tiles.push_back(Tile{ta * kTile, tb * kTile, k0, k1, 0});
    }
  return CCFJ_OK;
}

}  // namespace xc
}  // namespace ccfj
