// Internal interface of the time-domain front end (see fj_fft.cu).
#pragma once

#include <atomic>

#include "ccfj_core.cuh"

namespace ccfj {

// One window of the reference's `win`: its n1, n2 and ramp length delta
// (integers, computed on the host in float64 the way `win` computes them;
// taper_value in fj_fft.cu turns them into the per-sample window).
struct TaperSpec {
  int n1, n2, delta, pad;
};

struct FftJob {
  const float* u;          // traces [rows][u_ld], float32
  long long u_ld;
  const long long* perm;   // sorted trace i -> row of u (nullable)
  int ntr;                 // traces per window
  int npts;                // samples per trace (FFT length)
  int nbins;               // output bins per row
  int bin_stride;          // bin k of output kk is kk * bin_stride
  int log2n;               // filled in by rfft_bins
  const TaperSpec* taper;  // [nrows_out] or nullptr
  float2* out;             // [nrows_out][nbins]
};

// Runs the front end for nrows_out rows (row = w * ntr + i).
int rfft_bins(const FftJob& job, int nrows_out, cudaStream_t s, Scratch& sc);

// MWFJ transform of all windows at once from their spectra
// ([nwin][ntr][nf] complex, sorted traces), CUDA-core contraction.
int mwfj_cuda_core(const ccfj_eq_args& a, const float2* spec, cudaStream_t s, Scratch& sc);
// The same contraction on the tensor cores (tcgen05, scaled FP16x3): itype 1,
// func 0, 2 <= nr, nwin <= 128.
// call_err: a device word for this call's timeout flag (NULL: taken from sc).
// paired: the A-operand generator with paired FP32 arithmetic (else one
// interval at a time; the results agree to rounding).
int mwfj_tensor(const ccfj_eq_args& a, const float2* spec, cudaStream_t s, Scratch& sc,
                unsigned int* call_err, bool paired = true);
// Waits for `s` and reads one call's timeout flag.
int mw_tc_call_error(const unsigned int* err, cudaStream_t s, bool* failed);
// Waits for `s`, reads the process-wide timeout flag of the tensor kernel
// (set by any call since the last read) and clears it.
int mw_tc_sticky_error(cudaStream_t s, bool* failed);
// 0 = automatic, 1 = CUDA cores, 2 = tensor cores where supported.
extern std::atomic<int> g_mwfj_path;

}  // namespace ccfj
