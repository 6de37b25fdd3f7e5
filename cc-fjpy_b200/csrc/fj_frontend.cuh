// Internal interfaces between the transform and its device front ends.
#pragma once

#include "ccfj_core.cuh"

namespace ccfj {

// One input spectrum as the kernels read it: column fi of sorted pair i is
// p[row(i) * ld + fi * cs], row(i) = perm ? perm[i] : i.
struct InDesc {
  const float* p;
  long long ld;
  long long cs;
  const long long* perm;
};

// dst[i][fi] = (Hilbert transform along the full row of length n, element
// stride es, of row(i))[(col_begin + fi) * fstride]; dst is [nr][nf] float.
int hilbert_rows(const InDesc& in, int n, int es, int nr, int nf, int fstride, int col_begin,
                 float* dst, cudaStream_t s, Scratch& sc);

// The same by FFT (fj_fft.cu), for n a power of two from 512 to 8192.
bool hilbert_fft_supported(int n);
int hilbert_rows_fft(const InDesc& in, int n, int es, int nr, int nf, int fstride, int col_begin,
                     float* dst, cudaStream_t s, Scratch& sc);

// Device-resident transform (all pointers in args are device pointers);
// cpt > 0 forces that variant of the FP32 kernel (velocities per thread),
// nsplit > 0 that many station ranges (split launch, fixed-order sum).
int fj_device(const ccfj_fj_args& a, cudaStream_t s, int cpt = 0, int nsplit = 0);
// The argument checks of ccfj_fj_v1 (status and message as it returns them).
int fj_validate(const ccfj_fj_args* a);

}  // namespace ccfj
