/*
 * ccfj_b200_probe -- test library of ccfj_b200 (libccfj_b200_probe.so).
 *
 * Not part of the product library and not a drop-in for anything in the
 * reference: these entries exist only so that unit tests can evaluate the
 * special-function code that the transform kernels compile (J0, J1, Y0, Y1
 * and B = int_0^x Z0; the reference's counterparts are bessj0/bessj1/
 * bessy0/bessy1 and STVH0/STVH1, src/FJcpu.cpp:21-228).
 */
#ifndef CCFJ_B200_PROBE_H
#define CCFJ_B200_PROBE_H

#ifdef __cplusplus
#define CCFJ_PROBE_API extern "C" __attribute__((visibility("default")))
#else
#define CCFJ_PROBE_API __attribute__((visibility("default")))
#endif

/* Host-side evaluation of the kernels' special-function code.
 * precision: CCFJ_PREC_FP32 (0) or CCFJ_PREC_FP64 (1). For each x[i] >= 0
 * writes out[6*i .. 6*i+5] = J0, J1, BJ, Y0, Y1, BY with BZ(x) = int_0^x Z0.
 * Returns 0, or 1 (invalid argument). */
CCFJ_PROBE_API int ccfj_special_host(int precision, long long n, const double *x, double *out);
/* The same on the device (x, out device pointers, async on stream): the
 * kernels' own instruction sequences, fast sine/cosine included. Returns 0,
 * 1 (invalid argument) or 2 (launch failed). */
CCFJ_PROBE_API int ccfj_special_device(int precision, long long n, const double *x, double *out,
                                       void *stream);

/* The transform kernels' station values y0 = J0 / M, y1 = J1 / M of two
 * cells (f, c0) and (f, c1) at distance r, x = 2 pi f r / c >= 8 in both:
 * in[4*i .. 4*i+3] = f, c0, c1, r (device pointer, float32); out[8*i ..]
 * = the scalar path's y0, y1 of cell 0 and of cell 1, then the paired path's
 * (two cells per FFMA2 / FMUL2 / FADD2) in the same order. Async on stream.
 * Returns 0, 1 (invalid argument), 2 (launch failed) or 4 (not sm_100). */
CCFJ_PROBE_API int ccfj_paired_probe(long long n, const float *in, float *out, void *stream);

#endif /* CCFJ_B200_PROBE_H */
