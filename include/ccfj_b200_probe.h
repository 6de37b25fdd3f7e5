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

#endif /* CCFJ_B200_PROBE_H */
