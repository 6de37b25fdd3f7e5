// Link-time stand-in for the reference's FFTW-based cross-correlator, which
// is not on the F-J path and cannot build here (no fftw3 headers or library).
// It only lets the reference's Cython module (src/ccfj.pyx) link so that its
// fj_noise / fj_earthquake / MWFJ wrappers run over src/FJcpu.cpp.
// Test infrastructure only: never linked into the product library.
#include "CrossCorr.h"

int CrossCorrelation(CC_data) { return -1; }
