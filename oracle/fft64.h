/* Test infrastructure only: project-written FP64 complex FFT used by the oracle. */
#ifndef ORACLE_FFT64_H
#define ORACLE_FFT64_H
#include <complex.h>

/* In-place forward DFT of length n (a power of two): X[k] = sum_m x[m] exp(-2*pi*i*m*k/n),
 * unnormalised.  This is the transform FFTW_FORWARD computes (reference fmmfft.c:1217,1080). */
int fft64_forward(long n, double complex *x);

#endif
