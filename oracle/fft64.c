/*
 * Test infrastructure only (oracle): FP64 complex FFT, iterative radix-2 decimation in time.
 *
 * It stands in for FFTW3 at the one place the reference uses it, the local size-M forward
 * FFT (src/fmmfft.c:1217 plan, :1080 execute), both in the shim-built reference and in the
 * oracle restatement.  Twiddles are evaluated directly as cos/sin of 2*pi*k/n in double
 * (no recurrences), so the transform's error stays at a few ulps * log2(n); tests check it
 * against numpy's pocketfft.
 */
#include "fft64.h"
#include <math.h>
#include <stdlib.h>

int fft64_forward(long n, double complex *x) {
  if (n < 1 || (n & (n - 1)) != 0) return -1;
  if (n == 1) return 0;
  /* bit-reversal permutation */
  for (long i = 1, j = 0; i < n; ++i) {
    long bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j |= bit;
    if (i < j) {
      double complex t = x[i];
      x[i] = x[j];
      x[j] = t;
    }
  }
  /* twiddle table w[k] = exp(-2 pi i k / n), k < n/2 */
  long half = n / 2;
  double complex *w = (double complex *)malloc(sizeof(double complex) * (size_t)half);
  if (!w) return -2;
  const double two_pi = 6.283185307179586476925286766559;
  for (long k = 0; k < half; ++k) {
    double ang = two_pi * (double)k / (double)n;
    w[k] = cos(ang) - I * sin(ang);
  }
  for (long len = 2; len <= n; len <<= 1) {
    long hl = len >> 1;
    long stride = n / len;
    for (long s = 0; s < n; s += len) {
      for (long k = 0; k < hl; ++k) {
        double complex t = w[k * stride] * x[s + k + hl];
        double complex a = x[s + k];
        x[s + k] = a + t;
        x[s + k + hl] = a - t;
      }
    }
  }
  free(w);
  return 0;
}
