/*
 * Test infrastructure only (oracle): FP64 complex FFT, iterative radix-2 decimation in time.
 *
 * It stands in for FFTW3 at the one place the reference uses it, the local size-M forward
 * FFT (src/fmmfft.c:1217 plan, :1080 execute), both in the shim-built reference and in the
 * oracle restatement.  Twiddles are evaluated directly as cos/sin of 2*pi*k/n in double
 * (no recurrences), so the transform's error stays at a few ulps * log2(n); tests check it
 * against numpy's pocketfft.  The twiddles of a length are computed once per process and kept
 * (FFTW keeps them in its plan the same way), laid out stage by stage so that every butterfly
 * pass reads them contiguously; the values are the same as evaluating them per call.
 */
#include "fft64.h"
#include <math.h>
#include <pthread.h>
#include <stdlib.h>

#define FFT64_CACHE 16

typedef struct {
  long n;
  double complex *stages; /* stage len = 2, 4, .., n: len/2 twiddles each, at offset len/2 - 1 */
} twiddles;

static twiddles g_cache[FFT64_CACHE];
static int g_ncache;
static pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;

/* Twiddles of length n: w[k] = exp(-2 pi i k / n), k < n/2, gathered per stage. */
static const double complex *twiddles_for(long n) {
  const double complex *found = NULL;
  pthread_mutex_lock(&g_mu);
  for (int i = 0; i < g_ncache; ++i)
    if (g_cache[i].n == n) found = g_cache[i].stages;
  pthread_mutex_unlock(&g_mu);
  if (found) return found;
  const long half = n / 2;
  double complex *w = (double complex *)malloc(sizeof(double complex) * (size_t)half);
  double complex *st = (double complex *)malloc(sizeof(double complex) * (size_t)(n > 1 ? n - 1 : 1));
  if (!w || !st) {
    free(w), free(st);
    return NULL;
  }
  const double two_pi = 6.283185307179586476925286766559;
  for (long k = 0; k < half; ++k) {
    double ang = two_pi * (double)k / (double)n;
    w[k] = cos(ang) - I * sin(ang);
  }
  for (long len = 2; len <= n; len <<= 1) {
    const long hl = len >> 1, stride = n / len;
    for (long k = 0; k < hl; ++k) st[hl - 1 + k] = w[k * stride];
  }
  free(w);
  pthread_mutex_lock(&g_mu);
  for (int i = 0; i < g_ncache; ++i)
    if (g_cache[i].n == n) { /* another thread made it meanwhile */
      pthread_mutex_unlock(&g_mu);
      free(st);
      return g_cache[i].stages;
    }
  if (g_ncache < FFT64_CACHE) {
    g_cache[g_ncache].n = n, g_cache[g_ncache].stages = st;
    ++g_ncache;
  }
  /* a full cache keeps this table alive too (it is returned to the caller and not freed) */
  pthread_mutex_unlock(&g_mu);
  return st;
}

int fft64_forward(long n, double complex *x) {
  if (n < 1 || (n & (n - 1)) != 0) return -1;
  if (n == 1) return 0;
  const double complex *tw = twiddles_for(n);
  if (!tw) return -2;
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
  for (long len = 2; len <= n; len <<= 1) {
    const long hl = len >> 1;
    const double complex *w = tw + hl - 1;
    for (long s = 0; s < n; s += len) {
      for (long k = 0; k < hl; ++k) {
        double complex t = w[k] * x[s + k + hl];
        double complex a = x[s + k];
        x[s + k] = a + t;
        x[s + k + hl] = a - t;
      }
    }
  }
  return 0;
}
