/*
 * Test infrastructure only: FFTW3 subset for the shim-built reference (see fftw3.h).
 */
#include <complex.h>
#include <stdlib.h>
#include "fftw3.h"
#include "../fft64.h"

struct shim_fftw_plan_s {
  long n;
  fftw_complex *in;
  fftw_complex *out;
  int sign;
};

void *fftw_malloc(size_t n) {
  void *p = NULL;
  if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
  return p;
}

void fftw_free(void *p) { free(p); }

fftw_plan fftw_plan_dft(int rank, const void *n, fftw_complex *in, fftw_complex *out, int sign,
                        unsigned flags) {
  (void)flags;
  if (rank != 1) return NULL;
  fftw_plan p = (fftw_plan)malloc(sizeof(*p));
  if (!p) return NULL;
  p->n = *(const int *)n; /* low 32 bits of the caller's long on little-endian hosts */
  p->in = in;
  p->out = out;
  p->sign = sign;
  return p;
}

void fftw_execute(const fftw_plan p) {
  if (!p) return;
  if (p->out != p->in)
    for (long i = 0; i < p->n; ++i) p->out[i] = p->in[i];
  if (p->sign == FFTW_BACKWARD) {
    for (long i = 0; i < p->n; ++i) p->out[i] = conj(p->out[i]);
    fft64_forward(p->n, p->out);
    for (long i = 0; i < p->n; ++i) p->out[i] = conj(p->out[i]);
  } else {
    fft64_forward(p->n, p->out);
  }
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
