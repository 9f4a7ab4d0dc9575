/*
 * Test infrastructure only: the subset of the FFTW3 API that the reference FMM-FFT uses,
 * backed by the project-written FP64 FFT in oracle/fft64.c.  With <complex.h> included
 * before this header (as src/fmmfft.c:12-15 does), real FFTW also defines fftw_complex as
 * `double _Complex`, so the reference source compiles unchanged.
 *
 * Call sites in the reference: fftw_malloc :1215,1224-1225; fftw_plan_dft :1217;
 * fftw_execute :1080; fftw_destroy_plan/fftw_free :1283-1286.
 * FFTW is not vendored and no version is pinned (makefile:2 links -lfftw3); this stand-in
 * computes the same mathematical transform: forward sign -1, unnormalised, in place.
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H
#include <stddef.h>

typedef double _Complex fftw_complex;
typedef struct shim_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
/* `n` is untyped because the reference passes a `long *` (fmmfft.c:1217). */
fftw_plan fftw_plan_dft(int rank, const void *n, fftw_complex *in, fftw_complex *out, int sign,
                        unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#endif
