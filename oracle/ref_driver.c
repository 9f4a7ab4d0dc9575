/*
 * Test infrastructure only: drives the UNMODIFIED reference FMM-FFT (src/fmmfft.c, compiled
 * with -Dmain=fmmfft_reference_main against oracle/shim/) on P thread-ranks.
 *
 * It does what the reference's own main() does (src/fmmfft.c:1192-1288) with two changes that
 * a seeded-input driver needs: the input is the caller's vector instead of the ramp
 * (fmmfft.c:1227-1246), and each timed run restores the input first (the reference re-runs
 * mft on its previous output, fmmfft.c:1254-1273).  Per rank: getwlen2/getvlen sizes
 * (:1222-1223), mfti (:1249), then mft bracketed by barriers and timed (:1255-1263).
 */
#include <complex.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "shim/fftw3.h"
#include "shim/mpi.h"

/* Reference entry points (src/fmmfft.c:337, :980, :1110, :1160). */
void mfti(long lq, long p, long t, long b, double *wkkeep, double *wktemp, long szkeep, long sztemp);
void mft(long lq, double complex *qr, long dir, long p, long myid, long terms, long b, double *w,
         double *v, long sz1, long szwk, fftw_plan forward_plan);
long getvlen(long lq, long terms, long p, long b);
long getwlen2(long lq, long terms, long p, long b);

typedef struct {
  int rank;
  long N, P, terms, b;
  int runs;
  const double complex *x;
  double complex *y;
  double *times; /* per run, written by rank 0 */
  int status;
} rank_job;

static void *rank_main(void *arg) {
  rank_job *J = (rank_job *)arg;
  shim_mpi_set_rank(J->rank);
  long M = J->N / J->P;
  double complex *qr = (double complex *)fftw_malloc(sizeof(double complex) * (size_t)M);
  long wl = getwlen2(M, J->terms, J->P, J->b);
  long vl = getvlen(M, J->terms, J->P, J->b);
  double *w = (double *)fftw_malloc(sizeof(double) * (size_t)wl);
  double *v = (double *)fftw_malloc(sizeof(double) * (size_t)vl);
  int ok = qr && w && v;
  if (!ok) J->status = -2;
  int lm = (int)M;
  fftw_plan plan = ok ? fftw_plan_dft(1, &lm, qr, qr, FFTW_FORWARD, FFTW_ESTIMATE) : NULL;
  if (ok) {
    memset(w, 0, sizeof(double) * (size_t)wl);
    memset(v, 0, sizeof(double) * (size_t)vl);
    mfti(M, J->P, J->terms, J->b, w, v, 0, 0);
  }
  for (int run = 0; run < J->runs; ++run) {
    if (ok) memcpy(qr, J->x + (size_t)J->rank * (size_t)M, sizeof(double complex) * (size_t)M);
    MPI_Barrier(MPI_COMM_WORLD);
    double t0 = MPI_Wtime();
    if (ok) mft(M, qr, 1, J->P, J->rank, J->terms, J->b, w, v, 0, 0, plan);
    MPI_Barrier(MPI_COMM_WORLD);
    double t1 = MPI_Wtime();
    if (J->rank == 0 && J->times) J->times[run] = t1 - t0;
  }
  if (ok) memcpy(J->y + (size_t)J->rank * (size_t)M, qr, sizeof(double complex) * (size_t)M);
  if (plan) fftw_destroy_plan(plan);
  fftw_free(qr);
  fftw_free(w);
  fftw_free(v);
  return NULL;
}

/* Forward FMM-FFT of x (N complex128, interleaved re/im) on P thread-ranks with the
 * reference code.  y receives the N outputs in natural order.  times (optional, `runs`
 * entries) receives rank 0's barrier-to-barrier wall time of each mft call. */
int fmmref_forward(long N, long P, long terms, long b, const double *x, double *y, int runs,
                   double *times) {
  if (P < 2 || N % P || runs < 1) return -1;
  if (shim_mpi_world_begin((int)P) != 0) return -2;
  pthread_t *th = (pthread_t *)calloc((size_t)P, sizeof(pthread_t));
  rank_job *jobs = (rank_job *)calloc((size_t)P, sizeof(rank_job));
  if (!th || !jobs) return -2;
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, 16u << 20);
  for (long r = 0; r < P; ++r) {
    jobs[r] = (rank_job){(int)r, N, P, terms, b, runs, (const double complex *)x,
                         (double complex *)y, times, 0};
    pthread_create(&th[r], &attr, rank_main, &jobs[r]);
  }
  int status = 0;
  for (long r = 0; r < P; ++r) {
    pthread_join(th[r], NULL);
    if (jobs[r].status) status = jobs[r].status;
  }
  pthread_attr_destroy(&attr);
  shim_mpi_world_end();
  free(th);
  free(jobs);
  return status;
}

/* The operator buffer w that the reference's mfti builds (getwlen2 doubles). */
long fmmref_wlen(long M, long P, long terms, long b) { return getwlen2(M, terms, P, b); }
long fmmref_vlen(long M, long P, long terms, long b) { return getvlen(M, terms, P, b); }
int fmmref_mfti(long M, long P, long terms, long b, double *w, double *v) {
  mfti(M, P, terms, b, w, v, 0, 0);
  return 0;
}
