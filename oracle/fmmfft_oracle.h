/*
 * ORACLE — TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load this library, and only as the checker or as
 * the timed CPU baseline; the product path never links or calls it.
 *
 * A CPU restatement, in FP64, of the reference FMM-FFT forward transform
 * (97amarnathk/fmm-fft, src/fmmfft.c: plan mfti/mftii :81-382, execute mft/mftint
 * :384-1081).  Parity is pinned two ways: against the unmodified reference compiled with the
 * project's MPI/FFTW shims (oracle/_ref, oracle/Makefile) and against golden vectors that
 * build made (tests/golden/), plus the reference's recorded error envelope
 * (plotting/raw_data/cluster_output_error.csv).
 *
 * The reference distributes the tree over P MPI ranks; the restatement runs the same global
 * periodic tree in one address space (levels 2..n, level l has 2^l boxes), which is what the
 * rank-to-rank exchanges of fmmfft.c:494-515, :517-618, :620-685, :760-761 implement.
 */
#ifndef ORACLE_FMMFFT_ORACLE_H
#define ORACLE_FMMFFT_ORACLE_H
#include <complex.h>

typedef struct orc_plan {
  long M, P, terms, b, s, n; /* M = N/P points per section, s = M/b leaf boxes, n = log2 s */
  double *chnods;            /* [terms]                 fmmfft.c:273-275 */
  double *initch;            /* [b][terms]   S2M        fmmfft.c:242-259,277 */
  double *topflp;            /* [terms][terms]          fmmfft.c:279 */
  double *levops;            /* [n-2][8][terms][terms]  fmmfft.c:281-290, order ORC_OP_* */
  double *evalm;             /* [b][P-1][terms]  L2T    fmmfft.c:295-298 */
  double *evalmh;            /* [P/2][terms]            fmmfft.c:300-304 */
  double *cot;               /* [P-1][4b] Toeplitz cot table, index d+2b for d in [-2b,2b) */
  double complex *fo;        /* [P][P-1]  combine       fmmfft.c:325-331 */
} orc_plan;

enum { ORC_OP_SHFTFN = 0, ORC_OP_SHFTFP, ORC_OP_FLIP2N, ORC_OP_FLIP2P, ORC_OP_FLIP3N,
       ORC_OP_FLIP3P, ORC_OP_SHFTLN, ORC_OP_SHFTLP };

/* Validates (P, M, b powers of two; P >= 2; s = M/b >= 4; b >= 2; terms >= 2) and builds
 * every operator in FP64.  Returns NULL on invalid parameters or allocation failure. */
orc_plan *orc_plan_create(long M, long P, long terms, long b);
void orc_plan_destroy(orc_plan *pl);

/* Full forward transform of x (N = P*M complex128, natural order) into y (natural order).
 * Optional outputs (NULL to skip):
 *   u   [P-1][M]  far+near field u_sc[m] before the combine (fmmfft.c psiev after :954)
 *   z   [P][M]    combined blocks z_r[m] before the local FFT (fmmfft.c qr after :970)
 *   phi [nbox][P-1][terms], psi likewise: multipole / local expansions of every level,
 *                 level l stored at box offset 2^l - 4 (levels 2..n, nbox = 2^(n+1) - 4)
 *   ssum [P-1]    sumsec[sc] = (i/M) * sum_m x_sc[m]   (fmmfft.c:441-457) */
int orc_forward_ex(const orc_plan *pl, const double complex *x, double complex *y,
                   double complex *u, double complex *z, double complex *phi,
                   double complex *psi, double complex *ssum);
int orc_forward(long N, long P, long terms, long b, const double *x, double *y);

/* Fills w (getwlen2 doubles) with the oracle's operators in the reference's mfti layout
 * (fmmfft.c:343-374), so a test can compare it bit for bit with the reference's own w. */
int orc_fill_reference_w(const orc_plan *pl, double *w, long wlen);
long orc_getwlen2(long lq, long terms, long p, long b); /* fmmfft.c:1160-1183 */
long orc_getvlen(long lq, long terms, long p, long b);  /* fmmfft.c:1110-1135 */

/* FP64 FFT used for the local transforms (test-side helper, see fft64.c). */
int orc_fft64(long n, double *x);
/* Reference error metric: max_i |x_i - y_i| / |y_i| * 100 (fmmfft.c:1097-1108). */
double orc_max_error_percent(const double *x, const double *y, long len);

#endif
