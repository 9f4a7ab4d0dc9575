/*
 * ORACLE — TEST INFRASTRUCTURE ONLY (see fmmfft_oracle.h for who may use it).
 *
 * FP64 CPU restatement of the reference FMM-FFT forward transform, 97amarnathk/fmm-fft
 * src/fmmfft.c.  Each function cites the reference lines it follows.  Floating-point
 * expressions in the operator builders keep the reference's evaluation order so that the
 * operators agree with the reference's bit for bit (a test checks this against the
 * shim-built reference); the execute part keeps the reference's summation order inside each
 * dot product, so the restatement agrees with the reference to a few ulps.
 */
#include "fmmfft_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fft64.h"

static const double ORC_PI = 3.14159265358979323846264338327950288; /* fmmfft.c:17 */

static int is_pow2(long v) { return v > 0 && (v & (v - 1)) == 0; }
static long ilog2(long v) { /* fmmfft.c:57-64 */
  long r = 0;
  while (v > 1) {
    v /= 2;
    r++;
  }
  return r;
}

/* ---------------------------------------------------------------- operator builders */

/* Equivalent-source interpolation matrix of the upward/flip operators, fmmfft.c:81-114 (vx).
 * mat[k][j] (k = target node, j = equivalent point), rows = terms. */
static void orc_vx(double a, const double *x, double *mat, long T, const double *cn, double *mm,
                   double *acu) {
  double ac = 3 * tan(a);
  for (long j = 0; j < T; ++j) {
    double th = -1 * cos(((double)2 * (j + 1) - 2) / (2 * (T - 1)) * ORC_PI) * (2 * a);
    acu[j] = ac / tan(0.5 * th);
  }
  for (long k = 0; k < T; ++k) {
    double v = cn[k] - acu[k];
    for (long j = 0; j < T; ++j)
      if (j != k) v *= ((cn[k] - acu[j]) / (cn[k] - cn[j]));
    mm[k] = v;
  }
  for (long j = 0; j < T; ++j)
    for (long k = 0; k < T; ++k) {
      double v = mm[j] / (x[k] - acu[j]);
      for (long l = 0; l < T; ++l)
        if (l != j) v *= ((x[k] - cn[l]) / (x[k] - acu[l]));
      mat[k * T + j] = v;
    }
}

/* Local-expansion interpolation matrix, fmmfft.c:116-146 (wx).  Also (re)writes the
 * Chebyshev nodes cn, as the reference does at :122.  mat[k][j], rows = xlen. */
static void orc_wx(double a, const double *x, long xlen, double *mat, long T, double *cn,
                   double *acu) {
  double ac = 1 / tan(a);
  for (long j = 0; j < T; ++j) {
    double th = -cos(((double)(2 * (j + 1) - 2)) / (2 * (T - 1)) * ORC_PI) * (ORC_PI - 6 * a) + ORC_PI;
    acu[j] = ac * tan(0.5 * th);
    cn[j] = -cos(((double)2 * (j + 1) - 1) / (2 * T) * ORC_PI);
  }
  for (long j = 0; j < T; ++j) {
    double mm = cn[j] - acu[j];
    for (long k = 0; k < T; ++k)
      if (k != j) mm *= ((cn[j] - acu[k]) / (cn[j] - cn[k]));
    for (long k = 0; k < xlen; ++k) {
      double v = mm / (x[k] - acu[j]);
      for (long l = 0; l < T; ++l)
        if (l != j) v *= ((x[k] - cn[l]) / (x[k] - acu[l]));
      mat[k * T + j] = v;
    }
  }
}

/* M2M shift, fmmfft.c:148-159 (shftf). */
static void orc_shftf(long lev, long dir, double *mat, long T, double *cn, double *x, double *w1,
                      double *w2) {
  double dd = (double)dir;
  double a = ORC_PI / pow(2, lev);
  double ta3 = 3 * tan(a);
  double td2 = tan(0.5 * a);
  for (long j = 0; j < T; ++j) x[j] = 3 * td2 * (cn[j] + dd * ta3 * td2) / (ta3 - dd * td2 * cn[j]);
  orc_vx(0.5 * a, x, mat, T, cn, w1, w2);
}

/* L2T weights of one target position ffr in [-1,1] box coordinates, fmmfft.c:161-172. */
static void orc_evlmf(double ffr, long s, long lq, double *vec, long T, double *w, double *cn,
                      double *acu) {
  double a = (ORC_PI / s) * 0.5;
  double th = ffr * a;
  double x = tan(th) / tan(a);
  orc_wx(a, &x, 1, w, T, cn, acu);
  for (long t = 0; t < T; ++t) vec[t] = w[t] / lq;
}

/* L2L shift, fmmfft.c:186-197 (shftl). */
static void orc_shftl(long lev, long dir, double *mat, long T, double *cn, double *x, double *acu) {
  double dd = (double)dir;
  double a = ORC_PI / pow(2, lev);
  double c = tan(0.25 * a);
  double td2 = tan(0.5 * a);
  for (long j = 0; j < T; ++j) x[j] = (cn[j] - dd) / (1 / c + dd * c * cn[j]) / td2;
  orc_wx(0.5 * a, x, T, mat, T, cn, acu);
}

/* M2L flip by `shft` boxes, fmmfft.c:227-240 (flip). */
static void orc_flip(long lev, long shft, double *mat, long T, double *cn, double *x, double *w1,
                     double *w2) {
  double a = ORC_PI / (pow(2, lev));
  double bs = shft;
  double c = tan(0.5 * a);
  double td2 = tan(bs * a);
  for (long j = 0; j < T; ++j) x[j] = 3 * c * (1 - td2 * c * cn[j]) / (td2 + c * cn[j]);
  orc_vx(0.5 * a, x, mat, T, cn, w2, w1);
}

/* S2M matrix initch[j][k], fmmfft.c:242-259 (initg). */
static void orc_initg(long b, long s, double *initch, long T, double *tang, const double *cn) {
  double a = ORC_PI / (2.0 * s);
  for (long j = 0; j < b; ++j) tang[j] = tan(((double)(2 * (j + 1) - b - 1)) / (double)b * a);
  double ta3 = 3 * tan(a);
  for (long j = 0; j < b; ++j)
    for (long k = 0; k < T; ++k)
      initch[j * T + k] = (cn[k] + ta3 * tang[j]) / (ta3 - cn[k] * tang[j]);
}

/* Near-field cot value for integer offset d = l - m in section sc, the common formula of the
 * reference's cots/cotsh/cotprv tables (fmmfft.c:306,312,318). */
static double orc_cotval(long d, double gfrac, double dlq) {
  return -1 / tan(ORC_PI / dlq * ((double)d + gfrac)) / dlq;
}

orc_plan *orc_plan_create(long M, long P, long T, long b) {
  if (!is_pow2(P) || P < 2 || !is_pow2(M) || !is_pow2(b) || b < 2 || T < 2) return NULL;
  if (M % b) return NULL;
  long s = M / b;
  if (s < 4) return NULL;
  long n = ilog2(s);
  orc_plan *pl = (orc_plan *)calloc(1, sizeof(orc_plan));
  if (!pl) return NULL;
  pl->M = M, pl->P = P, pl->terms = T, pl->b = b, pl->s = s, pl->n = n;
  long nl = n - 2;
  pl->chnods = (double *)malloc(sizeof(double) * T);
  pl->initch = (double *)malloc(sizeof(double) * b * T);
  pl->topflp = (double *)malloc(sizeof(double) * T * T);
  pl->levops = (double *)malloc(sizeof(double) * (nl > 0 ? nl : 1) * 8 * T * T);
  pl->evalm = (double *)malloc(sizeof(double) * b * (P - 1) * T);
  pl->evalmh = (double *)malloc(sizeof(double) * (P / 2) * T);
  pl->cot = (double *)malloc(sizeof(double) * (P - 1) * 4 * b);
  pl->fo = (double complex *)malloc(sizeof(double complex) * P * (P - 1));
  double *wk1 = (double *)malloc(sizeof(double) * (b > T ? b : T));
  double *wk2 = (double *)malloc(sizeof(double) * T);
  double *wk3 = (double *)malloc(sizeof(double) * T);
  if (!pl->chnods || !pl->initch || !pl->topflp || !pl->levops || !pl->evalm || !pl->evalmh ||
      !pl->cot || !pl->fo || !wk1 || !wk2 || !wk3) {
    free(wk1), free(wk2), free(wk3);
    orc_plan_destroy(pl);
    return NULL;
  }
  double *cn = pl->chnods;
  double dlq = (double)M;
  /* fmmfft.c:273-275 */
  for (long j = 0; j < T; ++j) cn[j] = -1 * cos(((double)2 * (j + 1) - 1) / (2 * T) * ORC_PI);
  orc_initg(b, s, pl->initch, T, wk1, cn);      /* :277 */
  orc_flip(2, 2, pl->topflp, T, cn, wk1, wk2, wk3); /* :279 */
  for (long lev = 1; lev <= n - 2; ++lev) {      /* :281-290 */
    double *o = pl->levops + (lev - 1) * 8 * T * T;
    orc_shftf(lev + 2, -1, o + ORC_OP_SHFTFN * T * T, T, cn, wk1, wk2, wk3);
    orc_shftf(lev + 2, 1, o + ORC_OP_SHFTFP * T * T, T, cn, wk1, wk2, wk3);
    orc_flip(lev + 2, -2, o + ORC_OP_FLIP2N * T * T, T, cn, wk1, wk2, wk3);
    orc_flip(lev + 2, +2, o + ORC_OP_FLIP2P * T * T, T, cn, wk1, wk2, wk3);
    orc_flip(lev + 2, -3, o + ORC_OP_FLIP3N * T * T, T, cn, wk1, wk2, wk3);
    orc_flip(lev + 2, +3, o + ORC_OP_FLIP3P * T * T, T, cn, wk1, wk2, wk3);
    orc_shftl(lev + 1, -1, o + ORC_OP_SHFTLN * T * T, T, cn, wk1, wk2);
    orc_shftl(lev + 1, 1, o + ORC_OP_SHFTLP * T * T, T, cn, wk1, wk2);
  }
  for (long sc = 1; sc <= P - 1; ++sc) { /* :292-321 */
    double gfrac = ((double)sc) / P;
    for (long j = 1; j <= b; ++j) {
      double ffr = ((double)(2 * j - 1) - (((double)(2 * sc)) / P)) / b - 1;
      orc_evlmf(ffr, s, M, pl->evalm + ((j - 1) * (P - 1) + (sc - 1)) * T, T, wk1, cn, wk2);
    }
    if (sc >= P / 2) {
      long sce = sc - P / 2 + 1;
      double ffr = (((double)2 * b + 1) - ((double)2 * sc) / (P)) / (b)-1;
      orc_evlmf(ffr, s, M, pl->evalmh + (sce - 1) * T, T, wk1, cn, wk2);
    }
    for (long d = -2 * b; d < 2 * b; ++d) pl->cot[(sc - 1) * 4 * b + d + 2 * b] = orc_cotval(d, gfrac, dlq);
  }
  for (long sc = 1; sc <= P - 1; ++sc) { /* :325-331 */
    double ang = ORC_PI * ((double)sc) / P;
    for (long j = 1; j <= P; ++j) {
      double complex temp = (ang * (1 - 2 * j)) * I;
      pl->fo[(j - 1) * (P - 1) + (sc - 1)] = -cexp(temp) * sin(ang);
    }
  }
  free(wk1), free(wk2), free(wk3);
  return pl;
}

void orc_plan_destroy(orc_plan *pl) {
  if (!pl) return;
  free(pl->chnods), free(pl->initch), free(pl->topflp), free(pl->levops);
  free(pl->evalm), free(pl->evalmh), free(pl->cot), free(pl->fo);
  free(pl);
}

/* ---------------------------------------------------------------- execute */

/* out[sc][t] = sum_k v[sc][k] * mat[t][k] for each of `ns` sections, fmmfft.c:174-184 (mpp). */
static void orc_mpp(const double complex *v, long T, long ns, const double *mat,
                    double complex *out) {
  for (long sc = 0; sc < ns; ++sc)
    for (long t = 0; t < T; ++t) {
      double complex acc = v[sc * T] * mat[t * T];
      for (long k = 1; k < T; ++k) acc += v[sc * T + k] * mat[t * T + k];
      out[sc * T + t] = acc;
    }
}

/* dotp of fmmfft.c:72-79. */
static double complex orc_dot(long n, const double complex *x, const double *r) {
  double complex acc = 0;
  for (long i = 0; i < n; ++i) acc += x[i] * r[i];
  return acc;
}

/* Near-field sum over the 3b-point window that starts at point `w0` of section xs (periodic),
 * with window coefficient q given by cot[q + shift]; the sequential order of mn3,
 * fmmfft.c:213-225. */
static double complex orc_window(const double complex *xs, long M, long w0, long b3,
                                 const double *cot, long shift) {
  double complex acc = 0;
  for (long q = 0; q < b3; ++q) {
    long l = (w0 + q) & (M - 1);
    double complex term = xs[l] * cot[q + shift];
    acc = (q == 0) ? term : acc + term;
  }
  return acc;
}

int orc_forward_ex(const orc_plan *pl, const double complex *x, double complex *y,
                   double complex *u_out, double complex *z_out, double complex *phi_out,
                   double complex *psi_out, double complex *ssum_out) {
  const long M = pl->M, P = pl->P, T = pl->terms, b = pl->b, s = pl->s, n = pl->n;
  const long S1 = P - 1;
  const long nbox = (2L << n) - 4; /* boxes of levels 2..n */
  const size_t bs = (size_t)S1 * T; /* one box: [P-1][terms] */
  double complex *xs = (double complex *)malloc(sizeof(double complex) * P * M);
  double complex *phi = (double complex *)malloc(sizeof(double complex) * nbox * bs);
  double complex *psi = (double complex *)malloc(sizeof(double complex) * nbox * bs);
  double complex *u = (double complex *)malloc(sizeof(double complex) * S1 * M);
  double complex *z = (double complex *)malloc(sizeof(double complex) * P * M);
  double complex *sumsec = (double complex *)malloc(sizeof(double complex) * P);
  if (!xs || !phi || !psi || !u || !z || !sumsec) {
    free(xs), free(phi), free(psi), free(u), free(z), free(sumsec);
    return -2;
  }
#define LVOFF(l) ((1L << (l)) - 4) /* box offset of level l */
#define PHI(l, box) (phi + (size_t)(LVOFF(l) + (box)) * bs)
#define PSI(l, box) (psi + (size_t)(LVOFF(l) + (box)) * bs)
#define LOP(l, which) (pl->levops + ((l)-3) * 8 * T * T + (which) * T * T)

  /* Deinterleave into sections x_sc[m] = x[P m + sc], fmmfft.c:419-439. */
  for (long m = 0; m < M; ++m)
    for (long sc = 0; sc < P; ++sc) xs[sc * M + m] = x[m * P + sc];

  /* Section sums times i/M, fmmfft.c:441-457. */
  for (long sc = 1; sc < P; ++sc) {
    double complex acc = 0;
    for (long m = 0; m < M; ++m) acc = acc + xs[sc * M + m];
    sumsec[sc] = acc * (I / (double)M);
  }

  /* S2M at the leaves, fmmfft.c:199-211 (initmm), :465. */
#pragma omp parallel for schedule(static)
  for (long B = 0; B < s; ++B)
    for (long sc = 1; sc < P; ++sc)
      for (long k = 0; k < T; ++k) {
        const double complex *q = xs + sc * M + B * b;
        double complex acc = q[0] * pl->initch[k];
        for (long j = 1; j < b; ++j) acc += q[j] * pl->initch[j * T + k];
        PHI(n, B)[(sc - 1) * T + k] = acc;
      }

  /* Upward pass, fmmfft.c:476-515: phi_l[B] = shftfn*phi_{l+1}[2B] + shftfp*phi_{l+1}[2B+1]. */
  for (long l = n - 1; l >= 2; --l) {
    long nb = 1L << l;
#pragma omp parallel for schedule(static)
    for (long B = 0; B < nb; ++B) {
      double complex *tl = (double complex *)malloc(sizeof(double complex) * bs);
      double complex *tr = (double complex *)malloc(sizeof(double complex) * bs);
      orc_mpp(PHI(l + 1, 2 * B), T, S1, pl->levops + (l - 2) * 8 * T * T + ORC_OP_SHFTFN * T * T, tl);
      orc_mpp(PHI(l + 1, 2 * B + 1), T, S1, pl->levops + (l - 2) * 8 * T * T + ORC_OP_SHFTFP * T * T, tr);
      for (size_t i = 0; i < bs; ++i) PHI(l, B)[i] = tl[i] + tr[i];
      free(tl), free(tr);
    }
  }

  /* Top flip at level 2 (4 boxes, far field = the opposite box), fmmfft.c:620-639. */
  for (long c = 0; c < 4; ++c) orc_mpp(PHI(2, (c + 2) & 3), T, S1, pl->topflp, PSI(2, c));

  /* Downward pass, fmmfft.c:643-749: child c of level l gets the parent's L2L plus M2L from
   * the well-separated children of the parent's neighbours (offsets -2,+2,+3 for a left
   * child, -3,-2,+2 for a right child), all periodic. */
  for (long l = 3; l <= n; ++l) {
    long nb = 1L << l, mask = nb - 1;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nb; ++c) {
      double complex *sh = (double complex *)malloc(sizeof(double complex) * bs * 4);
      double complex *f2p = sh + bs, *f2n = sh + 2 * bs, *f3 = sh + 3 * bs;
      if ((c & 1) == 0) { /* left child, :697-721 */
        orc_mpp(PSI(l - 1, c >> 1), T, S1, LOP(l, ORC_OP_SHFTLP), sh);
        orc_mpp(PHI(l, (c - 2) & mask), T, S1, LOP(l, ORC_OP_FLIP2P), f2p);
        orc_mpp(PHI(l, (c + 2) & mask), T, S1, LOP(l, ORC_OP_FLIP2N), f2n);
        orc_mpp(PHI(l, (c + 3) & mask), T, S1, LOP(l, ORC_OP_FLIP3N), f3);
      } else { /* right child, :723-747 */
        orc_mpp(PSI(l - 1, c >> 1), T, S1, LOP(l, ORC_OP_SHFTLN), sh);
        orc_mpp(PHI(l, (c - 3) & mask), T, S1, LOP(l, ORC_OP_FLIP3P), f3);
        orc_mpp(PHI(l, (c - 2) & mask), T, S1, LOP(l, ORC_OP_FLIP2P), f2p);
        orc_mpp(PHI(l, (c + 2) & mask), T, S1, LOP(l, ORC_OP_FLIP2N), f2n);
      }
      for (size_t i = 0; i < bs; ++i) PSI(l, c)[i] = sh[i] + f2p[i] + f2n[i] + f3[i];
      free(sh);
    }
  }

  /* L2T evaluation (fmmfft.c:751-803) plus near-field direct sums (fmmfft.c:805-954).
   * Target j of leaf box B sits at m = B b + j, shifted by -sc/P.  Point j = 0 belongs to box
   * B for sc < P/2, to box B-1 (as its position b) for sc > P/2, and for sc = P/2 the two
   * evaluations are averaged. */
  const long b3 = 3 * b;
#pragma omp parallel for schedule(static)
  for (long sc = 1; sc < P; ++sc) {
    const double complex *xsc = xs + sc * M;
    const double *cot = pl->cot + (sc - 1) * 4 * b; /* cot[d + 2b] */
    double complex *usc = u + (sc - 1) * M;
    for (long B = 0; B < s; ++B) {
      const double complex *psB = PSI(n, B) + (sc - 1) * T;
      const double complex *psP = PSI(n, (B - 1) & (s - 1)) + (sc - 1) * T;
      for (long j = 0; j < b; ++j) {
        long m = B * b + j;
        double complex far, near;
        if (j > 0 || 2 * sc < P) {
          far = orc_dot(T, psB, pl->evalm + (j * (P - 1) + (sc - 1)) * T);
          near = orc_window(xsc, M, (B - 1) * b, b3, cot, b - j); /* cots / cotprv */
        } else if (2 * sc > P) {
          far = orc_dot(T, psP, pl->evalmh + (sc - P / 2) * T);
          near = orc_window(xsc, M, (B - 2) * b, b3, cot, 0); /* cotsh */
        } else {
          double complex f1 = orc_dot(T, psB, pl->evalm + (sc - 1) * T);
          double complex f2 = orc_dot(T, psP, pl->evalmh);
          far = 0.5 * (f1 + f2);
          double complex d1 = orc_window(xsc, M, (B - 1) * b, b3, cot, b);
          double complex d2 = orc_window(xsc, M, (B - 2) * b, b3, cot, 0);
          near = (d1 + d2) * 0.5;
        }
        usc[m] = far + near;
      }
    }
  }

  /* Combine, fmmfft.c:956-968: z_r[m] = x_0[m] + sum_sc fo[r][sc] (u_sc[m] - sumsec[sc]). */
#pragma omp parallel for schedule(static)
  for (long r = 0; r < P; ++r)
    for (long m = 0; m < M; ++m) {
      double complex acc = xs[m];
      for (long sc = 1; sc < P; ++sc) acc += pl->fo[r * (P - 1) + (sc - 1)] * (u[(sc - 1) * M + m] - sumsec[sc]);
      z[r * M + m] = acc;
    }

  /* Local size-M forward FFTs, fmmfft.c:1080; block r lands at y[r M .. r M + M). */
  if (z_out) memcpy(z_out, z, sizeof(double complex) * P * M);
#pragma omp parallel for schedule(static)
  for (long r = 0; r < P; ++r) fft64_forward(M, z + r * M);
  memcpy(y, z, sizeof(double complex) * P * M);

  if (u_out) memcpy(u_out, u, sizeof(double complex) * S1 * M);
  if (phi_out) memcpy(phi_out, phi, sizeof(double complex) * nbox * bs);
  if (psi_out) memcpy(psi_out, psi, sizeof(double complex) * nbox * bs);
  if (ssum_out)
    for (long sc = 1; sc < P; ++sc) ssum_out[sc - 1] = sumsec[sc];
#undef LVOFF
#undef PHI
#undef PSI
#undef LOP
  free(xs), free(phi), free(psi), free(u), free(z), free(sumsec);
  return 0;
}

int orc_forward(long N, long P, long T, long b, const double *x, double *y) {
  if (P < 2 || N % P) return -1;
  orc_plan *pl = orc_plan_create(N / P, P, T, b);
  if (!pl) return -1;
  int rc = orc_forward_ex(pl, (const double complex *)x, (double complex *)y, NULL, NULL, NULL,
                          NULL, NULL);
  orc_plan_destroy(pl);
  return rc;
}

/* ---------------------------------------------------------------- reference layout */

long orc_getwlen2(long lq, long terms, long p, long b) { /* fmmfft.c:1160-1183 */
  long s = lq / b;
  long n = ilog2(s);
  long ind = 0;
  ind += 8 * (terms * terms * (n - 2));
  ind += terms * terms;
  ind += terms * b;
  ind += terms * (p - 1) * b;
  ind += terms * p / 2;
  ind += (3 * b * p) / 2;
  ind += 3 * b * (b - 1) * (p - 1);
  ind += (3 * b * p) / 2;
  ind += terms;
  ind += 2 * (p - 1) * p;
  ind += p * (p - 1);
  ind += b;
  ind += 3 * terms;
  ind++;
  return ind;
}

long orc_getvlen(long lq, long terms, long p, long b) { /* fmmfft.c:1110-1135 */
  long s = lq / b;
  long t = s / p;
  long n = ilog2(s);
  long log2np = ilog2(p);
  long ind = 0;
  ind += 2 * (2 * terms * (p - 1) * (2 * t + log2np - 3));
  ind += 2 * (2 * p);
  ind += 3 * (2 * terms * (p - 1));
  ind += 2 * (2 * (p - 1) * (b + n * 2 * terms));
  ind += 2 * (2 * ((p - 1) * (b + n * 2 * terms) + p / 2));
  ind += 2 * b * p;
  ind += 2 * b * (p - 1);
  ind += 2 * (2 * (p / 2));
  ind += 10 * (2 * terms * (p - 1));
  ind += 2 * (2 * terms * (p - 1) * 2 * n);
  ind += 2 * lq;
  ind += 2 * (p - 1);
  ind += 2 * (2 * (p / 2));
  ind = ind + b;
  ind += 3 * terms;
  ind += 2 * (3 * p);
  ind++;
  return ind;
}

/* Lay the operators out as mfti does (fmmfft.c:343-374): eight [n-2][T][T] level tables,
 * topflp, initch, evalm, evalmh, cotsh, cots, cotprv, chnods, fo.  The scratch slots that
 * follow (wknie, wkp..) are left as zero. */
int orc_fill_reference_w(const orc_plan *pl, double *w, long wlen) {
  const long T = pl->terms, b = pl->b, P = pl->P, n = pl->n;
  if (wlen < orc_getwlen2(pl->M, T, P, b)) return -1;
  memset(w, 0, sizeof(double) * wlen);
  long ind = 0;
  for (long op = 0; op < 8; ++op) { /* ia[0..7] */
    for (long l = 0; l < n - 2; ++l)
      memcpy(w + ind + l * T * T, pl->levops + (l * 8 + op) * T * T, sizeof(double) * T * T);
    ind += T * T * (n - 2);
  }
  memcpy(w + ind, pl->topflp, sizeof(double) * T * T); /* ia[8] */
  ind += T * T;
  memcpy(w + ind, pl->initch, sizeof(double) * T * b); /* ia[9] */
  ind += T * b;
  memcpy(w + ind, pl->evalm, sizeof(double) * T * (P - 1) * b); /* ia[10] */
  ind += T * (P - 1) * b;
  memcpy(w + ind, pl->evalmh, sizeof(double) * T * (P / 2)); /* ia[11] */
  ind += (T * P) / 2;
  for (long sce = 1; sce <= P / 2; ++sce) { /* ia[12] cotsh[sce][jj+b-1], jj in [1-b, 2b] */
    long sc = sce - 1 + P / 2;
    if (sc < 1 || sc > P - 1) continue;
    const double *cot = pl->cot + (sc - 1) * 4 * b;
    for (long q = 0; q < 3 * b; ++q) w[ind + (sce - 1) * 3 * b + q] = cot[q]; /* d = q - 2b */
  }
  ind += (3 * b * P) / 2;
  for (long sc = 1; sc <= P - 1; ++sc) { /* ia[13] cots[sc][k-2][jj+b-1] */
    const double *cot = pl->cot + (sc - 1) * 4 * b;
    for (long k = 2; k <= b; ++k)
      for (long q = 0; q < 3 * b; ++q) /* d = jj - k = q - b + 1 - k */
        w[ind + ((sc - 1) * (b - 1) + (k - 2)) * 3 * b + q] = cot[q - b + 1 - k + 2 * b];
  }
  ind += 3 * b * (b - 1) * (P - 1);
  for (long sc = 1; sc <= P / 2; ++sc) { /* ia[14] cotprv[sc][jj+b-1], d = jj - 1 = q - b */
    const double *cot = pl->cot + (sc - 1) * 4 * b;
    for (long q = 0; q < 3 * b; ++q) w[ind + (sc - 1) * 3 * b + q] = cot[q - b + 2 * b];
  }
  ind += (3 * b * P) / 2;
  memcpy(w + ind, pl->chnods, sizeof(double) * T); /* ia[15] */
  ind += T;
  memcpy(w + ind, pl->fo, sizeof(double complex) * P * (P - 1)); /* ia[16] */
  return 0;
}

int orc_fft64(long n, double *x) { return fft64_forward(n, (double complex *)x); }

double orc_max_error_percent(const double *x, const double *y, long len) { /* :1097-1108 */
  const double complex *a = (const double complex *)x, *c = (const double complex *)y;
  double mx = cabs(a[0] - c[0]) / cabs(c[0]) * 100;
  for (long i = 1; i < len; ++i) {
    double e = cabs(a[i] - c[i]) / cabs(c[i]) * 100;
    if (mx < e) mx = e;
  }
  return mx;
}
