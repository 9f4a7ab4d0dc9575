/*
 * FMM operator construction in FP64 on the host (the plan step of the reference, src/fmmfft.c
 * mfti/mftii :81-382).
 *
 * The reference's interpolative FMM keeps every expansion as values at `T` Chebyshev nodes in a
 * tan-mapped box coordinate.  Every operator is a T-column interpolation matrix whose columns
 * are products over the nodes: two families differ only in where the "equivalent points" sit
 * (equiv_up, reference vx :81-114, for multipole-type operators; equiv_down, reference wx
 * :116-146, for local-type operators) and in which target points the rows evaluate.  The
 * floating-point expressions follow the reference's evaluation order so that the operators are
 * bit-identical to its own (the library's mfti returns them in the reference layout).
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fmmfft_internal.h"

static const double FMM_PI = 3.14159265358979323846264338327950288;

static int pow2(long v) { return v > 0 && (v & (v - 1)) == 0; }
static long lg2(long v) {
  long r = 0;
  while (v > 1) v /= 2, r++;
  return r;
}

int fmm_validate(long M, long P, long T, long b) {
  if (!pow2(P) || P < 2 || P > 1024) return 0;
  if (!pow2(M) || M > (1L << 26)) return 0;
  if (!pow2(b) || b < 2 || M % b) return 0;
  if (M / b < 4) return 0;
  if (T < 2 || T > 64) return 0;
  return 1;
}

/* Chebyshev node j (0-based) of order T on [-1,1] (reference :274, :122). */
static double cheb(long j, long T) { return -cos(((double)2 * (j + 1) - 1) / (2 * T) * FMM_PI); }

/* Fill one interpolation matrix mat[row][col] (rows = nx targets x[], cols = T):
 *   mat[k][j] = w_j / (x_k - e_j) * prod_{l != j} (x_k - c_l) / (x_k - e_l),
 *   w_j       = (c_j - e_j) * prod_{l != j} (c_j - e_l) / (c_j - c_l),
 * with Chebyshev nodes c and equivalent points e.  Products run in ascending l, skipping j. */
static void interp_matrix(const double *x, long nx, const double *c, const double *e, long T,
                          double *wgt, double *mat) {
  for (long j = 0; j < T; ++j) {
    double w = c[j] - e[j];
    for (long l = 0; l < T; ++l)
      if (l != j) w *= ((c[j] - e[l]) / (c[j] - c[l]));
    wgt[j] = w;
  }
  for (long j = 0; j < T; ++j)
    for (long k = 0; k < nx; ++k) {
      double v = wgt[j] / (x[k] - e[j]);
      for (long l = 0; l < T; ++l)
        if (l != j) v *= ((x[k] - c[l]) / (x[k] - e[l]));
      mat[k * T + j] = v;
    }
}

/* Equivalent points of multipole-type operators, reference vx :82-87. */
static void equiv_up(double a, long T, double *e) {
  double ac = 3 * tan(a);
  for (long j = 0; j < T; ++j) {
    double th = -1 * cos(((double)2 * (j + 1) - 2) / (2 * (T - 1)) * FMM_PI) * (2 * a);
    e[j] = ac / tan(0.5 * th);
  }
}

/* Equivalent points of local-type operators, reference wx :117-123. */
static void equiv_down(double a, long T, double *e) {
  double ac = 1 / tan(a);
  for (long j = 0; j < T; ++j) {
    double th = -cos(((double)(2 * (j + 1) - 2)) / (2 * (T - 1)) * FMM_PI) * (FMM_PI - 6 * a) + FMM_PI;
    e[j] = ac * tan(0.5 * th);
  }
}

typedef struct {
  long T;
  double *c, *e, *x, *wgt;
} op_scratch;

/* M2M child -> parent shift for tree level lev, direction dir = -1 / +1 (reference :148-159). */
static void op_shift_up(op_scratch *S, long lev, long dir, double *mat) {
  double dd = (double)dir, a = FMM_PI / pow(2, lev);
  double ta3 = 3 * tan(a), td2 = tan(0.5 * a);
  for (long j = 0; j < S->T; ++j)
    S->x[j] = 3 * td2 * (S->c[j] + dd * ta3 * td2) / (ta3 - dd * td2 * S->c[j]);
  equiv_up(0.5 * a, S->T, S->e);
  interp_matrix(S->x, S->T, S->c, S->e, S->T, S->wgt, mat);
}

/* L2L parent -> child shift (reference :186-197). */
static void op_shift_down(op_scratch *S, long lev, long dir, double *mat) {
  double dd = (double)dir, a = FMM_PI / pow(2, lev);
  double cq = tan(0.25 * a), td2 = tan(0.5 * a);
  for (long j = 0; j < S->T; ++j) S->x[j] = (S->c[j] - dd) / (1 / cq + dd * cq * S->c[j]) / td2;
  equiv_down(0.5 * a, S->T, S->e);
  interp_matrix(S->x, S->T, S->c, S->e, S->T, S->wgt, mat);
}

/* M2L between boxes `shft` apart at level lev (reference :227-240). */
static void op_flip(op_scratch *S, long lev, long shft, double *mat) {
  double a = FMM_PI / (pow(2, lev)), bs = shft;
  double cq = tan(0.5 * a), td = tan(bs * a);
  for (long j = 0; j < S->T; ++j) S->x[j] = 3 * cq * (1 - td * cq * S->c[j]) / (td + cq * S->c[j]);
  equiv_up(0.5 * a, S->T, S->e);
  interp_matrix(S->x, S->T, S->c, S->e, S->T, S->wgt, mat);
}

/* L2T weights of a leaf target at box coordinate ffr in [-1,1], scaled by 1/lq (reference
 * evlmf :161-172). */
static void op_eval_point(op_scratch *S, double ffr, long s, long lq, double *vec) {
  double a = (FMM_PI / s) * 0.5;
  double x = tan(ffr * a) / tan(a);
  equiv_down(a, S->T, S->e);
  interp_matrix(&x, 1, S->c, S->e, S->T, S->wgt, vec);
  for (long t = 0; t < S->T; ++t) vec[t] = vec[t] / lq;
}

void fmm_ops64_free(fmm_ops64 *o) {
  if (!o) return;
  free(o->chnods), free(o->initch), free(o->topflp), free(o->levops);
  free(o->evalm), free(o->evalmh), free(o->cot), free(o->fo);
  memset(o, 0, sizeof(*o));
}

int fmm_ops64_build(long M, long P, long T, long b, fmm_ops64 *o) {
  memset(o, 0, sizeof(*o));
  if (!fmm_validate(M, P, T, b)) return 1;
  long s = M / b, n = lg2(s), nlev = n - 2;
  o->M = M, o->P = P, o->T = T, o->b = b, o->s = s, o->n = n;
  o->chnods = (double *)malloc(sizeof(double) * T);
  o->initch = (double *)malloc(sizeof(double) * b * T);
  o->topflp = (double *)malloc(sizeof(double) * T * T);
  o->levops = (double *)malloc(sizeof(double) * (nlev > 0 ? nlev : 1) * FMM_NLEVOPS * T * T);
  o->evalm = (double *)malloc(sizeof(double) * b * (P - 1) * T);
  o->evalmh = (double *)malloc(sizeof(double) * (P / 2) * T);
  o->cot = (double *)malloc(sizeof(double) * (P - 1) * 4 * b);
  o->fo = (double *)malloc(sizeof(double) * 2 * P * (P - 1));
  op_scratch S = {T, NULL, NULL, NULL, NULL};
  S.e = (double *)malloc(sizeof(double) * T);
  S.x = (double *)malloc(sizeof(double) * (T > b ? T : b));
  S.wgt = (double *)malloc(sizeof(double) * T);
  if (!o->chnods || !o->initch || !o->topflp || !o->levops || !o->evalm || !o->evalmh ||
      !o->cot || !o->fo || !S.e || !S.x || !S.wgt) {
    free(S.e), free(S.x), free(S.wgt);
    fmm_ops64_free(o);
    return 2;
  }
  S.c = o->chnods;
  for (long j = 0; j < T; ++j) o->chnods[j] = cheb(j, T);

  /* S2M, reference initg :242-259: initch[j][k] for leaf point j (box coordinate
   * (2j+1)/b - 1 in tan form) and node k. */
  {
    double a = FMM_PI / (2.0 * s), ta3 = 3 * tan(a);
    for (long j = 0; j < b; ++j) S.x[j] = tan(((double)(2 * (j + 1) - b - 1)) / (double)b * a);
    for (long j = 0; j < b; ++j)
      for (long k = 0; k < T; ++k)
        o->initch[j * T + k] = (o->chnods[k] + ta3 * S.x[j]) / (ta3 - o->chnods[k] * S.x[j]);
  }
  op_flip(&S, 2, 2, o->topflp); /* :279 */
  for (long lev = 1; lev <= nlev; ++lev) { /* :281-290 */
    double *L = o->levops + (lev - 1) * FMM_NLEVOPS * T * T;
    op_shift_up(&S, lev + 2, -1, L + FMM_SHFTFN * T * T);
    op_shift_up(&S, lev + 2, +1, L + FMM_SHFTFP * T * T);
    op_flip(&S, lev + 2, -2, L + FMM_FLIP2N * T * T);
    op_flip(&S, lev + 2, +2, L + FMM_FLIP2P * T * T);
    op_flip(&S, lev + 2, -3, L + FMM_FLIP3N * T * T);
    op_flip(&S, lev + 2, +3, L + FMM_FLIP3P * T * T);
    op_shift_down(&S, lev + 1, -1, L + FMM_SHFTLN * T * T);
    op_shift_down(&S, lev + 1, +1, L + FMM_SHFTLP * T * T);
  }
  double dlq = (double)M;
  for (long sc = 1; sc <= P - 1; ++sc) { /* :292-321 */
    double gfrac = ((double)sc) / P;
    for (long j = 1; j <= b; ++j) {
      double ffr = ((double)(2 * j - 1) - (((double)(2 * sc)) / P)) / b - 1;
      op_eval_point(&S, ffr, s, M, o->evalm + ((j - 1) * (P - 1) + (sc - 1)) * T);
    }
    if (sc >= P / 2) {
      double ffr = (((double)2 * b + 1) - ((double)2 * sc) / (P)) / (b)-1;
      op_eval_point(&S, ffr, s, M, o->evalmh + (sc - P / 2) * T);
    }
    /* The reference's three near-field tables cots/cotsh/cotprv all hold
     * -1/tan(pi/M (d + sc/P))/M for integer offsets d = source - target; one Toeplitz row
     * per section covers them (d in [-2b, 2b)). */
    for (long d = -2 * b; d < 2 * b; ++d)
      o->cot[(sc - 1) * 4 * b + d + 2 * b] = -1 / tan(FMM_PI / dlq * ((double)d + gfrac)) / dlq;
  }
  for (long sc = 1; sc <= P - 1; ++sc) { /* :325-331 */
    double ang = FMM_PI * ((double)sc) / P;
    for (long j = 1; j <= P; ++j) {
      double complex v = -cexp((ang * (1 - 2 * j)) * I) * sin(ang);
      o->fo[2 * ((j - 1) * (P - 1) + (sc - 1))] = creal(v);
      o->fo[2 * ((j - 1) * (P - 1) + (sc - 1)) + 1] = cimag(v);
    }
  }
  free(S.e), free(S.x), free(S.wgt);
  return 0;
}

long fmm_getwlen2(long lq, long terms, long p, long b) { /* reference :1160-1183 */
  if (!fmm_validate(lq, p, terms, b)) return -1;
  long n = lg2(lq / b);
  return 8 * (terms * terms * (n - 2)) + terms * terms + terms * b + terms * (p - 1) * b +
         terms * p / 2 + (3 * b * p) / 2 + 3 * b * (b - 1) * (p - 1) + (3 * b * p) / 2 + terms +
         2 * (p - 1) * p + p * (p - 1) + b + 3 * terms + 1;
}

long fmm_getvlen(long lq, long terms, long p, long b) { /* reference :1110-1135 */
  if (!fmm_validate(lq, p, terms, b)) return -1;
  long s = lq / b, t = s / p, n = lg2(s), l2p = lg2(p);
  long v = 2 * (2 * terms * (p - 1) * (2 * t + l2p - 3)) + 2 * (2 * p) + 3 * (2 * terms * (p - 1)) +
           2 * (2 * (p - 1) * (b + n * 2 * terms)) + 2 * (2 * ((p - 1) * (b + n * 2 * terms) + p / 2)) +
           2 * b * p + 2 * b * (p - 1) + 2 * (2 * (p / 2)) + 10 * (2 * terms * (p - 1)) +
           2 * (2 * terms * (p - 1) * 2 * n) + 2 * lq + 2 * (p - 1) + 2 * (2 * (p / 2));
  v = v + b + 3 * terms + 2 * (3 * p) + 1;
  return v;
}

/* Reference mfti layout, :343-374: 8 level tables, topflp, initch, evalm, evalmh, cotsh, cots,
 * cotprv, chnods, fo; the trailing scratch slots are zeroed. */
void fmm_ops64_to_reference_w(const fmm_ops64 *o, double *w) {
  const long T = o->T, b = o->b, P = o->P, n = o->n;
  long len = fmm_getwlen2(o->M, T, P, b), at = 0;
  memset(w, 0, sizeof(double) * (size_t)len);
  for (long op = 0; op < FMM_NLEVOPS; ++op) {
    for (long l = 0; l < n - 2; ++l)
      memcpy(w + at + l * T * T, o->levops + (l * FMM_NLEVOPS + op) * T * T, sizeof(double) * T * T);
    at += T * T * (n - 2);
  }
  memcpy(w + at, o->topflp, sizeof(double) * T * T), at += T * T;
  memcpy(w + at, o->initch, sizeof(double) * T * b), at += T * b;
  memcpy(w + at, o->evalm, sizeof(double) * T * (P - 1) * b), at += T * (P - 1) * b;
  memcpy(w + at, o->evalmh, sizeof(double) * T * (P / 2)), at += (T * P) / 2;
  for (long sce = 1; sce <= P / 2; ++sce) { /* cotsh: d = q - 2b */
    const double *ct = o->cot + (sce - 2 + P / 2) * 4 * b;
    for (long q = 0; q < 3 * b; ++q) w[at + (sce - 1) * 3 * b + q] = ct[q];
  }
  at += (3 * b * P) / 2;
  for (long sc = 1; sc <= P - 1; ++sc) { /* cots: row k (2..b), d = q - b + 1 - k */
    const double *ct = o->cot + (sc - 1) * 4 * b;
    for (long k = 2; k <= b; ++k)
      for (long q = 0; q < 3 * b; ++q) w[at + ((sc - 1) * (b - 1) + (k - 2)) * 3 * b + q] = ct[q + b + 1 - k];
  }
  at += 3 * b * (b - 1) * (P - 1);
  for (long sc = 1; sc <= P / 2; ++sc) { /* cotprv: d = q - b */
    const double *ct = o->cot + (sc - 1) * 4 * b;
    for (long q = 0; q < 3 * b; ++q) w[at + (sc - 1) * 3 * b + q] = ct[q + b];
  }
  at += (3 * b * P) / 2;
  memcpy(w + at, o->chnods, sizeof(double) * T), at += T;
  memcpy(w + at, o->fo, sizeof(double) * 2 * P * (P - 1));
}

/* ------------------------------------------------------------------ build into given storage */

/* Doubles fmm_ops64_build_in needs for (M, P, T, b): the operator tables plus the builder's
 * scratch.  -1 for unsupported parameters. */
long fmm_ops64_doubles(long M, long P, long T, long b) {
  if (!fmm_validate(M, P, T, b)) return -1;
  long s = M / b, n = lg2(s), nlev = n - 2 > 0 ? n - 2 : 1;
  return T + b * T + T * T + nlev * FMM_NLEVOPS * T * T + b * (P - 1) * T + (P / 2) * T +
         (P - 1) * 4 * b + 2 * P * (P - 1) + T + (T > b ? T : b) + T;
}

/* The same operators as fmm_ops64_build, written into `store` (cap doubles) instead of the
 * heap; o's arrays point into store and must not be passed to fmm_ops64_free. */
int fmm_ops64_build_in(long M, long P, long T, long b, fmm_ops64 *o, double *store, long cap) {
  memset(o, 0, sizeof(*o));
  long need = fmm_ops64_doubles(M, P, T, b);
  if (need < 0) return 1;
  if (need > cap) return 2;
  long s = M / b, n = lg2(s), nlev = n - 2 > 0 ? n - 2 : 1;
  o->M = M, o->P = P, o->T = T, o->b = b, o->s = s, o->n = n;
  double *at = store;
  o->chnods = at, at += T;
  o->initch = at, at += b * T;
  o->topflp = at, at += T * T;
  o->levops = at, at += nlev * FMM_NLEVOPS * T * T;
  o->evalm = at, at += b * (P - 1) * T;
  o->evalmh = at, at += (P / 2) * T;
  o->cot = at, at += (P - 1) * 4 * b;
  o->fo = at, at += 2 * P * (P - 1);
  op_scratch S = {T, o->chnods, NULL, NULL, NULL};
  S.e = at, at += T;
  S.x = at, at += (T > b ? T : b);
  S.wgt = at;
  for (long j = 0; j < T; ++j) o->chnods[j] = cheb(j, T);
  {
    double a = FMM_PI / (2.0 * s), ta3 = 3 * tan(a);
    for (long j = 0; j < b; ++j) S.x[j] = tan(((double)(2 * (j + 1) - b - 1)) / (double)b * a);
    for (long j = 0; j < b; ++j)
      for (long k = 0; k < T; ++k)
        o->initch[j * T + k] = (o->chnods[k] + ta3 * S.x[j]) / (ta3 - o->chnods[k] * S.x[j]);
  }
  op_flip(&S, 2, 2, o->topflp);
  for (long lev = 1; lev <= n - 2; ++lev) {
    double *L = o->levops + (lev - 1) * FMM_NLEVOPS * T * T;
    op_shift_up(&S, lev + 2, -1, L + FMM_SHFTFN * T * T);
    op_shift_up(&S, lev + 2, +1, L + FMM_SHFTFP * T * T);
    op_flip(&S, lev + 2, -2, L + FMM_FLIP2N * T * T);
    op_flip(&S, lev + 2, +2, L + FMM_FLIP2P * T * T);
    op_flip(&S, lev + 2, -3, L + FMM_FLIP3N * T * T);
    op_flip(&S, lev + 2, +3, L + FMM_FLIP3P * T * T);
    op_shift_down(&S, lev + 1, -1, L + FMM_SHFTLN * T * T);
    op_shift_down(&S, lev + 1, +1, L + FMM_SHFTLP * T * T);
  }
  double dlq = (double)M;
  for (long sc = 1; sc <= P - 1; ++sc) {
    double gfrac = ((double)sc) / P;
    for (long j = 1; j <= b; ++j) {
      double ffr = ((double)(2 * j - 1) - (((double)(2 * sc)) / P)) / b - 1;
      op_eval_point(&S, ffr, s, M, o->evalm + ((j - 1) * (P - 1) + (sc - 1)) * T);
    }
    if (sc >= P / 2) {
      double ffr = (((double)2 * b + 1) - ((double)2 * sc) / (P)) / (b)-1;
      op_eval_point(&S, ffr, s, M, o->evalmh + (sc - P / 2) * T);
    }
    for (long d = -2 * b; d < 2 * b; ++d)
      o->cot[(sc - 1) * 4 * b + d + 2 * b] = -1 / tan(FMM_PI / dlq * ((double)d + gfrac)) / dlq;
  }
  for (long sc = 1; sc <= P - 1; ++sc) {
    double ang = FMM_PI * ((double)sc) / P;
    for (long j = 1; j <= P; ++j) {
      double complex v = -cexp((ang * (1 - 2 * j)) * I) * sin(ang);
      o->fo[2 * ((j - 1) * (P - 1) + (sc - 1))] = creal(v);
      o->fo[2 * ((j - 1) * (P - 1) + (sc - 1)) + 1] = cimag(v);
    }
  }
  return 0;
}
