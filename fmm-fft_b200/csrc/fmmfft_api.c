/*
 * Public C-ABI of libfmmfft_b200.so (declared in include/fmmfft.h): the reference-compatible
 * entry points getwlen2 / getvlen / mfti / mft (src/fmmfft.c:1160, :1110, :337, :980) and the
 * native plan API.  Host code only; device work is delegated to fmmfft_kernels.cu.
 */
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/fmmfft.h"
#include "fmmfft_internal.h"

struct fmmfft_plan_s {
  long N, P, M, T, b;
  int precision;
  int max_transforms; /* batch capacity: transforms one execute may carry */
  size_t refine_bytes; /* FP64 companion plan + scratch of the residual pass, once enabled */
  size_t device_bytes;
  fmmk_state *dev;
};

/* ------------------------------------------------------------------ last error (per thread) */
static __thread int t_status = FMMFFT_OK;
static __thread char t_msg[256];

static int set_err(int status, const char *msg) {
  t_status = status;
  snprintf(t_msg, sizeof t_msg, "%s", msg ? msg : "");
  if (status != FMMFFT_OK && msg && getenv("FMMFFT_QUIET") == NULL)
    fprintf(stderr, "fmmfft: %s\n", msg);
  return status;
}

int fmmfft_last_error(void) { return t_status; }
const char *fmmfft_last_error_string(void) { return t_msg; }

/* ------------------------------------------------------------------ native API */
int fmmfft_plan_create(fmmfft_plan *out, long N, long P, long terms, long b, int precision) {
  return fmmfft_plan_create_batched(out, N, P, terms, b, precision, 1);
}

static int check_shape(long N, long P, long terms, long b, int precision, int nb) {
  if (precision < FMMFFT_F64 || precision > FMMFFT_BF16X3)
    return set_err(FMMFFT_ERR_INVALID, "plan_create: unknown precision");
  if (nb < 1 || nb > 64) return set_err(FMMFFT_ERR_INVALID, "plan_create: max_transforms outside 1..64");
  if (P < 2 || N <= 0 || N % P)
    return set_err(FMMFFT_ERR_INVALID, "plan_create: N must be a positive multiple of P >= 2");
  if (!fmm_validate(N / P, P, terms, b)) {
    char m[200];
    snprintf(m, sizeof m,
             "plan_create: unsupported (N=%ld, P=%ld, terms=%ld, b=%ld): need powers of two, "
             "2<=P<=1024, b>=2, M/b>=4, 2<=terms<=64, M<=2^26", N, P, terms, b);
    return set_err(FMMFFT_ERR_INVALID, m);
  }
  return FMMFFT_OK;
}

int fmmfft_plan_bytes(long N, long P, long terms, long b, int precision, int max_transforms,
                      size_t *bytes) {
  if (!bytes) return set_err(FMMFFT_ERR_INVALID, "plan_bytes: NULL output pointer");
  int rc = check_shape(N, P, terms, b, precision, max_transforms);
  if (rc) return rc;
  char err[256] = {0};
  rc = fmmk_plan_bytes(N / P, P, terms, b, precision, max_transforms, bytes, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_plan_create_batched(fmmfft_plan *out, long N, long P, long terms, long b, int precision,
                               int max_transforms) {
  if (!out) return set_err(FMMFFT_ERR_INVALID, "plan_create: NULL output pointer");
  *out = NULL;
  int rc0 = check_shape(N, P, terms, b, precision, max_transforms);
  if (rc0) return rc0;
  long M = N / P;
  fmm_ops64 ops;
  int rc = fmm_ops64_build(M, P, terms, b, &ops);
  if (rc) return set_err(FMMFFT_ERR_NOMEM, "plan_create: host allocation failed");
  struct fmmfft_plan_s *pl = (struct fmmfft_plan_s *)calloc(1, sizeof *pl);
  if (!pl) {
    fmm_ops64_free(&ops);
    return set_err(FMMFFT_ERR_NOMEM, "plan_create: host allocation failed");
  }
  char err[256] = {0};
  rc = fmmk_create_n(&ops, precision, max_transforms, &pl->dev, &pl->device_bytes, err, sizeof err);
  fmm_ops64_free(&ops);
  if (rc) {
    free(pl);
    return set_err(rc, err);
  }
  pl->N = N, pl->P = P, pl->M = M, pl->T = terms, pl->b = b, pl->precision = precision;
  pl->max_transforms = max_transforms;
  *out = pl;
  return set_err(FMMFFT_OK, NULL);
}

int fmmfft_plan_destroy(fmmfft_plan plan) {
  if (!plan) return FMMFFT_OK;
  fmmk_destroy(plan->dev);
  free(plan);
  return FMMFFT_OK;
}

int fmmfft_plan_device_bytes(fmmfft_plan plan, size_t *bytes) {
  if (!plan || !bytes) return set_err(FMMFFT_ERR_INVALID, "plan_device_bytes: NULL argument");
  *bytes = plan->device_bytes + plan->refine_bytes;
  return FMMFFT_OK;
}

static int exec_common(fmmfft_plan plan, const void *d_in, void *d_out, void *stream, int inv) {
  if (!plan || !d_in || !d_out) return set_err(FMMFFT_ERR_INVALID, "execute: NULL argument");
  char err[256] = {0};
  int rc = fmmk_execute(plan->dev, d_in, d_out, stream, inv, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_execute(fmmfft_plan plan, const void *d_in, void *d_out, void *stream) {
  return exec_common(plan, d_in, d_out, stream, 0);
}

int fmmfft_execute_inverse(fmmfft_plan plan, const void *d_in, void *d_out, void *stream) {
  return exec_common(plan, d_in, d_out, stream, 1);
}

int fmmfft_execute_many(fmmfft_plan plan, int count, const void *d_in, void *d_out, void *stream) {
  if (!plan || !d_in || !d_out) return set_err(FMMFFT_ERR_INVALID, "execute_many: NULL argument");
  if (count < 1 || count > plan->max_transforms)
    return set_err(FMMFFT_ERR_INVALID, "execute_many: count outside 1..max_transforms of the plan");
  char err[256] = {0};
  int rc = fmmk_execute_n(plan->dev, d_in, d_out, stream, 0, count, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_execute_many_ptrs(fmmfft_plan plan, int count, const void *const *d_ins, void *const *d_outs,
                             void *stream) {
  if (!plan || !d_ins || !d_outs) return set_err(FMMFFT_ERR_INVALID, "execute_many_ptrs: NULL argument");
  if (count < 1 || count > plan->max_transforms)
    return set_err(FMMFFT_ERR_INVALID, "execute_many_ptrs: count outside 1..max_transforms of the plan");
  for (int i = 0; i < count; ++i)
    if (!d_ins[i] || !d_outs[i]) return set_err(FMMFFT_ERR_INVALID, "execute_many_ptrs: NULL buffer");
  char err[256] = {0};
  int rc = fmmk_execute_ptrs(plan->dev, count, d_ins, d_outs, stream, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_execute_many_graph(fmmfft_plan plan, int count, const void *d_in, void *d_out, void *stream) {
  if (!plan || !d_in || !d_out) return set_err(FMMFFT_ERR_INVALID, "execute_many_graph: NULL argument");
  if (count < 1 || count > plan->max_transforms)
    return set_err(FMMFFT_ERR_INVALID, "execute_many_graph: count outside 1..max_transforms of the plan");
  char err[256] = {0};
  int rc = fmmk_execute_graph_n(plan->dev, d_in, d_out, stream, 0, count, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_plan_describe(fmmfft_plan plan, char *buf, size_t len) {
  if (!plan || !buf || len == 0) return set_err(FMMFFT_ERR_INVALID, "plan_describe: NULL argument");
  fmmk_describe(plan->dev, buf, len);
  return FMMFFT_OK;
}

int fmmfft_plan_enable_refinement(fmmfft_plan plan) {
  if (!plan) return set_err(FMMFFT_ERR_INVALID, "enable_refinement: NULL plan");
  if (plan->precision == FMMFFT_F64)
    return set_err(FMMFFT_ERR_INVALID, "enable_refinement: the plan is FP64 already");
  fmm_ops64 ops;
  if (fmm_ops64_build(plan->M, plan->P, plan->T, plan->b, &ops))
    return set_err(FMMFFT_ERR_NOMEM, "enable_refinement: host allocation failed");
  char err[256] = {0};
  size_t extra = 0;
  int rc = fmmk_refine_enable(plan->dev, &ops, &extra, err, sizeof err);
  fmm_ops64_free(&ops);
  if (rc) return set_err(rc, err);
  plan->refine_bytes = extra;
  return FMMFFT_OK;
}

int fmmfft_execute_refined(fmmfft_plan plan, const void *d_in, void *d_out, void *stream) {
  if (!plan || !d_in || !d_out) return set_err(FMMFFT_ERR_INVALID, "execute_refined: NULL argument");
  char err[256] = {0};
  int rc = fmmk_execute_refined(plan->dev, d_in, d_out, stream, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_execute_host(fmmfft_plan plan, const void *h_in, void *h_out, void *stream) {
  if (!plan || !h_in || !h_out) return set_err(FMMFFT_ERR_INVALID, "execute_host: NULL argument");
  char err[256] = {0};
  int rc = fmmk_execute_host(plan->dev, h_in, h_out, stream, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_execute_host_many(fmmfft_plan plan, int n, const void *const *h_in, void *const *h_out,
                             void *stream) {
  if (!plan || n < 0 || (n > 0 && (!h_in || !h_out)))
    return set_err(FMMFFT_ERR_INVALID, "execute_host_many: NULL argument or n < 0");
  for (int i = 0; i < n; ++i)
    if (!h_in[i] || !h_out[i]) return set_err(FMMFFT_ERR_INVALID, "execute_host_many: NULL buffer");
  char err[256] = {0};
  int rc = fmmk_execute_host_many(plan->dev, n, h_in, h_out, stream, err, sizeof err);
  return rc ? set_err(rc == 2 ? FMMFFT_ERR_NOMEM : FMMFFT_ERR_CUDA, err) : FMMFFT_OK;
}

int fmmfft_debug_fetch(fmmfft_plan plan, double *u, double *z, double *phi, double *psi) {
  if (!plan) return set_err(FMMFFT_ERR_INVALID, "debug_fetch: NULL plan");
  int rc = fmmk_debug_fetch(plan->dev, u, z, phi, psi);
  return rc ? set_err(FMMFFT_ERR_CUDA, "debug_fetch: copy failed") : FMMFFT_OK;
}

int fmmfft_profile_start(fmmfft_plan plan, int max_executes) {
  if (!plan) return set_err(FMMFFT_ERR_INVALID, "profile_start: NULL plan");
  int rc = fmmk_profile_start(plan->dev, max_executes);
  return rc ? set_err(rc == 1 ? FMMFFT_ERR_INVALID : FMMFFT_ERR_CUDA, "profile_start failed")
            : FMMFFT_OK;
}

int fmmfft_profile_stop(fmmfft_plan plan, double *stage_ms, int *stage_launches, int cap,
                        int *nstages, int *nexecutes) {
  if (!plan || !stage_ms || !stage_launches || !nstages)
    return set_err(FMMFFT_ERR_INVALID, "profile_stop: NULL argument");
  int n = fmmk_profile_stop(plan->dev, stage_ms, stage_launches, cap, nexecutes);
  if (n < 0) return set_err(FMMFFT_ERR_INVALID, "profile_stop: profiling was not started");
  *nstages = n;
  return FMMFFT_OK;
}

const char *fmmfft_stage_name(int i) { return fmmk_stage_name(i); }

int fmmfft_plan_check(fmmfft_plan plan) {
  if (!plan) return set_err(FMMFFT_ERR_INVALID, "plan_check: NULL plan");
  int rc = fmmk_check(plan->dev);
  if (rc == FMMFFT_ERR_TIMEOUT)
    return set_err(rc, "plan_check: a bounded wait in a tensor-core kernel gave up");
  return rc ? set_err(rc, "plan_check: CUDA error") : FMMFFT_OK;
}

int fmmfft_plan_selftest_wait(fmmfft_plan plan, int which, long limit_us) {
  if (!plan || which != 0 || limit_us < 1 || limit_us > 2000000)
    return set_err(FMMFFT_ERR_INVALID, "plan_selftest_wait: which must be 0, limit 1..2e6 us");
  char err[256] = {0};
  int rc = fmmk_selftest_wait(plan->dev, which, limit_us, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_execute_graph(fmmfft_plan plan, const void *d_in, void *d_out, void *stream) {
  if (!plan || !d_in || !d_out) return set_err(FMMFFT_ERR_INVALID, "execute_graph: NULL argument");
  char err[256] = {0};
  int rc = fmmk_execute_graph(plan->dev, d_in, d_out, stream, 0, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

/* ------------------------------------------------------------------ batches */
struct fmmfft_batch_s {
  void *exec;
  int n, nbranch;
};

int fmmfft_batch_create(fmmfft_batch *out, const fmmfft_plan *plans, const void *const *d_in,
                        void *const *d_out, int n, int nbranch) {
  return fmmfft_batch_create_many(out, plans, NULL, d_in, d_out, n, nbranch);
}

int fmmfft_batch_create_many(fmmfft_batch *out, const fmmfft_plan *plans, const int *counts,
                             const void *const *d_in, void *const *d_out, int n, int nbranch) {
  if (!out || !plans || !d_in || !d_out || n < 1 || nbranch < 1 || nbranch > 64)
    return set_err(FMMFFT_ERR_INVALID, "batch_create: bad arguments");
  if (counts)
    for (int i = 0; i < n; ++i)
      if (!plans[i] || counts[i] < 1 || counts[i] > plans[i]->max_transforms)
        return set_err(FMMFFT_ERR_INVALID, "batch_create: count outside 1..max_transforms of its plan");
  *out = NULL;
  fmmk_state **sts = (fmmk_state **)calloc((size_t)n, sizeof(fmmk_state *));
  int *branch = (int *)calloc((size_t)n, sizeof(int));
  double *load = (double *)calloc((size_t)nbranch, sizeof(double));
  struct fmmfft_batch_s *b = (struct fmmfft_batch_s *)calloc(1, sizeof *b);
  if (!sts || !branch || !load || !b) {
    free(sts), free(branch), free(load), free(b);
    return set_err(FMMFFT_ERR_NOMEM, "batch_create: allocation failed");
  }
  /* every transform of one plan goes to the branch its plan first went to (shared workspace);
   * a new plan goes to the branch with the least work so far */
  for (int i = 0; i < n; ++i) {
    if (!plans[i]) {
      free(sts), free(branch), free(load), free(b);
      return set_err(FMMFFT_ERR_INVALID, "batch_create: NULL plan");
    }
    sts[i] = plans[i]->dev;
    int br = -1;
    for (int j = 0; j < i && br < 0; ++j)
      if (plans[j] == plans[i]) br = branch[j];
    if (br < 0) {
      br = 0;
      for (int k = 1; k < nbranch; ++k)
        if (load[k] < load[br]) br = k;
    }
    branch[i] = br;
    load[br] += (double)plans[i]->N * (counts ? counts[i] : 1);
  }
  char err[256] = {0};
  int rc = fmmk_batch_capture(sts, d_in, d_out, NULL, counts, branch, n, nbranch, &b->exec, err, sizeof err);
  free(sts), free(branch), free(load);
  if (rc) {
    free(b);
    return set_err(rc, err);
  }
  b->n = n, b->nbranch = nbranch;
  *out = b;
  return set_err(FMMFFT_OK, NULL);
}

int fmmfft_batch_launch(fmmfft_batch batch, void *stream) {
  if (!batch) return set_err(FMMFFT_ERR_INVALID, "batch_launch: NULL batch");
  return fmmk_batch_launch(batch->exec, stream) ? set_err(FMMFFT_ERR_CUDA, "batch_launch failed")
                                                : FMMFFT_OK;
}

int fmmfft_batch_destroy(fmmfft_batch batch) {
  if (!batch) return FMMFFT_OK;
  fmmk_batch_free(batch->exec);
  free(batch);
  return FMMFFT_OK;
}

/* ------------------------------------------------------------------ allocation-free entry */

/* FP64 operator tables for fmmfft_execute_noalloc, built in this file-scope store (no heap):
 * 2^21 doubles (16 MiB) of host memory, enough for every size the 32 MiB device array holds. */
#define FMMFFT_NOALLOC_OPS_DOUBLES (1L << 21)
static double g_na_store[FMMFFT_NOALLOC_OPS_DOUBLES];
static fmm_ops64 g_na_ops;
static long g_na_key[4];
static pthread_mutex_t g_na_mu = PTHREAD_MUTEX_INITIALIZER;

int fmmfft_execute_noalloc(long N, long P, long terms, long b, const void *d_in, void *d_out,
                           void *stream) {
  if (!d_in || !d_out) return set_err(FMMFFT_ERR_INVALID, "execute_noalloc: NULL argument");
  if (P < 2 || N <= 0 || N % P || !fmm_validate(N / P, P, terms, b))
    return set_err(FMMFFT_ERR_INVALID, "execute_noalloc: unsupported parameters");
  long M = N / P, key[4] = {M, P, terms, b};
  char err[256] = {0};
  pthread_mutex_lock(&g_na_mu);
  if (memcmp(key, g_na_key, sizeof key) != 0) {
    memset(g_na_key, 0, sizeof g_na_key);
    int rc = fmm_ops64_build_in(M, P, terms, b, &g_na_ops, g_na_store, FMMFFT_NOALLOC_OPS_DOUBLES);
    if (rc) {
      pthread_mutex_unlock(&g_na_mu);
      return set_err(FMMFFT_ERR_INVALID,
                     "execute_noalloc: operator tables exceed the allocation-free limit");
    }
    memcpy(g_na_key, key, sizeof key);
  }
  int rc = fmmk_execute_noalloc(&g_na_ops, 1, d_in, d_out, stream, err, sizeof err);
  pthread_mutex_unlock(&g_na_mu);
  return rc ? set_err(rc == 1 ? FMMFFT_ERR_INVALID : rc, err) : set_err(FMMFFT_OK, NULL);
}

/* ------------------------------------------------------------------ reference-compatible */

/* Device plans made by mfti, keyed by (lq, p, terms, b), kept until process exit: mft finds
 * the plan mfti made for the same parameters, as the reference's mft reuses mfti's w. */
typedef struct compat_entry {
  long lq, p, terms, b;
  fmmfft_plan plan;
  struct compat_entry *next;
} compat_entry;
static compat_entry *g_compat = NULL;
static pthread_mutex_t g_compat_mu = PTHREAD_MUTEX_INITIALIZER;

static fmmfft_plan compat_plan(long lq, long p, long terms, long b, int *status) {
  pthread_mutex_lock(&g_compat_mu);
  for (compat_entry *e = g_compat; e; e = e->next)
    if (e->lq == lq && e->p == p && e->terms == terms && e->b == b) {
      pthread_mutex_unlock(&g_compat_mu);
      *status = FMMFFT_OK;
      return e->plan;
    }
  fmmfft_plan pl = NULL;
  *status = fmmfft_plan_create(&pl, lq * p, p, terms, b, FMMFFT_F64);
  if (*status == FMMFFT_OK) {
    compat_entry *e = (compat_entry *)calloc(1, sizeof *e);
    if (!e) {
      fmmfft_plan_destroy(pl);
      pthread_mutex_unlock(&g_compat_mu);
      *status = set_err(FMMFFT_ERR_NOMEM, "compat plan cache: allocation failed");
      return NULL;
    }
    *e = (compat_entry){lq, p, terms, b, pl, g_compat};
    g_compat = e;
  }
  pthread_mutex_unlock(&g_compat_mu);
  return pl;
}

long getwlen2(long lq, long terms, long p, long b) {
  long v = fmm_getwlen2(lq, terms, p, b);
  set_err(v < 0 ? FMMFFT_ERR_INVALID : FMMFFT_OK, v < 0 ? "getwlen2: unsupported parameters" : NULL);
  return v;
}

long getvlen(long lq, long terms, long p, long b) {
  long v = fmm_getvlen(lq, terms, p, b);
  set_err(v < 0 ? FMMFFT_ERR_INVALID : FMMFFT_OK, v < 0 ? "getvlen: unsupported parameters" : NULL);
  return v;
}

void mfti(long lq, long p, long terms, long b, double *w, double *v, long szkeep, long sztemp) {
  (void)v, (void)szkeep, (void)sztemp;
  if (!fmm_validate(lq, p, terms, b)) {
    set_err(FMMFFT_ERR_INVALID, "mfti: unsupported parameters");
    return;
  }
  if (w) {
    fmm_ops64 ops;
    if (fmm_ops64_build(lq, p, terms, b, &ops)) {
      set_err(FMMFFT_ERR_NOMEM, "mfti: host allocation failed");
      return;
    }
    fmm_ops64_to_reference_w(&ops, w);
    fmm_ops64_free(&ops);
  }
  int st;
  compat_plan(lq, p, terms, b, &st);
  if (st == FMMFFT_OK) set_err(FMMFFT_OK, NULL);
}

/* ------------------------------------------------------------------ block-distributed I/O */
int fmmfft_execute_blocks(fmmfft_plan plan, const void *const *d_blocks_in, void *const *d_blocks_out,
                          void *stream) {
  if (!plan || !d_blocks_in || !d_blocks_out)
    return set_err(FMMFFT_ERR_INVALID, "execute_blocks: NULL argument");
  for (long r = 0; r < plan->P; ++r)
    if (!d_blocks_in[r] || !d_blocks_out[r]) return set_err(FMMFFT_ERR_INVALID, "execute_blocks: NULL block");
  char err[256] = {0};
  int rc = fmmk_execute_blocks(plan->dev, d_blocks_in, d_blocks_out, 0, stream, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_execute_blocks_host(fmmfft_plan plan, const void *const *h_blocks_in, void *const *h_blocks_out,
                               void *stream) {
  if (!plan || !h_blocks_in || !h_blocks_out)
    return set_err(FMMFFT_ERR_INVALID, "execute_blocks_host: NULL argument");
  for (long r = 0; r < plan->P; ++r)
    if (!h_blocks_in[r] || !h_blocks_out[r])
      return set_err(FMMFFT_ERR_INVALID, "execute_blocks_host: NULL block");
  char err[256] = {0};
  int rc = fmmk_execute_blocks(plan->dev, h_blocks_in, h_blocks_out, 1, stream, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

/* Rank mode of mft: the p calling threads (myid = 0 .. p-1) meet, as the reference's ranks do in
 * their collectives; the last to arrive runs the transform over every rank's block and all
 * return with their block transformed.  One collective at a time, like MPI_COMM_WORLD. */
static int g_rank_mode = 0;
static pthread_mutex_t g_meet_mu = PTHREAD_MUTEX_INITIALIZER;
static pthread_cond_t g_meet_cv = PTHREAD_COND_INITIALIZER;
static struct {
  int active;
  long lq, p, terms, b;
  void **blocks;
  long arrived;
  unsigned long gen;
  int status;
  char msg[256];
} g_meet;

int fmmfft_mft_rank_mode(int on) {
  pthread_mutex_lock(&g_meet_mu);
  int busy = g_meet.active;
  if (!busy) g_rank_mode = on != 0;
  pthread_mutex_unlock(&g_meet_mu);
  return busy ? set_err(FMMFFT_ERR_BUSY, "mft_rank_mode: a collective mft is in progress") : FMMFFT_OK;
}

static long rank_timeout_ms(void) {
  const char *ev = getenv("FMMFFT_RANK_TIMEOUT_MS");
  long v = ev ? atol(ev) : 0;
  return v > 0 ? v : 120000;
}

static void mft_rank(long lq, void *qr, long p, long myid, long terms, long b) {
  if (myid < 0 || myid >= p) {
    set_err(FMMFFT_ERR_INVALID, "mft: myid outside 0..p-1");
    return;
  }
  pthread_mutex_lock(&g_meet_mu);
  if (!g_meet.active) {
    g_meet.blocks = (void **)calloc((size_t)p, sizeof(void *));
    if (!g_meet.blocks) {
      pthread_mutex_unlock(&g_meet_mu);
      set_err(FMMFFT_ERR_NOMEM, "mft: host allocation failed");
      return;
    }
    g_meet.active = 1, g_meet.lq = lq, g_meet.p = p, g_meet.terms = terms, g_meet.b = b;
    g_meet.arrived = 0;
  } else if (g_meet.lq != lq || g_meet.p != p || g_meet.terms != terms || g_meet.b != b) {
    pthread_mutex_unlock(&g_meet_mu);
    set_err(FMMFFT_ERR_INVALID, "mft: ranks called with different (lq, p, terms, b)");
    return;
  }
  if (g_meet.blocks[myid]) {
    pthread_mutex_unlock(&g_meet_mu);
    set_err(FMMFFT_ERR_INVALID, "mft: two calls with the same myid in one collective");
    return;
  }
  g_meet.blocks[myid] = qr;
  const unsigned long my_gen = g_meet.gen;
  int status;
  char msg[256];
  if (++g_meet.arrived == p) {
    void **blocks = g_meet.blocks;
    pthread_mutex_unlock(&g_meet_mu);
    int st;
    fmmfft_plan pl = compat_plan(lq, p, terms, b, &st);
    if (pl) st = fmmfft_execute_blocks_host(pl, (const void *const *)blocks, blocks, NULL);
    pthread_mutex_lock(&g_meet_mu);
    g_meet.status = st;
    snprintf(g_meet.msg, sizeof g_meet.msg, "%s", st ? fmmfft_last_error_string() : "");
    free(g_meet.blocks);
    g_meet.blocks = NULL;
    g_meet.active = 0;
    g_meet.gen++;
    pthread_cond_broadcast(&g_meet_cv);
    status = st;
    snprintf(msg, sizeof msg, "%s", g_meet.msg);
  } else {
    struct timespec dl;
    clock_gettime(CLOCK_REALTIME, &dl);
    const long ms = rank_timeout_ms();
    dl.tv_sec += ms / 1000, dl.tv_nsec += (ms % 1000) * 1000000L;
    if (dl.tv_nsec >= 1000000000L) dl.tv_sec++, dl.tv_nsec -= 1000000000L;
    int w = 0;
    while (g_meet.gen == my_gen && w == 0) w = pthread_cond_timedwait(&g_meet_cv, &g_meet_mu, &dl);
    if (g_meet.gen == my_gen) { /* the other ranks never came: withdraw this rank's block */
      g_meet.blocks[myid] = NULL;
      if (--g_meet.arrived == 0) {
        free(g_meet.blocks);
        g_meet.blocks = NULL;
        g_meet.active = 0;
      }
      status = FMMFFT_ERR_TIMEOUT;
      snprintf(msg, sizeof msg, "mft: not every rank of the collective called within the time limit");
    } else {
      status = g_meet.status;
      snprintf(msg, sizeof msg, "%s", g_meet.msg);
    }
  }
  pthread_mutex_unlock(&g_meet_mu);
  set_err(status, status ? msg : NULL);
}

void mft(long lq, void *qr, long dir, long p, long myid, long terms, long b, double *w, double *v,
         long sz1, long szwk, void *forward_plan) {
  (void)w, (void)v, (void)sz1, (void)szwk, (void)forward_plan;
  if (!qr) {
    set_err(FMMFFT_ERR_INVALID, "mft: NULL qr");
    return;
  }
  if (dir < 0) {
    set_err(FMMFFT_ERR_UNSUPPORTED,
            "mft: dir < 0 is not served (the reference's inverse conjugates before its local "
            "FFT, src/fmmfft.c:976-977 vs :1080); use fmmfft_execute_inverse");
    return;
  }
  if (!fmm_validate(lq, p, terms, b)) {
    set_err(FMMFFT_ERR_INVALID, "mft: unsupported parameters");
    return;
  }
  if (g_rank_mode) {
    mft_rank(lq, qr, p, myid, terms, b);
    return;
  }
  (void)myid;
  int st;
  fmmfft_plan pl = compat_plan(lq, p, terms, b, &st);
  if (!pl) return;
  st = fmmfft_execute_host(pl, qr, qr, NULL);
  if (st == FMMFFT_OK) set_err(FMMFFT_OK, NULL);
}

/* ------------------------------------------------------------------ plain FFT comparator */

struct fmmfft_fft_s {
  fmmk_fft *dev;
  size_t bytes;
};

int fmmfft_fft_create(fmmfft_fft *out, long N, int precision) {
  if (!out) return set_err(FMMFFT_ERR_INVALID, "fft_create: NULL output pointer");
  *out = NULL;
  if (precision < FMMFFT_F64 || precision > FMMFFT_BF16X3)
    return set_err(FMMFFT_ERR_INVALID, "fft_create: unknown precision");
  struct fmmfft_fft_s *f = (struct fmmfft_fft_s *)calloc(1, sizeof *f);
  if (!f) return set_err(FMMFFT_ERR_NOMEM, "fft_create: host allocation failed");
  char err[256] = {0};
  int rc = fmmk_fft_create(N, precision == FMMFFT_F64, &f->dev, &f->bytes, err, sizeof err);
  if (rc) {
    free(f);
    return set_err(rc, err);
  }
  *out = f;
  return set_err(FMMFFT_OK, NULL);
}

int fmmfft_fft_execute(fmmfft_fft f, const void *d_in, void *d_out, void *stream) {
  if (!f || !d_in || !d_out) return set_err(FMMFFT_ERR_INVALID, "fft_execute: NULL argument");
  char err[256] = {0};
  int rc = fmmk_fft_execute(f->dev, d_in, d_out, stream, err, sizeof err);
  return rc ? set_err(rc, err) : FMMFFT_OK;
}

int fmmfft_fft_device_bytes(fmmfft_fft f, size_t *bytes) {
  if (!f || !bytes) return set_err(FMMFFT_ERR_INVALID, "fft_device_bytes: NULL argument");
  *bytes = f->bytes;
  return FMMFFT_OK;
}

int fmmfft_fft_destroy(fmmfft_fft f) {
  if (!f) return FMMFFT_OK;
  fmmk_fft_destroy(f->dev);
  free(f);
  return FMMFFT_OK;
}

/* ------------------------------------------------------------------ sharded transform */
struct fmmfft_shard_s {
  fmmk_shard *sh;
  int phase; /* the next phase to run */
};

int fmmfft_shard_create(fmmfft_shard *out, long N, long P, long terms, long b, int precision, int G, int g) {
  if (!out) return set_err(FMMFFT_ERR_INVALID, "shard_create: NULL output pointer");
  *out = NULL;
  int rc0 = check_shape(N, P, terms, b, precision, 1);
  if (rc0) return rc0;
  fmm_ops64 ops;
  if (fmm_ops64_build(N / P, P, terms, b, &ops)) return set_err(FMMFFT_ERR_NOMEM, "shard_create: host allocation failed");
  struct fmmfft_shard_s *s = (struct fmmfft_shard_s *)calloc(1, sizeof *s);
  if (!s) {
    fmm_ops64_free(&ops);
    return set_err(FMMFFT_ERR_NOMEM, "shard_create: host allocation failed");
  }
  char err[256] = {0};
  int rc = fmmk_shard_create(&ops, precision, G, g, &s->sh, err, sizeof err);
  fmm_ops64_free(&ops);
  if (rc) {
    free(s);
    return set_err(rc, err);
  }
  *out = s;
  return set_err(FMMFFT_OK, NULL);
}

int fmmfft_shard_buffers(fmmfft_shard sh, fmmfft_shard_bufs *bufs) {
  if (!sh || !bufs) return set_err(FMMFFT_ERR_INVALID, "shard_buffers: NULL argument");
  void *p[7];
  size_t c[5];
  fmmk_shard_buffers(sh->sh, p, c);
  bufs->x_ext = p[0], bufs->sums = p[1], bufs->phi_send = p[2], bufs->phi_all = p[3];
  bufs->z_send = p[4], bufs->z_recv = p[5], bufs->y = p[6];
  bufs->x_ext_elems = c[0], bufs->halo_elems = c[1], bufs->phi_elems = c[2], bufs->z_elems = c[3];
  bufs->y_elems = c[4];
  return FMMFFT_OK;
}

int fmmfft_shard_phase(fmmfft_shard sh, int phase, void *stream) {
  if (!sh) return set_err(FMMFFT_ERR_INVALID, "shard_phase: NULL shard");
  if (phase != sh->phase) return set_err(FMMFFT_ERR_INVALID, "shard_phase: phases run in the order 0, 1, 2");
  char err[256] = {0};
  int rc = fmmk_shard_phase(sh->sh, phase, stream, err, sizeof err);
  if (rc) return set_err(rc, err);
  sh->phase = (phase + 1) % 3;
  return FMMFFT_OK;
}

int fmmfft_shard_destroy(fmmfft_shard sh) {
  if (!sh) return FMMFFT_OK;
  fmmk_shard_destroy(sh->sh);
  free(sh);
  return FMMFFT_OK;
}
