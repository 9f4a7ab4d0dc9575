/*
 * Request server of the FMM-FFT with continuous batching.  No counterpart in the reference,
 * which runs one transform per mpirun.
 *
 *  - Lanes: one per request shape (N, P, terms, b, precision).  A lane owns up to
 *    SRV_LANE_PLANS resident plans, each on its own CUDA stream; small shapes get batched plans
 *    (capacity nbmax = SRV_BATCH_SAMPLES / N, at most SRV_MAX_BATCH) with contiguous staging
 *    buffers, shapes of SRV_PTR_MIN_N samples or more batched plans of SRV_PTR_BATCH that read and
 *    write the requests' own buffers (fmmfft_execute_many_ptrs).
 *  - Continuous batching: a request is queued on its lane; whenever one of the lane's plans is
 *    idle, every queued request (up to the plan's capacity) leaves in ONE launch sequence: their
 *    inputs are copied into the plan's staging buffer, the batched transform runs as one cached
 *    CUDA graph (fmmfft_execute_many_graph: each tree stage one contraction over the rows of all
 *    of them), and each output is copied back to its request's buffer.  Requests that arrive
 *    while a batch runs gather for the next one, and the lanes' streams overlap on the device.
 *    Shapes with nbmax = 1 run each request on its own buffers, directly.
 *  - A dispatcher thread keeps batches leaving as plans free up; submit, query and wait also
 *    dispatch, so a caller that polls never waits for it.
 *  - Admission by HBM budget: a plan's device bytes are computed BEFORE anything is allocated
 *    (fmmfft_plan_bytes); to make room, idle plans with no queued work are evicted least-
 *    recently-used.  A request whose shape has no plan and cannot get one even after eviction is
 *    refused with FMMFFT_ERR_BUSY, allocating nothing.  Plans are built (FP64 operators on the
 *    host, then the device upload) outside the server lock, so a new shape does not stall the
 *    other lanes.
 *  - Results do not depend on the mix: a batched transform gives bitwise the output of its own
 *    execute (tests/test_gpu_batched.py), and the arithmetic of a plan does not depend on what
 *    else runs.
 */
#include <cuda_runtime_api.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/fmmfft.h"

#define SRV_MAX_LANES 256
#define SRV_LANE_PLANS 3
#define SRV_MAX_BATCH 32
/* a batch carries about this many samples: measured on a B200 (split TF32, P = 64, 20 terms),
 * batches of 4 x 2^22 run at 17.0 G samples/s against 13.4 for one 2^22 transform, 2 x 2^23 at
 * 17.9 against 16.2; a batch of 2 x 2^24 gains 6% (0.93 -> 0.87 ms a transform), about what
 * its staging copies (4 x 128 MB a transform) cost, so 2^24 requests run alone */
#define SRV_BATCH_SAMPLES (1L << 24)
/* Shapes of at least SRV_PTR_MIN_N samples batch through fmmfft_execute_many_ptrs: each request
 * is read and written in its own buffers (no staging copies, no graph: at these sizes a batch runs
 * for milliseconds and its launches are a small part of that), up to SRV_PTR_BATCH requests */
#define SRV_PTR_MIN_N (1L << 22)
#define SRV_PTR_BATCH 4
#define SRV_TICKETS 65536            /* outstanding tickets a server tracks (a ring) */

typedef struct {
  fmmfft_plan plan;
  cudaStream_t st;
  void *bin, *bout;     /* staging buffers of batched plans: nbmax transforms each */
  cudaEvent_t done;     /* completion of the plan's last batch */
  int busy;
  size_t bytes;         /* plan + staging */
  unsigned long long last_use;
} srv_plan;

typedef struct {
  long N, P, T, b;
  int prec;
  int nbmax;
  int ptrs;             /* batches through per-request buffers (no staging) */
  size_t plan_bytes;    /* one plan of this lane with its staging, computed before allocating */
  int nplans, creating;
  srv_plan p[SRV_LANE_PLANS];
  int *queue;           /* ring of ticket slots, SRV_TICKETS entries */
  long qhead, qlen;
} srv_lane;

typedef struct {
  fmmfft_ticket id;
  const void *in;
  void *out;
  int lane;
  int state;            /* 0 free, 1 queued, 2 dispatched, 3 done, 4 failed to launch */
  cudaEvent_t ev;
  int has_ev;
} srv_ticket;

struct fmmfft_server_s {
  pthread_mutex_t mu;
  pthread_t pump;
  volatile int stop;
  int device;
  size_t budget, used;  /* used: plans + staging held or reserved */
  int nstreams;         /* plans (streams) per lane, at most SRV_LANE_PLANS */
  srv_lane lanes[SRV_MAX_LANES];
  int nlanes;
  srv_ticket *tickets;
  fmmfft_ticket next_ticket;
  unsigned long long clock;
  unsigned long long dispatched, launches; /* requests sent to the GPU, batches they went in */
};

static size_t elem_bytes(int prec) { return prec == FMMFFT_F64 ? 16 : 8; }

static int plan_idle(srv_plan *p) {
  if (!p->busy) return 1;
  if (cudaEventQuery(p->done) == cudaSuccess) p->busy = 0;
  return !p->busy;
}

static void free_plan(srv_plan *p) {
  if (p->st) cudaStreamSynchronize(p->st);
  if (p->done) cudaEventDestroy(p->done);
  if (p->st) cudaStreamDestroy(p->st);
  if (p->bin) cudaFree(p->bin);
  if (p->bout) cudaFree(p->bout);
  if (p->plan) fmmfft_plan_destroy(p->plan);
  memset(p, 0, sizeof *p);
}

/* Evict the least recently used idle plan of a lane with no queued work (not `keep`); 1 when one
 * was evicted.  Called with the lock held. */
static int evict_one(struct fmmfft_server_s *s, int keep) {
  int bl = -1, bp = -1;
  for (int l = 0; l < s->nlanes; ++l) {
    srv_lane *ln = &s->lanes[l];
    if (l == keep || ln->qlen > 0 || ln->creating) continue;
    for (int i = 0; i < ln->nplans; ++i)
      if (plan_idle(&ln->p[i]) && (bl < 0 || ln->p[i].last_use < s->lanes[bl].p[bp].last_use)) bl = l, bp = i;
  }
  if (bl < 0) return 0;
  srv_lane *ln = &s->lanes[bl];
  s->used -= ln->p[bp].bytes;
  free_plan(&ln->p[bp]);
  ln->p[bp] = ln->p[--ln->nplans];
  memset(&ln->p[ln->nplans], 0, sizeof(srv_plan));
  return 1;
}

/* Sends queued requests of lane l to its idle plans, one batch per plan.  Lock held. */
static void dispatch_lane(struct fmmfft_server_s *s, int l) {
  srv_lane *ln = &s->lanes[l];
  const size_t nbytes = (size_t)ln->N * elem_bytes(ln->prec);
  for (int i = 0; i < ln->nplans && ln->qlen > 0; ++i) {
    srv_plan *p = &ln->p[i];
    if (!plan_idle(p)) continue;
    /* a power of two: each plan caches one graph per batch size, so a handful of sizes keeps
     * every batch a single graph launch; the rest waits for the lane's next idle plan */
    int k = 1;
    while (2 * k <= ln->qlen && 2 * k <= ln->nbmax) k *= 2;
    if (ln->ptrs) k = ln->qlen < ln->nbmax ? ln->qlen : ln->nbmax; /* no graph per size */
    int rc = FMMFFT_OK;
    if (ln->ptrs) {
      const void *ins[SRV_PTR_BATCH];
      void *outs[SRV_PTR_BATCH];
      for (int j = 0; j < k; ++j) {
        srv_ticket *tk = &s->tickets[ln->queue[(ln->qhead + j) % SRV_TICKETS]];
        ins[j] = tk->in, outs[j] = tk->out;
      }
      rc = fmmfft_execute_many_ptrs(p->plan, k, ins, outs, p->st);
    } else if (ln->nbmax == 1) {
      srv_ticket *tk = &s->tickets[ln->queue[ln->qhead % SRV_TICKETS]];
      rc = fmmfft_execute(p->plan, tk->in, tk->out, p->st);
    } else {
      for (int j = 0; j < k && rc == FMMFFT_OK; ++j) {
        srv_ticket *tk = &s->tickets[ln->queue[(ln->qhead + j) % SRV_TICKETS]];
        if (cudaMemcpyAsync((char *)p->bin + j * nbytes, tk->in, nbytes, cudaMemcpyDeviceToDevice, p->st) !=
            cudaSuccess)
          rc = FMMFFT_ERR_CUDA;
      }
      if (rc == FMMFFT_OK) rc = fmmfft_execute_many_graph(p->plan, k, p->bin, p->bout, p->st);
    }
    for (int j = 0; j < k; ++j) {
      const int slot = ln->queue[(ln->qhead + j) % SRV_TICKETS];
      srv_ticket *tk = &s->tickets[slot];
      if (rc != FMMFFT_OK) {
        tk->state = 4;
        continue;
      }
      if (ln->nbmax > 1 && !ln->ptrs)
        cudaMemcpyAsync(tk->out, (char *)p->bout + j * nbytes, nbytes, cudaMemcpyDeviceToDevice, p->st);
      if (!tk->has_ev) {
        cudaEventCreateWithFlags(&tk->ev, cudaEventDisableTiming);
        tk->has_ev = 1;
      }
      cudaEventRecord(tk->ev, p->st);
      tk->state = 2;
    }
    cudaEventRecord(p->done, p->st);
    s->dispatched += (unsigned long long)k, s->launches += 1;
    p->busy = 1;
    p->last_use = ++s->clock;
    ln->qhead += k, ln->qlen -= k;
  }
}

static void dispatch_all(struct fmmfft_server_s *s) {
  for (int l = 0; l < s->nlanes; ++l)
    if (s->lanes[l].qlen > 0) dispatch_lane(s, l);
}

/* Builds one more plan for lane l if it has queued work, every plan of it is busy, it has fewer
 * than SRV_LANE_PLANS and the budget allows (after evicting idle plans).  The plan is built with
 * the lock released; `used` holds the reservation meanwhile.  Lock held on entry and exit. */
static void grow_lane(struct fmmfft_server_s *s, int l) {
  srv_lane *ln = &s->lanes[l];
  const int cap = s->nstreams < SRV_LANE_PLANS ? s->nstreams : SRV_LANE_PLANS;
  if (ln->qlen == 0 || ln->creating || ln->nplans >= cap) return;
  for (int i = 0; i < ln->nplans; ++i)
    if (plan_idle(&ln->p[i])) return;
  while (s->used + ln->plan_bytes > s->budget && evict_one(s, l)) {
  }
  if (s->used + ln->plan_bytes > s->budget) return;
  s->used += ln->plan_bytes;
  ln->creating = 1;
  const long N = ln->N, P = ln->P, T = ln->T, b = ln->b;
  const int prec = ln->prec, nb = ln->nbmax, ptrs = ln->ptrs;
  pthread_mutex_unlock(&s->mu);
  srv_plan np;
  memset(&np, 0, sizeof np);
  int ok = fmmfft_plan_create_batched(&np.plan, N, P, T, b, prec, nb) == FMMFFT_OK;
  ok = ok && cudaStreamCreateWithFlags(&np.st, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaEventCreateWithFlags(&np.done, cudaEventDisableTiming) == cudaSuccess;
  if (ok && nb > 1 && !ptrs) {
    const size_t bytes = (size_t)nb * (size_t)N * elem_bytes(prec);
    ok = cudaMalloc(&np.bin, bytes) == cudaSuccess && cudaMalloc(&np.bout, bytes) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    free_plan(&np);
  }
  pthread_mutex_lock(&s->mu);
  ln = &s->lanes[l];
  ln->creating = 0;
  if (!ok) {
    s->used -= ln->plan_bytes;
    return;
  }
  np.bytes = ln->plan_bytes;
  ln->p[ln->nplans++] = np;
}

static void pump_once(struct fmmfft_server_s *s) {
  dispatch_all(s);
  for (int l = 0; l < s->nlanes; ++l) grow_lane(s, l);
  dispatch_all(s);
}

static void *pump_main(void *arg) {
  struct fmmfft_server_s *s = (struct fmmfft_server_s *)arg;
  cudaSetDevice(s->device);
  while (!s->stop) {
    pthread_mutex_lock(&s->mu);
    pump_once(s);
    pthread_mutex_unlock(&s->mu);
    struct timespec nap = {0, 10000}; /* 10 us */
    nanosleep(&nap, NULL);
  }
  return NULL;
}

int fmmfft_server_create(fmmfft_server *out, size_t hbm_budget_bytes, int nstreams) {
  if (!out || nstreams < 1 || nstreams > 64) return FMMFFT_ERR_INVALID;
  struct fmmfft_server_s *s = (struct fmmfft_server_s *)calloc(1, sizeof *s);
  if (!s) return FMMFFT_ERR_NOMEM;
  s->tickets = (srv_ticket *)calloc(SRV_TICKETS, sizeof(srv_ticket));
  if (!s->tickets) {
    free(s);
    return FMMFFT_ERR_NOMEM;
  }
  pthread_mutex_init(&s->mu, NULL);
  cudaGetDevice(&s->device);
  s->budget = hbm_budget_bytes;
  s->nstreams = nstreams;
  s->next_ticket = 1;
  if (pthread_create(&s->pump, NULL, pump_main, s) != 0) {
    pthread_mutex_destroy(&s->mu);
    free(s->tickets), free(s);
    return FMMFFT_ERR_NOMEM;
  }
  *out = s;
  return FMMFFT_OK;
}

int fmmfft_server_destroy(fmmfft_server s) {
  if (!s) return FMMFFT_OK;
  /* every queued request still leaves, then everything in flight completes */
  for (;;) {
    pthread_mutex_lock(&s->mu);
    pump_once(s);
    long q = 0;
    int creating = 0;
    for (int l = 0; l < s->nlanes; ++l) q += s->lanes[l].qlen, creating |= s->lanes[l].creating;
    pthread_mutex_unlock(&s->mu);
    if (q == 0 && !creating) break;
    struct timespec nap = {0, 20000};
    nanosleep(&nap, NULL);
  }
  s->stop = 1;
  pthread_join(s->pump, NULL);
  for (int l = 0; l < s->nlanes; ++l) {
    srv_lane *ln = &s->lanes[l];
    for (int i = 0; i < ln->nplans; ++i) free_plan(&ln->p[i]);
    free(ln->queue);
  }
  for (int i = 0; i < SRV_TICKETS; ++i)
    if (s->tickets[i].has_ev) cudaEventDestroy(s->tickets[i].ev);
  pthread_mutex_destroy(&s->mu);
  free(s->tickets), free(s);
  return FMMFFT_OK;
}

/* The lane of a shape, made on first use (its plan size computed, nothing allocated on the
 * device); -1 + status when the shape is invalid or the lane table is full. */
static int find_lane(struct fmmfft_server_s *s, long N, long P, long T, long b, int prec, int *status) {
  for (int l = 0; l < s->nlanes; ++l) {
    srv_lane *ln = &s->lanes[l];
    if (ln->N == N && ln->P == P && ln->T == T && ln->b == b && ln->prec == prec) return l;
  }
  if (s->nlanes == SRV_MAX_LANES) {
    *status = FMMFFT_ERR_BUSY;
    return -1;
  }
  const int ptrs = N >= SRV_PTR_MIN_N;
  long nb = ptrs ? SRV_PTR_BATCH : SRV_BATCH_SAMPLES / N;
  if (nb < 1) nb = 1;
  if (nb > SRV_MAX_BATCH) nb = SRV_MAX_BATCH;
  size_t bytes = 0;
  int rc = fmmfft_plan_bytes(N, P, T, b, prec, (int)nb, &bytes);
  if (rc != FMMFFT_OK) {
    *status = rc;
    return -1;
  }
  if (nb > 1 && !ptrs) bytes += 2 * (size_t)nb * (size_t)N * elem_bytes(prec);
  int *q = (int *)malloc(sizeof(int) * SRV_TICKETS);
  if (!q) {
    *status = FMMFFT_ERR_NOMEM;
    return -1;
  }
  srv_lane *ln = &s->lanes[s->nlanes];
  memset(ln, 0, sizeof *ln);
  ln->N = N, ln->P = P, ln->T = T, ln->b = b, ln->prec = prec;
  ln->nbmax = (int)nb;
  ln->ptrs = ptrs;
  ln->plan_bytes = bytes;
  ln->queue = q;
  return s->nlanes++;
}

int fmmfft_server_submit(fmmfft_server s, long N, long P, long terms, long b, int precision,
                         const void *d_in, void *d_out, fmmfft_ticket *ticket) {
  if (!s || !d_in || !d_out || !ticket) return FMMFFT_ERR_INVALID;
  pthread_mutex_lock(&s->mu);
  const int slot = (int)(s->next_ticket % SRV_TICKETS);
  srv_ticket *tk = &s->tickets[slot];
  if (tk->state == 1 || (tk->state == 2 && cudaEventQuery(tk->ev) != cudaSuccess)) {
    pthread_mutex_unlock(&s->mu);
    return FMMFFT_ERR_BUSY; /* the ticket ring is full of requests still running */
  }
  int status = FMMFFT_OK;
  const int l = find_lane(s, N, P, terms, b, precision, &status);
  if (l < 0) {
    pthread_mutex_unlock(&s->mu);
    return status;
  }
  srv_lane *ln = &s->lanes[l];
  if (ln->nplans == 0 && !ln->creating) {
    /* admission: the lane's first plan must fit, after evicting idle plans, before anything of
     * it is allocated */
    size_t evictable = 0;
    for (int k = 0; k < s->nlanes; ++k) {
      srv_lane *o = &s->lanes[k];
      if (k == l || o->qlen > 0 || o->creating) continue;
      for (int i = 0; i < o->nplans; ++i)
        if (plan_idle(&o->p[i])) evictable += o->p[i].bytes;
    }
    if (s->used - evictable + ln->plan_bytes > s->budget) {
      pthread_mutex_unlock(&s->mu);
      return FMMFFT_ERR_BUSY;
    }
  }
  tk->id = s->next_ticket++;
  tk->in = d_in, tk->out = d_out, tk->lane = l, tk->state = 1;
  ln->queue[(ln->qhead + ln->qlen) % SRV_TICKETS] = slot;
  ln->qlen++;
  dispatch_lane(s, l);
  *ticket = tk->id;
  pthread_mutex_unlock(&s->mu);
  return FMMFFT_OK;
}

int fmmfft_server_query(fmmfft_server s, fmmfft_ticket t) {
  if (!s) return FMMFFT_ERR_INVALID;
  pthread_mutex_lock(&s->mu);
  srv_ticket *tk = &s->tickets[t % SRV_TICKETS];
  int rc;
  if (tk->state == 0 || tk->id != t) {
    rc = FMMFFT_ERR_INVALID;
  } else if (tk->state == 3) {
    rc = FMMFFT_OK;
  } else if (tk->state == 4) {
    rc = FMMFFT_ERR_CUDA;
  } else if (tk->state == 2 && cudaEventQuery(tk->ev) == cudaSuccess) {
    tk->state = 3, rc = FMMFFT_OK;
  } else {
    if (tk->state == 1) dispatch_lane(s, tk->lane);
    rc = FMMFFT_ERR_BUSY;
  }
  pthread_mutex_unlock(&s->mu);
  return rc;
}

int fmmfft_server_wait(fmmfft_server s, fmmfft_ticket t, long timeout_ms) {
  struct timespec t0, now;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (;;) {
    int rc = fmmfft_server_query(s, t);
    if (rc != FMMFFT_ERR_BUSY) return rc;
    clock_gettime(CLOCK_MONOTONIC, &now);
    long ms = (now.tv_sec - t0.tv_sec) * 1000 + (now.tv_nsec - t0.tv_nsec) / 1000000;
    if (ms > timeout_ms) return FMMFFT_ERR_TIMEOUT;
    struct timespec nap = {0, 20000}; /* 20 us */
    nanosleep(&nap, NULL);
  }
}

int fmmfft_server_stats(fmmfft_server s, size_t *hbm_used, int *plans, int *slots) {
  if (!s) return FMMFFT_ERR_INVALID;
  pthread_mutex_lock(&s->mu);
  int np = 0;
  for (int l = 0; l < s->nlanes; ++l) np += s->lanes[l].nplans;
  if (hbm_used) *hbm_used = s->used;
  if (plans) *plans = np;
  if (slots) *slots = s->nstreams;
  pthread_mutex_unlock(&s->mu);
  return FMMFFT_OK;
}

int fmmfft_server_counts(fmmfft_server s, uint64_t *requests, uint64_t *launches) {
  if (!s) return FMMFFT_ERR_INVALID;
  pthread_mutex_lock(&s->mu);
  if (requests) *requests = s->dispatched;
  if (launches) *launches = s->launches;
  pthread_mutex_unlock(&s->mu);
  return FMMFFT_OK;
}

/* Makes `nplans` plans of a shape resident (at most the server's plans per shape), built in the
 * caller's thread, and instantiates each batched plan's graphs for every batch size it will use
 * (powers of two up to its capacity), so that no request of this shape later waits for a plan to
 * be built or a graph to be captured.  Refused with FMMFFT_ERR_BUSY when the budget cannot hold
 * them after evicting idle plans. */
int fmmfft_server_reserve(fmmfft_server s, long N, long P, long terms, long b, int precision, int nplans) {
  if (!s || nplans < 1) return FMMFFT_ERR_INVALID;
  const int cap = s->nstreams < SRV_LANE_PLANS ? s->nstreams : SRV_LANE_PLANS;
  if (nplans > cap) nplans = cap;
  for (;;) {
    pthread_mutex_lock(&s->mu);
    int status = FMMFFT_OK;
    const int l = find_lane(s, N, P, terms, b, precision, &status);
    if (l < 0) {
      pthread_mutex_unlock(&s->mu);
      return status;
    }
    srv_lane *ln = &s->lanes[l];
    if (ln->nplans >= nplans) {
      pthread_mutex_unlock(&s->mu);
      return FMMFFT_OK;
    }
    if (ln->creating) { /* the dispatcher is building one: wait for it */
      pthread_mutex_unlock(&s->mu);
      struct timespec nap = {0, 100000};
      nanosleep(&nap, NULL);
      continue;
    }
    while (s->used + ln->plan_bytes > s->budget && evict_one(s, l)) {
    }
    if (s->used + ln->plan_bytes > s->budget) {
      pthread_mutex_unlock(&s->mu);
      return FMMFFT_ERR_BUSY;
    }
    s->used += ln->plan_bytes;
    ln->creating = 1;
    const int nb = ln->nbmax, ptrs = ln->ptrs;
    pthread_mutex_unlock(&s->mu);
    srv_plan np;
    memset(&np, 0, sizeof np);
    int ok = fmmfft_plan_create_batched(&np.plan, N, P, terms, b, precision, nb) == FMMFFT_OK;
    ok = ok && cudaStreamCreateWithFlags(&np.st, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&np.done, cudaEventDisableTiming) == cudaSuccess;
    if (ok && nb > 1 && !ptrs) {
      const size_t bytes = (size_t)nb * (size_t)N * elem_bytes(precision);
      ok = cudaMalloc(&np.bin, bytes) == cudaSuccess && cudaMalloc(&np.bout, bytes) == cudaSuccess;
      ok = ok && cudaMemsetAsync(np.bin, 0, bytes, np.st) == cudaSuccess;
      for (int k = 1; ok && k <= nb; k *= 2) /* every batch size's graph, captured and run once */
        ok = fmmfft_execute_many_graph(np.plan, k, np.bin, np.bout, np.st) == FMMFFT_OK;
      ok = ok && cudaStreamSynchronize(np.st) == cudaSuccess;
    }
    if (!ok) {
      cudaGetLastError();
      free_plan(&np);
    }
    pthread_mutex_lock(&s->mu);
    ln = &s->lanes[l];
    ln->creating = 0;
    if (!ok) {
      s->used -= ln->plan_bytes;
      pthread_mutex_unlock(&s->mu);
      return FMMFFT_ERR_NOMEM;
    }
    np.bytes = ln->plan_bytes;
    np.last_use = ++s->clock;
    ln->p[ln->nplans++] = np;
    pthread_mutex_unlock(&s->mu);
  }
}
