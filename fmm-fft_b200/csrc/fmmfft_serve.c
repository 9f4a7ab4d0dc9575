/*
 * Request server of the FMM-FFT: admits transforms of mixed sizes and accuracy classes onto a
 * set of CUDA streams ("slots") so that requests arriving while others run overlap on the
 * device.  No counterpart in the reference, which runs one transform per mpirun.
 *
 *  - Plans (operators + workspace) stay resident per (N, P, terms, b, precision) and per slot,
 *    so two requests in flight never share a workspace; each runs through the plan's cached
 *    CUDA graph (one graph launch instead of ~35 kernel launches).
 *  - Admission by HBM budget: a request whose plan is not resident needs a new plan; idle
 *    plans (no request in flight) are evicted least-recently-used until it fits, otherwise the
 *    request is refused with FMMFFT_ERR_BUSY and the caller retries later.
 *  - Every request gets a ticket backed by a CUDA event; results are deterministic, so a
 *    request gives the same output alone and in a mix (tests/test_gpu_serving.py).
 */
#include <cuda_runtime_api.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/fmmfft.h"

#define SRV_MAX_PLANS 512
#define SRV_TICKETS 65536 /* outstanding tickets a server tracks (a ring) */

typedef struct {
  long N, P, T, b;
  int prec;
  int slot;
  fmmfft_plan plan;
  size_t bytes;
  unsigned long long last_use;
  cudaEvent_t last_done; /* completion of the newest request on this plan */
  int has_event;
} srv_plan;

typedef struct {
  fmmfft_ticket id;
  cudaEvent_t ev;
  int live;
  int done;
} srv_ticket;

struct fmmfft_server_s {
  pthread_mutex_t mu;
  size_t budget, used;
  int nslots;
  cudaStream_t *streams;
  unsigned long long *slot_load; /* requests submitted per slot (for choosing a slot) */
  srv_plan plans[SRV_MAX_PLANS];
  int nplans;
  srv_ticket *tickets;
  fmmfft_ticket next_ticket;
  unsigned long long clock;
};

static int plan_idle(srv_plan *p) {
  return !p->has_event || cudaEventQuery(p->last_done) == cudaSuccess;
}

static void drop_plan(struct fmmfft_server_s *s, int i) {
  srv_plan *p = &s->plans[i];
  if (p->has_event) cudaEventDestroy(p->last_done);
  fmmfft_plan_destroy(p->plan);
  s->used -= p->bytes;
  s->plans[i] = s->plans[--s->nplans];
}

int fmmfft_server_create(fmmfft_server *out, size_t hbm_budget_bytes, int nstreams) {
  if (!out || nstreams < 1 || nstreams > 64) return FMMFFT_ERR_INVALID;
  struct fmmfft_server_s *s = (struct fmmfft_server_s *)calloc(1, sizeof *s);
  if (!s) return FMMFFT_ERR_NOMEM;
  s->tickets = (srv_ticket *)calloc(SRV_TICKETS, sizeof(srv_ticket));
  s->streams = (cudaStream_t *)calloc((size_t)nstreams, sizeof(cudaStream_t));
  s->slot_load = (unsigned long long *)calloc((size_t)nstreams, sizeof(unsigned long long));
  if (!s->tickets || !s->streams || !s->slot_load) {
    free(s->tickets), free(s->streams), free(s->slot_load), free(s);
    return FMMFFT_ERR_NOMEM;
  }
  for (int i = 0; i < nstreams; ++i)
    if (cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking) != cudaSuccess) {
      for (int j = 0; j < i; ++j) cudaStreamDestroy(s->streams[j]);
      free(s->tickets), free(s->streams), free(s->slot_load), free(s);
      return FMMFFT_ERR_CUDA;
    }
  pthread_mutex_init(&s->mu, NULL);
  s->budget = hbm_budget_bytes;
  s->nslots = nstreams;
  s->next_ticket = 1;
  *out = s;
  return FMMFFT_OK;
}

int fmmfft_server_destroy(fmmfft_server s) {
  if (!s) return FMMFFT_OK;
  for (int i = 0; i < s->nslots; ++i) cudaStreamSynchronize(s->streams[i]);
  while (s->nplans) drop_plan(s, s->nplans - 1);
  for (int i = 0; i < SRV_TICKETS; ++i)
    if (s->tickets[i].live) cudaEventDestroy(s->tickets[i].ev);
  for (int i = 0; i < s->nslots; ++i) cudaStreamDestroy(s->streams[i]);
  pthread_mutex_destroy(&s->mu);
  free(s->tickets), free(s->streams), free(s->slot_load), free(s);
  return FMMFFT_OK;
}

/* The resident plan for (shape, slot), making room in the budget if needed; NULL + status. */
static srv_plan *get_plan(struct fmmfft_server_s *s, long N, long P, long T, long b, int prec,
                          int slot, int *status) {
  for (int i = 0; i < s->nplans; ++i) {
    srv_plan *p = &s->plans[i];
    if (p->N == N && p->P == P && p->T == T && p->b == b && p->prec == prec && p->slot == slot) {
      *status = FMMFFT_OK;
      return p;
    }
  }
  if (s->nplans == SRV_MAX_PLANS) {
    *status = FMMFFT_ERR_BUSY;
    return NULL;
  }
  fmmfft_plan pl = NULL;
  int rc = fmmfft_plan_create(&pl, N, P, T, b, prec);
  if (rc != FMMFFT_OK) {
    *status = rc == FMMFFT_ERR_NOMEM ? FMMFFT_ERR_BUSY : rc;
    return NULL;
  }
  size_t bytes = 0;
  fmmfft_plan_device_bytes(pl, &bytes);
  while (s->used + bytes > s->budget) { /* evict the least recently used idle plan */
    int victim = -1;
    for (int i = 0; i < s->nplans; ++i)
      if (plan_idle(&s->plans[i]) && (victim < 0 || s->plans[i].last_use < s->plans[victim].last_use))
        victim = i;
    if (victim < 0) break;
    drop_plan(s, victim);
  }
  if (s->used + bytes > s->budget) {
    fmmfft_plan_destroy(pl);
    *status = FMMFFT_ERR_BUSY;
    return NULL;
  }
  srv_plan *p = &s->plans[s->nplans++];
  memset(p, 0, sizeof *p);
  p->N = N, p->P = P, p->T = T, p->b = b, p->prec = prec, p->slot = slot, p->plan = pl;
  p->bytes = bytes;
  s->used += bytes;
  *status = FMMFFT_OK;
  return p;
}

int fmmfft_server_submit(fmmfft_server s, long N, long P, long terms, long b, int precision,
                         const void *d_in, void *d_out, fmmfft_ticket *ticket) {
  if (!s || !d_in || !d_out || !ticket) return FMMFFT_ERR_INVALID;
  pthread_mutex_lock(&s->mu);
  srv_ticket *tk = &s->tickets[s->next_ticket % SRV_TICKETS];
  if (tk->live && !tk->done && cudaEventQuery(tk->ev) != cudaSuccess) {
    pthread_mutex_unlock(&s->mu);
    return FMMFFT_ERR_BUSY; /* the ticket ring is full of requests still running */
  }
  /* slot: one that already holds this shape's plan and has the least work, else the least
   * loaded slot */
  int slot = -1;
  for (int i = 0; i < s->nplans; ++i) {
    srv_plan *p = &s->plans[i];
    if (p->N == N && p->P == P && p->T == terms && p->b == b && p->prec == precision &&
        (slot < 0 || s->slot_load[p->slot] < s->slot_load[slot]) && plan_idle(p))
      slot = p->slot;
  }
  if (slot < 0) {
    slot = 0;
    for (int i = 1; i < s->nslots; ++i)
      if (s->slot_load[i] < s->slot_load[slot]) slot = i;
  }
  int status;
  srv_plan *p = get_plan(s, N, P, terms, b, precision, slot, &status);
  if (!p) {
    pthread_mutex_unlock(&s->mu);
    return status;
  }
  cudaStream_t st = s->streams[slot];
  int rc = fmmfft_execute_graph(p->plan, d_in, d_out, st);
  if (rc != FMMFFT_OK) {
    pthread_mutex_unlock(&s->mu);
    return rc;
  }
  if (!p->has_event) {
    cudaEventCreateWithFlags(&p->last_done, cudaEventDisableTiming);
    p->has_event = 1;
  }
  cudaEventRecord(p->last_done, st);
  if (tk->live) cudaEventDestroy(tk->ev);
  cudaEventCreateWithFlags(&tk->ev, cudaEventDisableTiming);
  cudaEventRecord(tk->ev, st);
  tk->id = s->next_ticket++;
  tk->live = 1, tk->done = 0;
  p->last_use = ++s->clock;
  s->slot_load[slot] += (unsigned long long)N;
  *ticket = tk->id;
  pthread_mutex_unlock(&s->mu);
  return FMMFFT_OK;
}

int fmmfft_server_query(fmmfft_server s, fmmfft_ticket t) {
  if (!s) return FMMFFT_ERR_INVALID;
  pthread_mutex_lock(&s->mu);
  srv_ticket *tk = &s->tickets[t % SRV_TICKETS];
  int rc;
  if (!tk->live || tk->id != t)
    rc = FMMFFT_ERR_INVALID;
  else if (tk->done || cudaEventQuery(tk->ev) == cudaSuccess)
    tk->done = 1, rc = FMMFFT_OK;
  else
    rc = FMMFFT_ERR_BUSY;
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
  if (hbm_used) *hbm_used = s->used;
  if (plans) *plans = s->nplans;
  if (slots) *slots = s->nslots;
  pthread_mutex_unlock(&s->mu);
  return FMMFFT_OK;
}
