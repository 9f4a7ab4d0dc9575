/*
 * Test infrastructure only: thread-based MPI subset for the shim-built reference.
 *
 * Each rank is a pthread bound to a rank id (shim_mpi_set_rank).  Point-to-point sends are
 * buffered (the payload is copied into the destination's mailbox and the call returns), which
 * is what the reference relies on at fmmfft.c:760-761 where every rank sends before it
 * receives.  Receives match on (source, tag) in arrival order, as MPI's non-overtaking rule
 * requires.  Collectives publish per-rank buffer pointers between two barriers; the reduction
 * sums contributions in rank order, so runs are deterministic.
 */
#include "mpi.h"

#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define SHIM_ELEM_BYTES 16 /* MPI_C_DOUBLE_COMPLEX, the only datatype the reference uses */
#define SHIM_RECV_TIMEOUT_S 600

typedef struct shim_msg {
  int src;
  int tag;
  size_t bytes;
  struct shim_msg *next;
  unsigned char data[];
} shim_msg;

typedef struct {
  pthread_mutex_t mu;
  pthread_cond_t cv;
  shim_msg *head;
  shim_msg *tail;
} shim_mailbox;

static struct {
  int nranks;
  shim_mailbox *boxes;
  pthread_barrier_t barrier;
  const void **published;
} g_world;

static __thread int t_rank = -1;

int shim_mpi_world_begin(int nranks) {
  if (nranks < 1) return -1;
  g_world.nranks = nranks;
  g_world.boxes = (shim_mailbox *)calloc((size_t)nranks, sizeof(shim_mailbox));
  g_world.published = (const void **)calloc((size_t)nranks, sizeof(void *));
  if (!g_world.boxes || !g_world.published) return -2;
  for (int r = 0; r < nranks; ++r) {
    pthread_mutex_init(&g_world.boxes[r].mu, NULL);
    pthread_cond_init(&g_world.boxes[r].cv, NULL);
  }
  pthread_barrier_init(&g_world.barrier, NULL, (unsigned)nranks);
  return 0;
}

void shim_mpi_world_end(void) {
  for (int r = 0; r < g_world.nranks; ++r) {
    shim_msg *m = g_world.boxes[r].head;
    while (m) {
      shim_msg *n = m->next;
      free(m);
      m = n;
    }
    pthread_mutex_destroy(&g_world.boxes[r].mu);
    pthread_cond_destroy(&g_world.boxes[r].cv);
  }
  pthread_barrier_destroy(&g_world.barrier);
  free(g_world.boxes);
  free((void *)g_world.published);
  memset(&g_world, 0, sizeof(g_world));
}

void shim_mpi_set_rank(int rank) { t_rank = rank; }

int MPI_Init(void *argc, void *argv) {
  (void)argc;
  (void)argv;
  return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, void *rank) {
  (void)comm;
  *(int *)rank = t_rank;
  return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, void *size) {
  (void)comm;
  *(int *)size = g_world.nranks;
  return MPI_SUCCESS;
}

int MPI_Finalize(void) { return MPI_SUCCESS; }

double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Barrier(MPI_Comm comm) {
  (void)comm;
  pthread_barrier_wait(&g_world.barrier);
  return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm) {
  (void)dt;
  (void)comm;
  if (dest < 0 || dest >= g_world.nranks) {
    fprintf(stderr, "shim MPI_Send: bad destination %d\n", dest);
    abort();
  }
  size_t bytes = (size_t)(count > 0 ? count : 0) * SHIM_ELEM_BYTES;
  shim_msg *m = (shim_msg *)malloc(sizeof(shim_msg) + bytes);
  if (!m) abort();
  m->src = t_rank;
  m->tag = tag;
  m->bytes = bytes;
  m->next = NULL;
  if (bytes) memcpy(m->data, buf, bytes);
  shim_mailbox *mb = &g_world.boxes[dest];
  pthread_mutex_lock(&mb->mu);
  if (mb->tail)
    mb->tail->next = m;
  else
    mb->head = m;
  mb->tail = m;
  pthread_cond_broadcast(&mb->cv);
  pthread_mutex_unlock(&mb->mu);
  return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm,
             MPI_Status *status) {
  (void)dt;
  (void)comm;
  shim_mailbox *mb = &g_world.boxes[t_rank];
  struct timespec deadline;
  clock_gettime(CLOCK_REALTIME, &deadline);
  deadline.tv_sec += SHIM_RECV_TIMEOUT_S;
  pthread_mutex_lock(&mb->mu);
  for (;;) {
    shim_msg *prev = NULL, *m = mb->head;
    while (m && !(m->src == source && m->tag == tag)) {
      prev = m;
      m = m->next;
    }
    if (m) {
      if (prev)
        prev->next = m->next;
      else
        mb->head = m->next;
      if (mb->tail == m) mb->tail = prev;
      pthread_mutex_unlock(&mb->mu);
      size_t want = (size_t)(count > 0 ? count : 0) * SHIM_ELEM_BYTES;
      memcpy(buf, m->data, want < m->bytes ? want : m->bytes);
      if (status) {
        status->MPI_SOURCE = m->src;
        status->MPI_TAG = m->tag;
        status->MPI_ERROR = 0;
      }
      free(m);
      return MPI_SUCCESS;
    }
    if (pthread_cond_timedwait(&mb->cv, &mb->mu, &deadline) == ETIMEDOUT) {
      fprintf(stderr, "shim MPI_Recv: rank %d timed out waiting for (src=%d, tag=%d)\n", t_rank,
              source, tag);
      abort();
    }
  }
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status) {
  MPI_Send(sendbuf, sendcount, sendtype, dest, sendtag, comm);
  return MPI_Recv(recvbuf, recvcount, recvtype, source, recvtag, comm, status);
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root,
               MPI_Comm comm) {
  (void)dt;
  (void)op;
  g_world.published[t_rank] = sendbuf;
  MPI_Barrier(comm);
  if (t_rank == root) {
    double *out = (double *)recvbuf;
    for (int i = 0; i < 2 * count; ++i) out[i] = 0.0;
    for (int r = 0; r < g_world.nranks; ++r) {
      const double *in = (const double *)g_world.published[r];
      for (int i = 0; i < 2 * count; ++i) out[i] += in[i];
    }
  }
  MPI_Barrier(comm);
  return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm) {
  (void)dt;
  if (t_rank == root) g_world.published[root] = buf;
  MPI_Barrier(comm);
  if (t_rank != root)
    memcpy(buf, g_world.published[root], (size_t)count * SHIM_ELEM_BYTES);
  MPI_Barrier(comm);
  return MPI_SUCCESS;
}

int MPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                 int recvcount, MPI_Datatype recvtype, MPI_Comm comm) {
  (void)sendtype;
  (void)recvtype;
  (void)recvcount;
  g_world.published[t_rank] = sendbuf;
  MPI_Barrier(comm);
  size_t blk = (size_t)sendcount * SHIM_ELEM_BYTES;
  for (int src = 0; src < g_world.nranks; ++src) {
    const unsigned char *s = (const unsigned char *)g_world.published[src];
    memcpy((unsigned char *)recvbuf + (size_t)src * blk, s + (size_t)t_rank * blk, blk);
  }
  MPI_Barrier(comm);
  return MPI_SUCCESS;
}
