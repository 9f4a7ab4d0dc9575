/*
 * Test infrastructure only: a thread-based stand-in for the subset of MPI that the
 * reference FMM-FFT (src/fmmfft.c, src/fmmfft_error.c) calls.  It lets the UNMODIFIED
 * reference source compile with plain gcc and run its P ranks as P pthreads inside one
 * process, so its output can be compared with the oracle restatement and with the GPU
 * path.  Nothing in the product links this file.
 *
 * Calls used by the reference (file:line in src/fmmfft.c):
 *   MPI_Barrier :396,972,981      MPI_Reduce/MPI_Bcast :452-453
 *   MPI_Send/MPI_Recv :501,513,652,670,760-761   MPI_Sendrecv :570-576,627,636,653-655,669-672
 *   MPI_Alltoall :970             MPI_Init/Comm_rank/Comm_size/Finalize/Wtime (main only)
 * Every message is MPI_C_DOUBLE_COMPLEX (16 bytes) on MPI_COMM_WORLD.
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_C_DOUBLE_COMPLEX 1
#define MPI_SUM 1
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

/* The reference passes `long *` where MPI takes `int *` (fmmfft.c:1196-1198); these three
 * take untyped pointers so that main() still compiles although the shim driver never calls it. */
int MPI_Init(void *argc, void *argv);
int MPI_Comm_rank(MPI_Comm comm, void *rank);
int MPI_Comm_size(MPI_Comm comm, void *size);
int MPI_Finalize(void);
double MPI_Wtime(void);

int MPI_Barrier(MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm,
             MPI_Status *status);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root,
               MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                 int recvcount, MPI_Datatype recvtype, MPI_Comm comm);

/* Shim control, used only by the oracle's reference driver. */
int shim_mpi_world_begin(int nranks);  /* create the world of nranks thread-ranks */
void shim_mpi_world_end(void);
void shim_mpi_set_rank(int rank);      /* bind the calling thread to a rank */

#endif
