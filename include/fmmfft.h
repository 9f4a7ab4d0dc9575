/*
 * fmmfft.h — C-ABI of the B200-native FMM-accelerated FFT (libfmmfft_b200.so).
 *
 * Drop-in boundary for the forward FMM-FFT of 97amarnathk/fmm-fft (src/fmmfft.c).  The
 * reference ships no header (README.md:38-39 lists it as a TODO); the four compatibility entry
 * points below keep its names, argument order and argument meaning:
 *
 *   getwlen2  src/fmmfft.c:1160   size (doubles) of the operator buffer w
 *   getvlen   src/fmmfft.c:1110   size (doubles) of the scratch buffer v
 *   mfti      src/fmmfft.c:337    build the operators for (lq, p, terms, b) into w
 *   mft       src/fmmfft.c:980    run the transform
 *
 * What changes at the boundary: the reference runs as P MPI ranks that each pass their own
 * lq = N/P block; here the P ranks are P blocks of one GPU, so `mft` takes the FULL vector of
 * N = p*lq complex128 values (rank r's block at offset r*lq, i.e. natural order) on the host,
 * transforms it on the GPU and writes the result back in place, natural order.  `myid` is
 * ignored.  The FFTW plan argument is ignored (it may be NULL): the size-lq FFTs run on the GPU.
 * The reference does no validation (bad sizes are undefined behaviour there); these functions
 * validate, leave the buffers untouched on error and record a status that
 * fmmfft_last_error() returns.
 *
 * The native API (fmmfft_plan_*) keeps operators and workspace resident on the device and runs
 * on caller-provided device buffers and a CUDA stream.  Every function returns an fmmfft_status.
 * No function takes or returns framework (torch) types: plain pointers and sizes only.
 */
#ifndef FMMFFT_B200_H
#define FMMFFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
typedef enum {
  FMMFFT_OK = 0,
  FMMFFT_ERR_INVALID = 1,     /* parameter outside the supported set */
  FMMFFT_ERR_NOMEM = 2,       /* host or device allocation failed */
  FMMFFT_ERR_CUDA = 3,        /* a CUDA call failed (message in fmmfft_last_error_string) */
  FMMFFT_ERR_NO_DEVICE = 4,   /* no CUDA device, or the kernels were not built for it */
  FMMFFT_ERR_UNSUPPORTED = 5, /* valid request this build does not serve (e.g. dir < 0 in mft) */
  FMMFFT_ERR_TIMEOUT = 6,     /* a bounded device-side wait gave up */
  FMMFFT_ERR_BUSY = 7         /* admission refused (serving queue / HBM budget) */
} fmmfft_status;

/* Arithmetic of a plan.  Input/output element type follows: complex128 for F64, complex64 for
 * the others (interleaved re, im). */
typedef enum {
  FMMFFT_F64 = 0,     /* FP64 everywhere (the reference's precision) */
  FMMFFT_F32 = 1,     /* FP32 on CUDA cores: the plain GPU FMM-FFT.  For complex64 plans with
                         terms >= 10 the P block-DC bins y[r M] (r < P) are the exact sums
                         sum_n x[n] e^{-2 pi i n r / P} (FP64 on the GPU) instead of the FMM's
                         value: at those bins the FMM's FP32 value carries the largest error of
                         the transform (7e-5 relative at P = 64), while its truncation there is
                         below 3.3e-8 for terms >= 10.  FP64 plans keep the FMM's value. */
  FMMFFT_F32_TC = 2,  /* operator contractions on tcgen05 tensor cores in split TF32 (operands
                         split into TF32 hi + lo, three products, FP32 accumulation), rest FP32 */
  FMMFFT_BF16X3 = 3   /* the same contractions in BF16x3 (BF16 hi + lo, three products, FP32
                         accumulation, ~2^-17 per product): for orders whose truncation error is
                         well above 1e-5 (the 1e-4 accuracy class); rest FP32 */
} fmmfft_precision;

/* ------------------------------------------------------------------ reference-compatible */

/* src/fmmfft.c:1160.  Number of doubles the caller allocates for w.  Returns -1 for sizes the
 * library rejects. */
long getwlen2(long lq, long terms, long p, long b);

/* src/fmmfft.c:1110.  Number of doubles the caller allocates for v (kept identical to the
 * reference so callers allocate the same; this library does not use v).  -1 if invalid. */
long getvlen(long lq, long terms, long p, long b);

/* src/fmmfft.c:337.  Builds every FMM operator for lq points per block, p blocks, `terms`
 * Chebyshev terms and b points per leaf box into w, in the reference's layout and bit for bit
 * equal to it, and makes the device plan for (lq, p, terms, b) resident.  szkeep / sztemp are
 * ignored, as in the reference. */
void mfti(long lq, long p, long terms, long b, double *w, double *v, long szkeep, long sztemp);

/* src/fmmfft.c:980.  Forward FMM-FFT of the full vector qr (p*lq complex128, host memory) in
 * place.  dir must be +1 (the reference's dir < 0 path is not a correct inverse,
 * fmmfft.c:976-977 vs :1080; use fmmfft_execute_inverse).  myid, w, v, sz1, szwk and
 * forward_plan are accepted for signature compatibility and not used (w may be NULL): the
 * operators come from the device plan that mfti made for the same (lq, p, terms, b) (made here
 * on first use if mfti was not called), which holds what mfti wrote into w; a w modified by the
 * caller after mfti is not seen. */
void mft(long lq, void *qr, long dir, long p, long myid, long terms, long b, double *w, double *v,
         long sz1, long szwk, void *forward_plan);

/* Rank mode of mft for SPMD callers whose ranks are threads of one process (the reference's
 * ranks are MPI processes, src/fmmfft.c:980): after fmmfft_mft_rank_mode(1), mft(lq, qr, dir,
 * p, myid, ...) is collective over p calls from p threads with myid = 0 .. p-1, each passing
 * ONLY its own block qr of lq complex128 values (rank myid's block, the reference's per-rank
 * buffer); the last caller to arrive runs the transform of the whole vector on the GPU, and
 * every call returns with its block holding its lq outputs, as the reference's mft does.  A
 * call whose partners do not all arrive within FMMFFT_RANK_TIMEOUT_MS (120 s by default) returns
 * with FMMFFT_ERR_TIMEOUT and its block untouched.  Calls with mismatched (lq, p, terms, b) or
 * a repeated myid are refused.  fmmfft_mft_rank_mode(0) restores full-vector calls; switching
 * is refused with FMMFFT_ERR_BUSY while a collective is in progress.  MPI callers whose ranks
 * are processes gather the blocks to one rank and call fmmfft_execute_blocks_host there
 * (INTEGRATION.md shows the binding). */
int fmmfft_mft_rank_mode(int on);

/* Status of the calling thread's last compatibility call (FMMFFT_OK after success). */
int fmmfft_last_error(void);
const char *fmmfft_last_error_string(void);

/* ------------------------------------------------------------------ native plan API */
typedef struct fmmfft_plan_s *fmmfft_plan;

/* Plan for one forward transform of length N = P*M split into P blocks, with `terms`
 * Chebyshev terms and b points per leaf box (tree depth n = log2(M/b)).  Requirements: P, M, b
 * powers of two; 2 <= P <= 1024; 2 <= b; M/b >= 4; 2 <= terms <= 64; M <= 2^26.  Operators are
 * built in FP64 on the host and kept resident on the current device; the workspace is
 * plan-owned. */
int fmmfft_plan_create(fmmfft_plan *out, long N, long P, long terms, long b, int precision);
int fmmfft_plan_destroy(fmmfft_plan plan);
/* complex64 plans are autotuned when the first plan of their (N, P, terms, b, precision) is
 * made in a process: FFT block size, coarse-tree threshold, tensor-core row
 * threshold and the fused S2M are timed and the fastest kept; later plans of that key take the
 * same choice (so they compute the same bits).  FMMFFT_AUTOTUNE=0 keeps the defaults; a knob
 * set by its environment switch is not tuned.  fmmfft_plan_describe writes the plan's choices
 * as text ("fft_threads=512 coarse_rows=4096 ..."). */
int fmmfft_plan_describe(fmmfft_plan plan, char *buf, size_t len);
/* Device bytes the plan holds (operators + workspace). */
int fmmfft_plan_device_bytes(fmmfft_plan plan, size_t *bytes);

/* Batched plans: no counterpart in the reference, which transforms one vector per run.  A plan
 * for up to max_transforms (1..64) transforms of one shape; fmmfft_execute_many runs `count` of
 * them in one launch sequence: every tree stage is one contraction over the rows of all of them,
 * the other stages carry the transform as a grid dimension.  Inputs and outputs are contiguous:
 * transform i at d_in + i*N and d_out + i*N elements.  Each transform's result is bitwise the
 * same as its own fmmfft_execute on a plan of capacity 1 (the arithmetic per row does not depend
 * on the rows beside it).  Workspace is max_transforms times a single plan's. */
int fmmfft_plan_create_batched(fmmfft_plan *out, long N, long P, long terms, long b, int precision,
                               int max_transforms);
int fmmfft_execute_many(fmmfft_plan plan, int count, const void *d_in, void *d_out, void *stream);
/* The same with each transform in a buffer of its own: transform i reads d_ins[i] and writes
 * d_outs[i] (device pointers, N elements each; d_ins[i] == d_outs[i] runs in place).  The tables
 * are host arrays, read during the call and passed to the kernels by value, so they may be reused
 * as soon as the call returns.  No counterpart in the reference; the request server batches large
 * requests this way, with no copies through staging buffers. */
int fmmfft_execute_many_ptrs(fmmfft_plan plan, int count, const void *const *d_ins, void *const *d_outs,
                             void *stream);
/* The same through a CUDA graph cached per (d_in, d_out, count), as fmmfft_execute_graph. */
int fmmfft_execute_many_graph(fmmfft_plan plan, int count, const void *d_in, void *d_out, void *stream);
/* Device bytes a plan of this shape, precision and capacity would hold, computed without
 * allocating anything (for admission under a memory budget). */
int fmmfft_plan_bytes(long N, long P, long terms, long b, int precision, int max_transforms,
                      size_t *bytes);

/* Forward transform: d_in, d_out = N interleaved complex values in device memory (complex128
 * for FMMFFT_F64, complex64 otherwise), natural order; d_in is not modified; d_in == d_out is
 * allowed.  Enqueued on `stream` (a cudaStream_t, NULL = legacy default stream); returns once
 * enqueued.  Calls on one plan must not overlap in time (the workspace is shared). */
int fmmfft_execute(fmmfft_plan plan, const void *d_in, void *d_out, void *stream);

/* Inverse transform (unnormalised: returns N * IDFT), computed as conj(F(conj(x))) with the
 * conjugations around the whole forward transform. */
int fmmfft_execute_inverse(fmmfft_plan plan, const void *d_in, void *d_out, void *stream);

/* Optional FP64 residual correction of complex64 plans (no counterpart in the reference, which
 * computes in FP64 throughout).  fmmfft_plan_enable_refinement builds, once, an FP64 plan of the
 * same (N, P, terms, b) and 32 N bytes of scratch beside the plan.  fmmfft_execute_refined then
 * computes y1 = F x with the plan's own arithmetic, the residual r = x - F64^-1(y1) / N in FP64
 * through the FP64 plan (an inverse FMM-FFT), and y = y1 + F r accumulated in FP64: d_in holds N
 * complex64, d_out receives N complex128.  The result agrees with the FP64 FMM-FFT (the
 * reference's arithmetic) to about the square of the plan's own relative error, and with the
 * exact DFT to the FMM's truncation at this order. */
int fmmfft_plan_enable_refinement(fmmfft_plan plan);
int fmmfft_execute_refined(fmmfft_plan plan, const void *d_in, void *d_out, void *stream);

/* Same transform from and to HOST memory: copies in, executes, copies out, synchronises. */
int fmmfft_execute_host(fmmfft_plan plan, const void *h_in, void *h_out, void *stream);
/* n transforms of host arrays, h_in[i] -> h_out[i] (N complex each; h_in[i] == h_out[i] is
 * allowed), pipelined: the copy-in of transform i+1, the execute of transform i and the copy-out
 * of transform i-1 overlap on three streams (with page-locked host memory PCIe carries both
 * directions at once), so a sequence of host-resident transforms costs about max(copy-in,
 * execute, copy-out) each instead of their sum.  Three device staging buffers of N complex and
 * two copy streams are made on the first call and kept with the plan.  Each output is bitwise
 * what fmmfft_execute_host gives.  Returns when every output is in host memory.  Replaces a loop
 * over the reference's mft (fmmfft.c:980) for a stream of inputs. */
int fmmfft_execute_host_many(fmmfft_plan plan, int n, const void *const *h_in, void *const *h_out,
                             void *stream);

/* Block-distributed transform: P input blocks of M = N/P complex values each (block r = rank
 * r's lq-block qr of the reference's SPMD layout, i.e. elements r*M .. r*M+M-1 of the vector)
 * and P output blocks (block r receives outputs r*M .. r*M+M-1, rank r's result in the
 * reference).  _blocks: device pointers, enqueued on `stream`; _blocks_host: host pointers,
 * synchronises.  Input and output blocks may be the same buffers. */
int fmmfft_execute_blocks(fmmfft_plan plan, const void *const *d_blocks_in, void *const *d_blocks_out,
                          void *stream);
int fmmfft_execute_blocks_host(fmmfft_plan plan, const void *const *h_blocks_in, void *const *h_blocks_out,
                               void *stream);

/* Stage-level access for parity tests: copies the plan's intermediate arrays after the last
 * execute into host memory as float64 (NULL to skip):
 *   u   [P-1][2][M]  far+near field per section, planar re/im
 *   z   [P][M] complex  (interleaved) combined blocks before the local FFTs
 *   phi, psi [levels 2..n][P-1][2][2^l][terms] planar expansions (level l at offset
 *        (2^l - 4) * (P-1) * 2 * terms) */
int fmmfft_debug_fetch(fmmfft_plan plan, double *u, double *z, double *phi, double *psi);

/* Synchronises the device and reports FMMFFT_ERR_TIMEOUT if, since the last check, a bounded
 * device-side wait (the tensor-core kernels' mbarrier waits) gave up instead of completing;
 * FMMFFT_OK otherwise.  Clears the recorded status. */
int fmmfft_plan_check(fmmfft_plan plan);

/* Self-test of the bounded device waits, for tests and health checks; no counterpart in the
 * reference (which has no device code).  Runs one small kernel that waits, with the same wait
 * routine as the tensor-core kernels, on an mbarrier nobody arrives on while it holds tensor
 * memory (which must be 0), with a limit of limit_us microseconds (1 .. 2e6).  The wait gives up,
 * records the timeout in the plan's status word, frees the tensor memory and returns; the call
 * synchronises the device.  The next fmmfft_plan_check(plan) then returns FMMFFT_ERR_TIMEOUT,
 * and the plan stays usable. */
int fmmfft_plan_selftest_wait(fmmfft_plan plan, int which, long limit_us);

/* Same transform as fmmfft_execute through a CUDA graph: the first call for a given
 * (d_in, d_out) captures the plan's launch sequence and instantiates it (make that call outside
 * any stream capture); later calls are a single graph launch on `stream`.  Up to 8 buffer pairs
 * per plan stay cached. */
int fmmfft_execute_graph(fmmfft_plan plan, const void *d_in, void *d_out, void *stream);

/* ------------------------------------------------------------------ batches */
/* Many transforms, of uneven sizes, as one graph: transform i runs plans[i] from d_in[i] to
 * d_out[i] (device buffers).  The transforms are spread over `nbranch` parallel branches of the
 * graph; all transforms that use the same plan share its workspace, so they are placed in the
 * same branch and run one after another there.  fmmfft_batch_launch runs the whole batch with
 * one graph launch on `stream`.  The plans and buffers must outlive the batch. */
typedef struct fmmfft_batch_s *fmmfft_batch;
int fmmfft_batch_create(fmmfft_batch *out, const fmmfft_plan *plans, const void *const *d_in,
                        void *const *d_out, int n, int nbranch);
/* The same with batched plans: entry i runs counts[i] transforms of plans[i] (contiguous, N
 * apart, from d_in[i] to d_out[i]) in one launch sequence; counts[i] <= the plan's capacity.  An
 * uneven batch grouped by shape is then one graph of one launch sequence per shape. */
int fmmfft_batch_create_many(fmmfft_batch *out, const fmmfft_plan *plans, const int *counts,
                             const void *const *d_in, void *const *d_out, int n, int nbranch);
int fmmfft_batch_launch(fmmfft_batch batch, void *stream);
int fmmfft_batch_destroy(fmmfft_batch batch);

/* ------------------------------------------------------------------ sharded transform */
/* One transform split over G devices (G a power of two; P >= 16, P a multiple of 2G, at least 8
 * leaf boxes of b points per shard), replacing the reference's P-rank mft (src/fmmfft.c:384-978,
 * its halo exchanges :517-618, section-sum reduction :452-453 and all-to-all :970).  Shard g holds
 * the contiguous block g of N/G input points and ends with the block g of N/G outputs, as the
 * reference's ranks hold their qr.  The library computes; the caller moves data between the
 * shards (NCCL through torch.distributed in fmm-fft_b200/sharded.py), with the shard's buffers:
 *   phase 0 needs x_ext = [the last halo_elems points of shard g-1's block | the shard's own N/G
 *           points | the first halo_elems points of shard g+1's block] (cyclic in g);
 *   between 0 and 1: `sums` (P complex) summed over the shards, in place on every shard, and
 *           phi_all = the shards' phi_send buffers (phi_elems reals each) back to back, in shard
 *           order;
 *   between 1 and 2: an all-to-all: z_send holds G chunks of z_elems/G complex, chunk h for shard
 *           h; z_recv receives the chunk for this shard from every shard, in shard order;
 *   after phase 2: y holds the shard's y_elems outputs.
 * Elements are complex64 (FP32 plans) or complex128 (FP64), reals float or double.  Forward only.
 * Phases run in the order 0, 1, 2 on one stream; a stream-ordered exchange between them needs no
 * synchronisation. */
typedef struct fmmfft_shard_s *fmmfft_shard;
typedef struct {
  void *x_ext, *sums, *phi_send, *phi_all, *z_send, *z_recv, *y;
  size_t x_ext_elems, halo_elems, phi_elems, z_elems, y_elems;
} fmmfft_shard_bufs;
int fmmfft_shard_create(fmmfft_shard *out, long N, long P, long terms, long b, int precision, int G, int g);
int fmmfft_shard_buffers(fmmfft_shard sh, fmmfft_shard_bufs *bufs);
int fmmfft_shard_phase(fmmfft_shard sh, int phase, void *stream);
int fmmfft_shard_destroy(fmmfft_shard sh);

/* ------------------------------------------------------------------ serving */
/* A request server with continuous batching: transforms of mixed sizes and precisions are
 * submitted one at a time; requests of one shape (N, P, terms, b, precision) that arrive while
 * that shape's plans are busy are queued and leave together, as ONE batched launch sequence, as
 * soon as a plan frees up (shapes below 2^22 samples: up to 2^24 samples, at most 32 requests,
 * per batch, through staging buffers; from 2^22 samples: up to 4 requests per batch, each read
 * and written in its own buffers); each shape keeps up to
 * `nstreams` (at most 3) resident plans on their own streams, so batches of different shapes and
 * of one shape overlap on the device.  A dispatcher thread sends queued batches; submit, query and
 * wait dispatch too.  The device memory of the plans is capped by hbm_budget_bytes: a plan's size
 * is computed before anything is allocated, idle plans are evicted least-recently-used to make
 * room, and a request whose shape cannot get a plan is refused with FMMFFT_ERR_BUSY (retry later)
 * with nothing allocated.  d_in / d_out are caller-owned device buffers that must stay valid until
 * the request completes.  Results do not depend on what else is in flight: a batched transform
 * gives bitwise the output of its own execute. */
typedef struct fmmfft_server_s *fmmfft_server;
typedef uint64_t fmmfft_ticket;
int fmmfft_server_create(fmmfft_server *out, size_t hbm_budget_bytes, int nstreams);
int fmmfft_server_destroy(fmmfft_server server); /* waits for every request in flight */
int fmmfft_server_submit(fmmfft_server server, long N, long P, long terms, long b, int precision,
                         const void *d_in, void *d_out, fmmfft_ticket *ticket);
/* Makes nplans plans of a shape resident ahead of its requests (at most nstreams), each batched
 * plan with its graphs for every batch size instantiated, so that no request waits for a plan to
 * be built; FMMFFT_ERR_BUSY when the budget cannot hold them.  Blocks until they are ready. */
int fmmfft_server_reserve(fmmfft_server server, long N, long P, long terms, long b, int precision,
                          int nplans);
/* FMMFFT_OK when the request is complete, FMMFFT_ERR_BUSY while it runs. */
int fmmfft_server_query(fmmfft_server server, fmmfft_ticket ticket);
/* Waits up to timeout_ms; FMMFFT_OK or FMMFFT_ERR_TIMEOUT. */
int fmmfft_server_wait(fmmfft_server server, fmmfft_ticket ticket, long timeout_ms);
int fmmfft_server_stats(fmmfft_server server, size_t *hbm_used, int *plans, int *streams);
/* Requests sent to the GPU so far and the batched launch sequences they went in (their ratio is
 * the mean batch size). */
int fmmfft_server_counts(fmmfft_server server, uint64_t *requests, uint64_t *launches);

/* ------------------------------------------------------------------ stage timing */
/* Records CUDA events around every stage of the next `max_executes` executes of this plan (on
 * the stream each execute runs on).  No counterpart in the reference, which only times the
 * whole mft call (src/fmmfft.c:1259-1263). */
int fmmfft_profile_start(fmmfft_plan plan, int max_executes);
/* Synchronises on the last recorded execute and returns, per stage, the summed device time in
 * ms over the recorded executes (stage_ms) and the kernel launches one execute makes in that
 * stage (stage_launches); *nstages = number of stages (<= cap filled), *nexecutes = executes
 * recorded.  Stops profiling. */
int fmmfft_profile_stop(fmmfft_plan plan, double *stage_ms, int *stage_launches, int cap,
                        int *nstages, int *nexecutes);
/* Name of stage i ("sections", "s2m", "m2l_l2l", "fft_pass1", ...), "" when out of range. */
const char *fmmfft_stage_name(int i);

/* ------------------------------------------------------------------ allocation-free entry */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc: code that runs
 * under a device-memory budget owned by someone else (a pool or arena it may not grow), or in a
 * phase where it must not allocate at all.  Forward transform of N complex64 values (FP32, the
 * FMMFFT_F32 arithmetic, same result as fmmfft_execute on an FMMFFT_F32 plan) from d_in to
 * d_out, both caller-owned device buffers, enqueued on `stream`.  Nothing is allocated: the
 * operator tables and the workspace live in one file-scope device array of 32 MiB that every
 * GPU which loads this library holds until process exit (the FP64 operator build uses a
 * file-scope 16 MiB host array).  Sizes whose tables plus workspace exceed 32 MiB (about
 * N = 2^18 complex64 at 24 terms, b = 32) return FMMFFT_ERR_INVALID.
 * The first call on a device sets that device up (it looks up the array's device address) and
 * the first call for new (N, P, terms, b) uploads the tables and synchronises `stream`; make
 * those calls before any stream capture.  All calls share the one array, which keeps the last
 * call's tables: calls whose work overlaps on the GPU (other streams, other threads) race on
 * it and must be serialised by the caller. */
int fmmfft_execute_noalloc(long N, long P, long terms, long b, const void *d_in, void *d_out,
                           void *stream);

/* ------------------------------------------------------------------ plain FFT comparator */
/* A conventional (non-FMM) forward FFT of length N on the GPU: the reference's plain FFTW
 * comparators, src/fftw_serial.c:53-58 (fftw_plan_dft + fftw_execute, FFTW_FORWARD) and
 * src/fftw_mpi.c:54-58, which the reference times beside mft.  Same sign and scaling as
 * fmmfft_execute (y[k] = sum_n x[n] exp(-2 pi i n k / N), unnormalised); out of place, unlike
 * FFTW's in-place x -> x there (d_in != d_out).  N a power of two in [16, 2^30]; precision
 * FMMFFT_F64 (complex128) or FMMFFT_F32 / FMMFFT_F32_TC (complex64: both the same FP32 FFT).
 * The handle owns one N-element workspace and the twiddle tables. */
typedef struct fmmfft_fft_s *fmmfft_fft;
int fmmfft_fft_create(fmmfft_fft *out, long N, int precision);
int fmmfft_fft_execute(fmmfft_fft f, const void *d_in, void *d_out, void *stream);
int fmmfft_fft_device_bytes(fmmfft_fft f, size_t *bytes);
int fmmfft_fft_destroy(fmmfft_fft f);

#ifdef __cplusplus
}
#endif
#endif /* FMMFFT_B200_H */
