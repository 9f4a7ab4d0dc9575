/*
 * Internal interface between the C host layer (fmmfft_ops.c, fmmfft_api.c) and the CUDA layer
 * (fmmfft_kernels.cu).  Not part of the public C-ABI.
 */
#ifndef FMMFFT_INTERNAL_H
#define FMMFFT_INTERNAL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Operator indices inside one level's block of fmm_ops64.levops, in the order the reference
 * builds them (src/fmmfft.c:282-289). */
enum { FMM_SHFTFN = 0, FMM_SHFTFP, FMM_FLIP2N, FMM_FLIP2P, FMM_FLIP3N, FMM_FLIP3P, FMM_SHFTLN,
       FMM_SHFTLP, FMM_NLEVOPS };

/* Every FMM operator of one (M, P, terms, b), built in FP64 on the host. */
typedef struct fmm_ops64 {
  long M, P, T, b, s, n;
  double *chnods; /* [T]                        src/fmmfft.c:273-275 */
  double *initch; /* [b][T]      S2M            :242-259 */
  double *topflp; /* [T][T]      level-2 M2L    :279 */
  double *levops; /* [n-2][8][T][T]  per level  :281-290 (index 0 = level 3) */
  double *evalm;  /* [b][P-1][T] L2T weights    :295-298 */
  double *evalmh; /* [P/2][T]    half-shifted   :300-304 */
  double *cot;    /* [P-1][4b]   cot(pi(d + sc/P)/M), index d + 2b, d in [-2b, 2b) :306-318 */
  double *fo;     /* [P][P-1] complex (re, im)  :325-331 */
} fmm_ops64;

int fmm_validate(long M, long P, long T, long b);
int fmm_ops64_build(long M, long P, long T, long b, fmm_ops64 *o);
void fmm_ops64_free(fmm_ops64 *o);
/* Lays the operators out as the reference's mfti does (src/fmmfft.c:343-374). */
void fmm_ops64_to_reference_w(const fmm_ops64 *o, double *w);
long fmm_getwlen2(long lq, long terms, long p, long b);
long fmm_ops64_doubles(long M, long P, long T, long b);
int fmm_ops64_build_in(long M, long P, long T, long b, fmm_ops64 *o, double *store, long cap);
long fmm_getvlen(long lq, long terms, long p, long b);

/* ---- CUDA layer (fmmfft_kernels.cu) ---- */
typedef struct fmmk_state fmmk_state;
int fmmk_create(const fmm_ops64 *ops, int precision, fmmk_state **out, size_t *device_bytes,
                char *err, size_t errlen);
void fmmk_destroy(fmmk_state *st);
int fmmk_execute(fmmk_state *st, const void *d_in, void *d_out, void *stream, int inverse,
                 char *err, size_t errlen);
/* Batched forms: a plan made for up to nb transforms of its shape; an execute of nbt <= nb
 * transforms whose inputs and outputs are N apart. */
int fmmk_create_n(const fmm_ops64 *ops, int precision, int nb, fmmk_state **out, size_t *device_bytes,
                  char *err, size_t errlen);
int fmmk_execute_n(fmmk_state *st, const void *d_in, void *d_out, void *stream, int inverse, int nbt,
                   char *err, size_t errlen);
/* The same with transform i read from ins[i] and written to outs[i] (nbt <= 64). */
int fmmk_execute_ptrs(fmmk_state *st, int nbt, const void *const *ins, void *const *outs, void *stream,
                      char *err, size_t errlen);
int fmmk_execute_blocks(fmmk_state *st, const void *const *in, void *const *out, int host, void *stream,
                        char *err, size_t errlen);
int fmmk_describe(fmmk_state *st, char *buf, size_t len);
/* Shard g of G of one sharded transform (fmmfft_kernels.cu, "sharded transform"). */
typedef struct fmmk_shard fmmk_shard;
int fmmk_shard_create(const fmm_ops64 *ops, int precision, int G, int g, fmmk_shard **out, char *err,
                      size_t errlen);
void fmmk_shard_destroy(fmmk_shard *sh);
/* ptr: x_ext, sums, phi_send, phi_all, z_send, z_recv, y; cnt: x_ext and halo (complex), phi_send
 * (reals), z_send and y (complex) */
void fmmk_shard_buffers(fmmk_shard *sh, void **ptr, size_t *cnt);
int fmmk_shard_phase(fmmk_shard *sh, int phase, void *stream, char *err, size_t errlen);
int fmmk_refine_enable(fmmk_state *st, const fmm_ops64 *ops, size_t *bytes, char *err, size_t errlen);
int fmmk_execute_refined(fmmk_state *st, const void *d_in, void *d_out, void *stream, char *err,
                         size_t errlen);
int fmmk_plan_bytes(long M, long P, long T, long b, int precision, int nb, size_t *bytes, char *err,
                    size_t errlen);
int fmmk_execute_graph_n(fmmk_state *st, const void *d_in, void *d_out, void *stream, int inverse,
                         int nbt, char *err, size_t errlen);
int fmmk_execute_host(fmmk_state *st, const void *h_in, void *h_out, void *stream, char *err,
                      size_t errlen);
int fmmk_execute_host_many(fmmk_state *st, int n, const void *const *h_in, void *const *h_out,
                           void *stream, char *err, size_t errlen);
int fmmk_debug_fetch(fmmk_state *st, double *u, double *z, double *phi, double *psi);
int fmmk_device_ok(char *err, size_t errlen);
int fmmk_profile_start(fmmk_state *st, int cap);
int fmmk_profile_stop(fmmk_state *st, double *stage_ms, int *stage_launches, int cap, int *nexec);
const char *fmmk_stage_name(int i);
int fmmk_check(fmmk_state *st);
int fmmk_selftest_wait(fmmk_state *st, int which, long limit_us, char *err, size_t errlen);
int fmmk_execute_graph(fmmk_state *st, const void *d_in, void *d_out, void *stream, int inverse,
                       char *err, size_t errlen);
int fmmk_batch_capture(fmmk_state *const *sts, const void *const *ins, void *const *outs,
                       const int *inverse, const int *counts, const int *branch, int n, int nbranch,
                       void **exec_out, char *err, size_t errlen);
int fmmk_batch_launch(void *exec, void *stream);
void fmmk_batch_free(void *exec);
int fmmk_execute_noalloc(const fmm_ops64 *ops, int reuse_ops, const void *d_in, void *d_out,
                         void *stream, char *err, size_t errlen);

typedef struct fmmk_fft fmmk_fft;
int fmmk_fft_create(long N, int dbl, fmmk_fft **out, size_t *device_bytes, char *err, size_t errlen);
int fmmk_fft_execute(fmmk_fft *f, const void *in, void *out, void *stream, char *err, size_t errlen);
size_t fmmk_fft_bytes(const fmmk_fft *f);
void fmmk_fft_destroy(fmmk_fft *f);

#ifdef __cplusplus
}
#endif
#endif
