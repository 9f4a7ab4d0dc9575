/*
 * CUDA layer of the B200-native FMM-FFT (sm_100a).
 *
 * One forward transform of N = P*M points runs as these device stages (reference call stack
 * src/fmmfft.c mft -> mftint, :384-1081):
 *
 *   1  k_sections      x[M][P] -> xt[2P][M] planar sections + per-tile section sums
 *                      (deinterleave :419-439, section sums :441-457); when a tile holds whole
 *                      leaf boxes it also computes their S2M multipoles (:199-211, :465)
 *   2  k_sum_sections  tiles -> Sigma_m x_sc[m] (the MPI_Reduce/Bcast of :452-453)
 *   3  S2M             (when not fused into 1) row contraction: phi_n = xt . initch
 *   4  M2M             row contraction per level: phi_L = [phi_L+1 pair] . [S_L;S_R]  (:476-515)
 *   5  top flip        psi_2[c] = topflp . phi_2[c+2]                    (:620-639)
 *   6  M2L + L2L       row contraction per level over parent boxes, both children at once
 *                      (:643-749); the tree levels of stages 4-6 with fewer than 4096 rows (at
 *                      most 64 boxes per plane) run in one launch, k_coarse, a block per plane
 *   7  leaf            row contraction per section: u = [psi_n | x window] . [E_sc ; cot
 *                      Toeplitz] with the half-shifted first point as one more operator column
 *                      (tensor cores) + k_leaf_mid for section P/2; k_leaf (direct, CUDA cores)
 *                      for FP32 / FP64 plans; rowgemm + k_leaf_fix when b % 8 != 0 (:751-954)
 *   8  combine         pre-twiddle and length-P DFT over sections, transposed store, as a
 *                      register Stockham pass (k_fft_reg with CombineLd; k_combine otherwise)
 *                      (:956-968 and the MPI_Alltoall of :970)
 *   9  size-M FFTs     register Stockham passes k_fft_reg (k_fft_pass for shapes they do not
 *                      take) (FFTW at :1080)
 *  10  k_block_dc      FP32 plans: the block-DC bins from the exact identity in FP64
 *
 * Row contractions run on the tensor cores for split-TF32 plans (fmmfft_tc.cuh: k_tc_rowgemm,
 * k_tc_rowgemm16) and as rowgemm on the CUDA cores otherwise.
 * All tree operators are shared by every section and box, so each tree stage is one dense
 * contraction over "rows" (section, re/im plane, box) with a small operator; rowgemm is the
 * CUDA-core form of that contraction.  Real type R = float (complex64 plans) or double
 * (complex128 plans).  Expansions are stored planar: phi_l[(sc-1)*2 + ri][box][T].
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <new>

#include "fmmfft_internal.h"
#include "fmmfft_tc.cuh"

#define FMM_CUDA_TRY(call)                                                              \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      if (err) snprintf(err, errlen, "%s failed: %s", #call, cudaGetErrorString(e_));   \
      return 3;                                                                         \
    }                                                                                   \
  } while (0)

template <typename R> struct cplx;
template <> struct cplx<float> { using T = float2; };
template <> struct cplx<double> { using T = double2; };

/* Per-transform buffers of a batched execute whose inputs or outputs are not N elements apart
 * (fmmfft_execute_many_ptrs): the sections pass reads transform tr from in[tr]; the last FFT
 * pass and the block-DC pass write the rows of transform tr at out[tr].  Passed by value. */
constexpr int kMaxIo = 64; /* transforms of one execute: a batched plan holds at most 64 */
struct InTab {
  const void *p[kMaxIo];
  int n; /* 0: inputs N apart from the execute's d_in */
};
struct OutTab {
  void *p[kMaxIo];
  int rpp; /* the pass's rows per transform; 0: outputs N apart from the execute's d_out */
};

template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
/* a * (h + l) for a twiddle carried as an FP32 pair (h its rounding, l the rounding of the
 * remainder): the small product a l first, then a h added through fused multiply-adds, so the
 * twiddle enters with about 2^-48 relative error instead of its 2^-24 rounding ("compensated"
 * twiddles; the arithmetic's own roundings remain). */
__device__ __forceinline__ float2 cmul_comp(float2 a, float2 h, float2 l) {
  const float tx = a.x * l.x - a.y * l.y, ty = a.x * l.y + a.y * l.x;
  return make_float2(fmaf(a.x, h.x, fmaf(-a.y, h.y, tx)), fmaf(a.x, h.y, fmaf(a.y, h.x, ty)));
}
__device__ __forceinline__ double2 cmul_comp(double2 a, double2 h, double2 l) { /* same, in FP64 */
  const double tx = a.x * l.x - a.y * l.y, ty = a.x * l.y + a.y * l.x;
  return make_double2(fma(a.x, h.x, fma(-a.y, h.y, tx)), fma(a.x, h.y, fma(a.y, h.x, ty)));
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) {
  a.x += b.x, a.y += b.y;
  return a;
}
template <typename C> __device__ __forceinline__ C csub(C a, C b) {
  a.x -= b.x, a.y -= b.y;
  return a;
}

/* ======================================================================== device plan */

/* Stages of one execute, for per-stage CUDA-event timing (fmmfft_profile_*). */
enum { ST_SECTIONS = 0, ST_SUMS, ST_S2M, ST_M2M, ST_TOP, ST_M2L, ST_LEAF, ST_LEAFFIX, ST_COMBINE,
       ST_FFT1, ST_FFT2, ST_DC, ST_COUNT };
static const char *const kStageNames[ST_COUNT] = {
    "sections", "section_sums", "s2m", "m2m", "coarse_tree", "m2l_l2l", "leaf_l2t_near",
    "leaf_halfshift", "combine_dftP", "fft_pass1", "fft_pass2", "block_dc"};

struct Prof {
  int on, cap, count;
  cudaEvent_t *ev; /* cap x (ST_COUNT + 1) */
  int launches[ST_COUNT];
};


template <typename R> struct Dev {
  using C = typename cplx<R>::T;
  long M, P, T, b, s, n, N, S1;
  int precision;
  int nbmax;    /* transforms one execute may carry (the workspace holds nbmax of each array) */
  int last_nbt; /* transforms in the last execute (debug_fetch reads the first of them) */
  /* operators */
  R *initch;  /* [b][T] */
  R *btop;    /* [T][T]       btop[k][t] = topflp[t][k] */
  R *bm2m;    /* [n-2][2T][T] index L-2 for parent level L = 2..n-1 */
  R *bm2l;    /* [n-2][5T][2T] index l-3 for child level l = 3..n */
  R *evalmT;  /* [P-1][T][b]  evalmT[sc-1][k][j] = evalm[j][sc-1][k] */
  R *evalmh;  /* [P-1][T]     row sc-1 used for sc >= P/2 */
  R *cot;     /* [P-1][4b] */
  C *pretw;   /* [P]  c_sc = -exp(-i pi sc/P) sin(pi sc/P) */
  C *twP;     /* [P]  exp(-2 pi i k / P) */
  C *twM;     /* [M]  exp(-2 pi i k / M) */
  /* compensated twiddles (FP32 plans with comp_tw): the FP32 rounding of each entry's remainder */
  C *pretw_lo, *twP_lo, *twM_lo;
  int comp_tw;
  /* workspace */
  R *xt;      /* [2P][M] */
  C *part;    /* [ntile][P] */
  C *ssum;    /* [P] */
  R *phi, *psi; /* per level l: [transform][2(P-1)][2^l][T], levels 2..n back to back */
  R *u;       /* [transform][2(P-1)][M] */
  C *z;       /* [transform][P][M] */
  C *tmp;     /* [transform][P][M] */
  long ntile, tileM;
  long M1, M2; /* size-M FFT split (M2 = 1 when one pass) */
  size_t bytes;
  void *pool;
  Prof prof;
  /* tensor-core (FMMFFT_F32_TC) operators: pre-split TF32 hi/lo, [npad][kpad] K-major */
  int tc, num_sms;
  int *status;          /* device word: non-zero after a bounded device wait gave up */
  /* the section sums run on a stream of their own, forked after the sections pass and joined
   * before the combine (their only reader), so they overlap the tree stages; null: in line */
  cudaStream_t side;
  cudaEvent_t ev_fork, ev_join;
  /* operator images: [0] the row forms' shared-memory image (hi rows then lo rows, K-major
   * core matrices, K extent kpad; 2 kp np floats per level / section), [1] the 16-lane form's
   * (K and N permuted, K extent round16(kp); tc_*_stride16 floats per level / section) */
  float *tc_s2m[2];
  float *tc_m2m[2];     /* per parent level L = 2..n-1 */
  float *tc_m2l[2];     /* per child level l = 3..n */
  float *tc_leaf[2];    /* per section */
  float *tc_lnb[2];     /* the leaf's neighbour-sum operators, per section (row image only) */
  float *leaf_fix;      /* tensor-core leaf, section P/2: [2][s] first points from box-1 */
  float *lnb_w01;       /* neighbour-sum leaf: per section the near-field weights of offsets 0
                         * and -1, applied in FP32 in the epilogue (not in the operator) */
  long tc_m2m_stride, tc_m2l_stride, tc_leaf_stride, tc_lnb_stride; /* kp np */
  long tc_s2m_stride16, tc_m2m_stride16, tc_m2l_stride16, tc_leaf_stride16;
  /* the same operators for the warp-specialised kernel: hi rows then lo rows in the MMA's
   * core-matrix layout (tc::ws_b_index), one block per level or section */
  float *ws_s2m, *ws_m2m, *ws_m2l, *ws_leaf;
  long ws_m2m_stride, ws_m2l_stride, ws_leaf_stride;
  int kp_s2m, np_s2m, kp_m2m, np_m2m, kp_m2l, np_m2l, kp_leaf, np_leaf;
  int ok_s2m, ok_m2m, ok_m2l, ok_leaf;
  int kp_lnb, np_lnb, ok_lnb; /* neighbour-sum leaf (tc::k_tc_nbr): the leaf's default form */
  long tc_min_rows; /* stages with fewer rows use the CUDA-core kernel */
  int fft_threads;  /* threads per block of the register FFT pass (power of two, <= 512) */
  /* tensor-core kernel: 0 row form (32 lanes), 3 row form (16 lanes), 4 warp-specialised; -1
   * per stage: S2M, M2M and M2L the 16-lane row form (form_m2l), the leaf its neighbour-sum form
   * (or the 32-lane window form).  The autotuner chooses among -1, 3 and 4; BF16x3 plans always
   * use 4 (the only BF16x3 kernel). */
  int tc_form;
  int form_m2l; /* M2L's tensor-core form when tc_form does not force one */
  int bf16;    /* FMMFFT_BF16X3: the tensor-core stages in BF16x3 instead of split TF32 */
  int pdl;     /* row-form launches as programmatic dependent launches (FMMFFT_PDL=0: off) */
  unsigned *sync;   /* grid barrier of the coarse-tree kernel: [0] arrivals, [32] generation */
  long coarse_rows; /* levels with fewer rows go to the coarse-tree kernel (0: none) */
  int coarse_grid;  /* blocks of the coarse-tree kernel an SM holds (0: its operators do not fit) */
  int coarse_dbuf;  /* the coarse-tree kernel's operators in two alternating buffers */
  int fuse_s2m;     /* S2M inside the sections pass where tiles hold whole boxes */
  unsigned env_set; /* knobs an environment switch fixed (the autotuner leaves them): bits below */
  int tuned;        /* the knobs come from the autotuner */
};
enum { KNOB_FFT = 1, KNOB_COARSE = 2, KNOB_TCMIN = 4, KNOB_FUSE = 8, KNOB_FORM = 16 };

/* Instantiated CUDA graphs of one plan's execute, keyed by (input, output, direction): the
 * ~35 kernel launches of a transform become one graph launch. */
#define FMMK_GRAPHS 24
#define FMMK_MAX_BATCH 64 /* transforms one batched execute may carry */
struct GraphSlot {
  const void *in;
  void *out;
  int inverse, nbt;
  unsigned long long last_use;
  cudaGraphExec_t exec;
};

/* FP64 residual-correction companion of a complex64 plan (fmmk_refine_enable) */
struct Refine {
  fmmk_state *f64;  /* FP64 plan of the same (N, P, terms, b) */
  float2 *a, *c;    /* [N] complex64 scratch */
  double2 *bq;      /* [N] complex128 scratch */
  size_t bytes;
};

/* Staging of fmmk_execute_host_many: three device buffers of one transform each, so that the
 * copy-in of transform i+1, the execute of transform i and the copy-out of transform i-1 run at
 * once on three streams; events order each buffer's reuse. */
#define FMMK_HOST_SLOTS 3
struct HostPipe {
  void *buf[FMMK_HOST_SLOTS];
  cudaStream_t cin, cout;
  cudaEvent_t in_done[FMMK_HOST_SLOTS], ex_done[FMMK_HOST_SLOTS], out_done[FMMK_HOST_SLOTS];
};

struct fmmk_state {
  int precision;
  void *dev; /* Dev<float> or Dev<double> */
  Refine *refine;
  GraphSlot graphs[FMMK_GRAPHS];
  unsigned long long graph_clock;
  HostPipe *pipe; /* made on the first fmmk_execute_host_many */
};

static void host_pipe_free(HostPipe *hp) {
  if (!hp) return;
  for (int i = 0; i < FMMK_HOST_SLOTS; ++i) {
    if (hp->buf[i]) cudaFree(hp->buf[i]);
    if (hp->in_done[i]) cudaEventDestroy(hp->in_done[i]);
    if (hp->ex_done[i]) cudaEventDestroy(hp->ex_done[i]);
    if (hp->out_done[i]) cudaEventDestroy(hp->out_done[i]);
  }
  if (hp->cin) cudaStreamDestroy(hp->cin);
  if (hp->cout) cudaStreamDestroy(hp->cout);
  free(hp);
}

__host__ __device__ __forceinline__ long lvl_off(long l, long S1, long T) {
  return 2 * S1 * T * ((1L << l) - 4);
}

/* ======================================================================== stage 1-2 */

/* Two FP32 FMAs in one instruction (fma.rn.f32x2, sm_100): d = a * b + c per lane, each an
 * IEEE fused multiply-add rounded to nearest, the same as fmaf. */
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
      "mov.b64 {%0, %1}, rd;\n\t}\n"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}

/* 8 consecutive values into registers (16-byte loads; p 16-byte aligned). */
template <typename R> __device__ __forceinline__ void ld8(const R *p, R *o) {
#pragma unroll
  for (int i = 0; i < 8; ++i) o[i] = p[i];
}
template <> __device__ __forceinline__ void ld8<float>(const float *p, float *o) {
  float4 a = *reinterpret_cast<const float4 *>(p), c = *reinterpret_cast<const float4 *>(p + 4);
  o[0] = a.x, o[1] = a.y, o[2] = a.z, o[3] = a.w, o[4] = c.x, o[5] = c.y, o[6] = c.z, o[7] = c.w;
}
template <> __device__ __forceinline__ void ld8<double>(const double *p, double *o) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    double2 a = *reinterpret_cast<const double2 *>(p + 2 * i);
    o[2 * i] = a.x, o[2 * i + 1] = a.y;
  }
}

/* Deinterleave a tile of TMt points x all P sections into planar sections and write the
 * tile's per-section sums (and, when fused, the S2M of its leaf boxes).
 * x[m*P + sc] -> xt[(2 sc + ri) * M + m]. */
template <typename R>
__global__ void k_sections(const typename cplx<R>::T *__restrict__ x, R *__restrict__ xt,
                           typename cplx<R>::T *__restrict__ part, long M, int P, int TMt,
                           int conj_in, const R *__restrict__ initch, R *__restrict__ phi_n, int b,
                           int T, const InTab xin) {
  using C = typename cplx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  { /* transform blockIdx.y of a batch: inputs N apart, workspace arrays per transform */
    const long tr = blockIdx.y;
    x = xin.n ? reinterpret_cast<const C *>(xin.p[tr]) : x + tr * M * P;
    xt += tr * 2 * M * P, part += tr * (long)gridDim.x * P;
    if (phi_n != nullptr) phi_n += tr * 2 * (long)(P - 1) * (M / b) * T;
  }
  C *tile = reinterpret_cast<C *>(smem_raw); /* [TMt][P + 1]: the pad spreads a column over banks */
  R *ich = reinterpret_cast<R *>(tile + (long)TMt * (P + 1)); /* initch [b][T] when S2M is fused */
  const int PP = P + 1, lp = __ffs(P) - 1, lt = __ffs(TMt) - 1;
  const long m0 = (long)blockIdx.x * TMt;
  const int E = TMt * P;
  /* loads issued 8 at a time before their stores, so their latencies overlap */
  for (int e0 = threadIdx.x; e0 < E; e0 += 8 * blockDim.x) {
    C v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e < E) v[u] = x[m0 * P + e];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e < E) {
        if (conj_in) v[u].y = -v[u].y;
        tile[(e >> lp) * PP + (e & (P - 1))] = v[u];
      }
    }
  }
  if (phi_n != nullptr)
    for (int e = threadIdx.x; e < b * T; e += blockDim.x) ich[e] = initch[e];
  __syncthreads();
  /* planar stores: point mm of section sc to planes 2sc (re) and 2sc+1 (im), TMt contiguous
   * points a plane */
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    const int mm = e & (TMt - 1), sc = e >> lt;
    const C v = tile[mm * PP + sc];
    R *dst = xt + (long)(2 * sc) * M + m0 + mm;
    dst[0] = v.x;
    dst[M] = v.y;
  }
  /* S2M of the tile's leaf boxes (reference initmm, fmmfft.c:199-211), when the tile holds
   * whole boxes (b | TMt) and T % 4 == 0: phi_n[(2(sc-1) + ri) s + box][k] =
   * sum_j x_sc[box b + j] initch[j][k].  Work item: one section, 4 consecutive k, both planes;
   * the P tile sums are extra work items, so no thread waits for another. */
  /* work item: sections sc, sc + 1 (sc odd; the last one alone when P - 1 is odd), 4 k */
  const int T4 = T >> 2, nbox = phi_n != nullptr ? TMt / b : 0, npair = P / 2;
  const int nitems = nbox * npair * T4;
  for (int o = threadIdx.x; o < nitems + P; o += blockDim.x) {
    if (o >= nitems) { /* tile sum of one section, fixed order */
      const int sc = o - nitems;
      C acc;
      acc.x = 0, acc.y = 0;
      for (int mm = 0; mm < TMt; ++mm) acc = cadd(acc, tile[mm * PP + sc]);
      part[(long)blockIdx.x * P + sc] = acc;
      continue;
    }
    const long s = M / b;
    const int k0 = (o % T4) * 4, rest = o / T4, sc = 2 * (rest % npair) + 1, bx = rest / npair;
    const bool two = sc + 1 <= P - 1;
    R re[2][4] = {}, im[2][4] = {};
    if constexpr (sizeof(R) == 4) { /* (re, im) of one point in one f32x2 FMA per weight */
      float2 acc[2][4];
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[h][q] = make_float2(0.f, 0.f);
      for (int j = 0; j < b; ++j) {
        const C *tr = tile + (bx * b + j) * PP + sc;
        const C v0 = tr[0], v1 = two ? tr[1] : C{0.f, 0.f};
        const float4 w = *reinterpret_cast<const float4 *>(ich + j * T + k0);
        const float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc[0][q] = ffma2(v0, make_float2(wv[q], wv[q]), acc[0][q]);
          acc[1][q] = ffma2(v1, make_float2(wv[q], wv[q]), acc[1][q]);
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int q = 0; q < 4; ++q) re[h][q] = acc[h][q].x, im[h][q] = acc[h][q].y;
    } else {
      for (int j = 0; j < b; ++j) {
        const C *tr = tile + (bx * b + j) * PP + sc;
        const C v0 = tr[0];
        C v1;
        v1.x = 0, v1.y = 0;
        if (two) v1 = tr[1];
        const R *w = ich + j * T + k0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          re[0][q] = fma(v0.x, w[q], re[0][q]), im[0][q] = fma(v0.y, w[q], im[0][q]);
          re[1][q] = fma(v1.x, w[q], re[1][q]), im[1][q] = fma(v1.y, w[q], im[1][q]);
        }
      }
    }
    const long box = m0 / b + bx;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h == 1 && !two) break;
      R *pr = phi_n + ((2L * (sc + h - 1)) * s + box) * T + k0, *pi = pr + s * T;
      if constexpr (sizeof(R) == 4) { /* 16-byte aligned: T and k0 are multiples of 4 */
        *reinterpret_cast<float4 *>(pr) = make_float4(re[h][0], re[h][1], re[h][2], re[h][3]);
        *reinterpret_cast<float4 *>(pi) = make_float4(im[h][0], im[h][1], im[h][2], im[h][3]);
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) pr[q] = re[h][q], pi[q] = im[h][q];
      }
    }
  }
}

/* ssum[sc] = sum over tiles of part[tile][sc]: fixed-shape tree, so results do not depend on
 * scheduling. */
template <typename R>
__global__ void k_sum_sections(const typename cplx<R>::T *__restrict__ part, long ntile, int P,
                               typename cplx<R>::T *__restrict__ ssum) {
  using C = typename cplx<R>::T;
  __shared__ C red[256];
  const int sc = blockIdx.x;
  part += (long)blockIdx.y * ntile * P, ssum += (long)blockIdx.y * P; /* transform of a batch */
  C acc;
  acc.x = 0, acc.y = 0;
  /* loads 8 at a time, additions in the same fixed order */
  for (long t0 = threadIdx.x; t0 < ntile; t0 += 8L * blockDim.x) {
    C v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const long t = t0 + (long)u * blockDim.x;
      if (t < ntile) v[u] = part[t * P + sc];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (t0 + (long)u * blockDim.x < ntile) acc = cadd(acc, v[u]);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) ssum[sc] = red[0];
}

/* ======================================================================== rowgemm */
/* D[r][n] = sum_k A(r,k) B(k,n) for rows r < rows, n < N.  A rows are gathered from the
 * stage's arrays by the problem object; B is a dense operator in global memory or generated
 * (leaf).  Tile BM x BN x BK; each thread owns a TM x TN block of outputs. */

template <typename R> struct ProbS2M { /* batch z = transform: its sections 1..P-1, planar */
  const R *xt, *B;
  R *out;
  long rows, M; /* rows per transform: 2 (P - 1) s */
  int K, N, P;
  const R *xs;
  R *os;
  __device__ void begin(int z) { xs = xt + (2L * P * z + 2) * M, os = out + (long)z * rows * N; }
  __device__ R a(long r, int k) const { return xs[r * K + k]; }
  __device__ R bv(int k, int n) const { return B[k * N + n]; }
  __device__ R *d(long r) const { return os + r * N; }
};

template <typename R> struct ProbM2M { /* parent level L: A row = children pair of level L+1 */
  const R *child, *B;
  R *out;
  long rows;
  int K, N;
  __device__ void begin(int) {}
  __device__ R a(long r, int k) const { return child[r * K + k]; }
  __device__ R bv(int k, int n) const { return B[k * N + n]; }
  __device__ R *d(long r) const { return out + r * N; }
};

template <typename R> struct ProbTop { /* level 2: psi[c] = topflp . phi[c+2 mod 4] */
  const R *phi2, *B;
  R *out;
  long rows;
  int K, N;
  __device__ void begin(int) {}
  __device__ R a(long r, int k) const {
    long pl = r >> 2, c = r & 3;
    return phi2[(pl * 4 + ((c + 2) & 3)) * K + k];
  }
  __device__ R bv(int k, int n) const { return B[k * N + n]; }
  __device__ R *d(long r) const { return out + r * N; }
};

/* Child level l, one row per parent box B (plane pl): A = [psi_{l-1}[B] | phi_l[2B-2, 2B-1] |
 * phi_l[2B+2, 2B+3]] (K = 5T), output = psi_l[2B], psi_l[2B+1] (N = 2T). */
template <typename R> struct ProbM2L {
  const R *psi_par, *phi, *B;
  R *out;
  long rows;
  int K, N, T, lpar; /* lpar = l - 1 */
  __device__ void begin(int) {}
  __device__ R a(long r, int k) const {
    if (k < T) return psi_par[r * T + k];
    long pl = r >> lpar, Bx = r & ((1L << lpar) - 1), mask = (2L << lpar) - 1;
    long base = pl << (lpar + 1);
    if (k < 3 * T) return phi[(base + ((2 * Bx - 2) & mask)) * T + (k - T)];
    return phi[(base + ((2 * Bx + 2) & mask)) * T + (k - 3 * T)];
  }
  __device__ R bv(int k, int n) const { return B[k * N + n]; }
  __device__ R *d(long r) const { return out + r * N; }
};

/* Leaf stage for one section (batch z = sc - 1): rows (ri, box), A = [psi_n[box] | x_sc over
 * boxes box-1..box+1] (K = T + 3b), B = [E_sc ; Toeplitz cot], output u[plane][box*b + j]. */
template <typename R> struct ProbLeaf {
  const R *psi_n, *xt, *evalmT, *cot;
  R *u;
  long rows, M, s;
  int K, N, T, b;
  /* per batch */
  const R *ps, *xs, *E, *ct;
  R *us;
  __device__ void begin(int z) {
    long pl0 = 2L * z;
    ps = psi_n + pl0 * s * T;
    xs = xt + (pl0 + 2) * M;
    E = evalmT + (long)z * T * b;
    ct = cot + (long)z * 4 * b;
    us = u + pl0 * M;
  }
  __device__ R a(long r, int k) const {
    if (k < T) return ps[r * T + k];
    long ri = r / s, bx = r - ri * s;
    long m = (bx * b - b + (k - T)) & (M - 1);
    return xs[ri * M + m];
  }
  __device__ R bv(int k, int n) const {
    if (k < T) return E[k * b + n];
    return ct[(k - T) + b - n];
  }
  __device__ R *d(long r) const {
    long ri = r / s, bx = r - ri * s;
    return us + ri * M + bx * b;
  }
};

/* ---- the same four contractions for the tcgen05 kernel (fmmfft_tc.cuh) ---- */
struct TcBase {
  long rows;
  int batches, nchunks, clen[4], coff[4], kpad, npad, nout;
  /* the operator of batch z as the row forms' shared-memory image (bimg + z bimg_stride) and
   * as the 16-lane form's (bimg16 + z bimg16_stride); either may be null when its form is unused */
  const float *bimg, *bimg16;
  long bimg_stride, bimg16_stride;
  const float *wsb; /* warp-specialised form: operator of batch z at wsb + z * wsb_stride */
  long wsb_stride;
  int nap; /* ns an epilogue warp sleeps between failed polls (producers nap / 4, MMA nap / 8) */
  static constexpr bool kEpiAlternate = false; /* row-form epilogue: one half of N per warp */
  /* output columns c0..c0+7 of a row into dst (columns below nout; nout a multiple of 4) */
  __device__ void put8(float *dst, long, int, int c0, const float *t) const {
    if (c0 + 8 <= nout) {
      *reinterpret_cast<float4 *>(dst + c0) = make_float4(t[0], t[1], t[2], t[3]);
      *reinterpret_cast<float4 *>(dst + c0 + 4) = make_float4(t[4], t[5], t[6], t[7]);
    } else if (c0 + 4 <= nout) {
      *reinterpret_cast<float4 *>(dst + c0) = make_float4(t[0], t[1], t[2], t[3]);
    }
  }
  /* output columns c..c+3 of a row (16-lane row form; c a multiple of 4) */
  __device__ void put4(float *dst, long, int, int c, float4 v) const {
    if (c + 4 <= nout) *reinterpret_cast<float4 *>(dst + c) = v;
  }
};

struct TcS2M : TcBase { /* batch z = transform (one operator for all: wsb_stride 0) */
  const float *xt;
  float *out;
  long M;
  int b, T, P;
  __device__ const float *src(int, long r, int z) const { return xt + (2L * P * z + 2) * M + r * b; }
  __device__ float *dst(long r, int z) const { return out + ((long)z * rows + r) * T; }
};

struct TcM2M : TcBase {
  const float *child;
  float *out;
  int T;
  __device__ const float *src(int, long r, int) const { return child + r * 2 * T; }
  __device__ float *dst(long r, int) const { return out + r * T; }
};

struct TcM2L : TcBase {
  const float *psi_par, *phi;
  float *out;
  int T, lpar;
  __device__ const float *src(int c, long r, int) const {
    if (c == 0) return psi_par + r * T;
    long pl = r >> lpar, Bx = r & ((1L << lpar) - 1), mask = (2L << lpar) - 1;
    long base = pl << (lpar + 1);
    long box = (c == 1) ? ((2 * Bx - 2) & mask) : ((2 * Bx + 2) & mask);
    return phi + (base + box) * T;
  }
  __device__ float *dst(long r, int) const { return out + r * 2 * T; }
};

/* Leaf far field + near field of one section per batch (reference fmmfft.c:751-954).  The
 * operator has b + 1 output columns: columns [0, b) are the box's targets; column b, for sections
 * sc >= P/2, is the first target of the NEXT box shifted back into this one (weights evalmh and
 * cot[0..3b), over exactly this row's A: the expansion of box B-1 and the window B-2..B), the
 * reference's half-shifted first point (:771-803, :839-954).  For sc > P/2 that value replaces
 * the next box's in-box first point, which is then not stored; for sc = P/2 it goes to fixbuf
 * and k_leaf_mid averages the two. */
struct TcLeaf : TcBase { /* batch z = section - 1; s is a power of two (log2s) */
  /* N = b + 1 padded to a multiple of 16: the upper half of N holds few stored columns, so the
   * epilogue's 8-column chunks go alternately to the two halves of the warps */
  static constexpr bool kEpiAlternate = true;
  const float *psi_n, *xt;
  float *u, *fixbuf;
  long M, s;
  int T, b, log2s, P;
  /* row r = (transform tr, plane ri, box bx), r = (2 tr + ri) s + bx; plane pl of transform tr
   * (pl = 2 z + ri) is expansion / field plane tr (2 (P - 1)) + pl and sample plane tr 2 P + pl + 2 */
  __device__ long plane(long r, int z) const {
    return (r >> (log2s + 1)) * 2 * (P - 1) + 2L * z + ((r >> log2s) & 1);
  }
  __device__ const float *src(int c, long r, int z) const {
    const long bx = r & (s - 1), pl = plane(r, z);
    if (c == 0) return psi_n + (pl * s + bx) * T;
    return xt + (pl + 2 * (r >> (log2s + 1)) + 2) * M + (((bx - 2 + c) * b) & (M - 1));
  }
  __device__ float *dst(long r, int z) const { return u + plane(r, z) * M + (r & (s - 1)) * b; }
  const float *w01; /* per section z: the near-field weights of offsets 0 and -1 (not in B) */
  /* adds w0 x[j] + w1 x[j-1] (FP32) to outputs j = c .. c+n-1 (those below b) of row r's box */
  __device__ void near01(long r, int z, int c, int n, float *t) const {
    const long bx = r & (s - 1), pl = plane(r, z);
    const float *xp = xt + (pl + 2 * (r >> (log2s + 1)) + 2) * M;
    const long j0 = bx * b + c;
    const float w0 = w01[2 * z], w1 = w01[2 * z + 1];
    float prev = xp[(j0 - 1) & (M - 1)];
    for (int i = 0; i < n && c + i < b; ++i) {
      const float xi = xp[j0 + i];
      t[i] = fmaf(w0, xi, fmaf(w1, prev, t[i]));
      prev = xi;
    }
  }
  __device__ void put8(float *dst, long r, int z, int c0, const float *t0) const {
    const int sc = z + 1;
    const bool shifted = 2 * sc > P; /* the in-box first point is replaced */
    float t[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i] = t0[i];
    near01(r, z, c0, 8, t);
    if (c0 + 4 <= b) {
      if (c0 == 0 && shifted) {
        dst[1] = t[1], dst[2] = t[2], dst[3] = t[3];
      } else {
        *reinterpret_cast<float4 *>(dst + c0) = make_float4(t[0], t[1], t[2], t[3]);
      }
      if (c0 + 8 <= b) *reinterpret_cast<float4 *>(dst + c0 + 4) = make_float4(t[4], t[5], t[6], t[7]);
    }
    if (2 * sc >= P && c0 <= b && b < c0 + 8) { /* column b: b - c0 is 0 or 4 */
      const float v = b == c0 ? t[0] : t[4];
      const long nb = (r + 1) & (s - 1);
      if (shifted)
        u[plane(r, z) * M + nb * b] = v;
      else
        fixbuf[((r >> log2s) << log2s) + nb] = v; /* [transform][plane][box] */
    }
  }
  __device__ void put4(float *dst, long r, int z, int c, float4 v) const { /* c a multiple of 4 */
    const int sc = z + 1;
    if (c < b) {
      float t[4] = {v.x, v.y, v.z, v.w};
      near01(r, z, c, 4, t);
      v = make_float4(t[0], t[1], t[2], t[3]);
      if (c == 0 && 2 * sc > P) /* the in-box first point is replaced */
        dst[1] = v.y, dst[2] = v.z, dst[3] = v.w;
      else
        *reinterpret_cast<float4 *>(dst + c) = v;
    } else if (c == b && 2 * sc >= P) { /* column b */
      const long nb = (r + 1) & (s - 1);
      if (2 * sc > P)
        u[plane(r, z) * M + nb * b] = v.x;
      else
        fixbuf[((r >> log2s) << log2s) + nb] = v.x;
    }
  }
};

/* The same leaf in neighbour-sum form (tc::k_tc_nbr): row r = (transform, plane, box B) holds
 * only box B's own data, A = [psi_B (T) | x_B (b)], and the operator of section sc has the
 * column blocks
 *   [0, b)     box B's targets: far field (evalm) + x_B as the window's middle box,
 *   [b, 2b)    box B+1's targets: x_B as the first box of B+1's window,
 *   [2b, 3b)   box B-1's targets: x_B as the last box of B-1's window,
 *   3b .. 3b+2 (sc >= P/2) the half-shifted first point H(B) of box B+1 (evalmh, and x_B as the
 *              middle of the window B-1..B+1), x_B's part of H(B+1), x_B's part of H(B-1);
 * the kernel adds the blocks of rows B-1, B, B+1.  Each sample is loaded and split once per row
 * instead of three times (K = T + b instead of T + 3b). */
struct TcLeafNb : TcLeaf {
  long strips;
  /* adds w0 x[j] + w1 x[j-1] (FP32) to targets j = c0 .. c0+7 of a row, x = x[c0-1 .. c0+7] */
  __device__ void fix_apply(int z, const float (&x)[9], float *t) const {
    const float w0 = w01[2 * z], w1 = w01[2 * z + 1];
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i] = fmaf(w0, x[i + 1], fmaf(w1, x[i], t[i]));
  }
  __device__ const float *src(int c, long r, int z) const {
    const long bx = r & (s - 1), pl = plane(r, z);
    if (c == 0) return psi_n + (pl * s + bx) * T;
    return xt + (pl + 2 * (r >> (log2s + 1)) + 2) * M + bx * b;
  }
  __device__ bool has_h(int z) const { return 2 * (z + 1) >= P; }
  __device__ void put8_nb(long r, int z, int c0, const float *t) const {
    float *dst = u + plane(r, z) * M + (r & (s - 1)) * b;
    if (c0 == 0 && 2 * (z + 1) > P) /* the in-box first point is replaced by H(B - 1) */
      dst[1] = t[1], dst[2] = t[2], dst[3] = t[3];
    else
      *reinterpret_cast<float4 *>(dst + c0) = make_float4(t[0], t[1], t[2], t[3]);
    *reinterpret_cast<float4 *>(dst + c0 + 4) = make_float4(t[4], t[5], t[6], t[7]);
  }
  __device__ void put_h(long r, int z, float v) const { /* H(B): first point of box B + 1 */
    const long nb = (r + 1) & (s - 1);
    if (2 * (z + 1) > P)
      u[plane(r, z) * M + nb * b] = v;
    else
      fixbuf[((r >> log2s) << log2s) + nb] = v;
  }
};

template <typename R, int BM, int BN, int BK, int TM, int TN, class Prob>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) k_rowgemm(Prob pb) {
  constexpr int NTX = BN / TN;
  constexpr int NT = (BM / TM) * NTX;
  __shared__ R As[BK][BM + 1];
  __shared__ R Bs[BK][BN + 1];
  const int tid = threadIdx.x;
  const int tn = tid % NTX, tm = tid / NTX;
  const long row0 = (long)blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  pb.begin(blockIdx.z);
  R acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = R(0);
  for (int k0 = 0; k0 < pb.K; k0 += BK) {
    for (int e = tid; e < BM * BK; e += NT) {
      int m = e / BK, kk = e - m * BK;
      long r = row0 + m;
      int k = k0 + kk;
      As[kk][m] = (r < pb.rows && k < pb.K) ? pb.a(r, k) : R(0);
    }
    for (int e = tid; e < BK * BN; e += NT) {
      int kk = e / BN, nn = e - kk * BN;
      int k = k0 + kk, nc = n0 + nn;
      Bs[kk][nn] = (k < pb.K && nc < pb.N) ? pb.bv(k, nc) : R(0);
    }
    __syncthreads();
    /* Each BK slice is summed into its own partial before it joins the running total, so
     * FP32 rounding grows like sqrt(BK) + sqrt(K/BK) instead of sqrt(K) for long K (the
     * 3b-point near-field windows reach K = 6160 at b = 2048). */
    R part[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) part[i][j] = R(0);
#pragma unroll 4
    for (int kk = 0; kk < BK; ++kk) {
      R av[TM], bw[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) av[i] = As[kk][tm * TM + i];
#pragma unroll
      for (int j = 0; j < TN; ++j) bw[j] = Bs[kk][tn * TN + j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) part[i][j] = fma(av[i], bw[j], part[i][j]);
    }
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] += part[i][j];
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    long r = row0 + tm * TM + i;
    if (r >= pb.rows) continue;
    R *dst = pb.d(r);
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      int nc = n0 + tn * TN + j;
      if (nc < pb.N) dst[nc] = acc[i][j];
    }
  }
}

template <typename R, class Prob>
static void launch_rowgemm(const Prob &pb, long rows_per_batch, int N, int batches,
                           cudaStream_t st) {
  if (rows_per_batch <= 32 && N > 64) {
    dim3 g((unsigned)((rows_per_batch + 15) / 16), (unsigned)((N + 63) / 64), batches);
    k_rowgemm<R, 16, 64, 16, 2, 2, Prob><<<g, 256, 0, st>>>(pb);
  } else if (N <= 32) {
    dim3 g((unsigned)((rows_per_batch + 127) / 128), 1, batches);
    k_rowgemm<R, 128, 32, 16, 8, 4, Prob><<<g, 128, 0, st>>>(pb);
  } else {
    dim3 g((unsigned)((rows_per_batch + 63) / 64), (unsigned)((N + 63) / 64), batches);
    k_rowgemm<R, 64, 64, 16, 4, 4, Prob><<<g, 256, 0, st>>>(pb);
  }
}

constexpr long kTcMinRows = 4096; /* default: below this a stage runs on the CUDA-core kernel */

template <class Prob> static size_t tc_smem_bytes(const Prob &pb) {
  return tc::smem_bytes(pb.kpad, pb.npad);
}

static int ws_nap_ns() {
  static int v = -1;
  if (v < 0) {
    const char *ev = getenv("FMMFFT_WS_NAP");
    v = ev ? atoi(ev) : 256;
    if (v < 0 || v > 100000) v = 256;
  }
  return v;
}

template <class Prob>
static void launch_tc(const Prob &pb0, int num_sms, int *status, cudaStream_t st, int form, int pdl,
                      int bf16 = 0) {
  Prob pb = pb0;
  pb.nap = ws_nap_ns();
  if (bf16) form = 4; /* BF16x3 exists in the warp-specialised form only */
  if (!tc::ws_fits(pb.kpad, pb.npad)) form = form == 4 ? 0 : form;
  if (form == 4 && tc::ws_fits(pb.kpad, pb.npad)) {
    const long tiles = (pb.rows + tc::kRows - 1) / tc::kRows * pb.batches;
    const int grid = (int)(tiles < num_sms ? tiles : num_sms); /* one CTA per SM: all of TMEM */
    const size_t smem = tc::ws_smem_bytes(pb.kpad, pb.npad, bf16 ? 2 : 4);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(tc::kWThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    if (bf16)
      cudaLaunchKernelEx(&cfg, tc::k_tc_ws<Prob, true>, pb, status);
    else
      cudaLaunchKernelEx(&cfg, tc::k_tc_ws<Prob, false>, pb, status);
    return;
  }
  long tiles = (pb.rows + tc::kRows - 1) / tc::kRows * pb.batches;
  long cap = 2L * num_sms; /* two CTAs per SM */
  int grid = (int)(tiles < cap ? tiles : cap);
  const bool r16 = form == 3; /* the 16-lane row form */
  const size_t smem = r16 ? tc::smem16_bytes(pb.kpad, pb.npad) : tc_smem_bytes(pb);
  if (pdl) {
    /* programmatic dependent launch: the CTAs may start (and stage their operator) while the
     * kernel before them finishes; the kernel waits for it before touching its data.  Only the
     * row form is launched this way: two CTAs per SM by registers, so a waiting CTA never sits
     * on tensor memory that a running one needs. */
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (r16)
      cudaLaunchKernelEx(&cfg, tc::k_tc_rowgemm16<Prob>, pb, status);
    else
      cudaLaunchKernelEx(&cfg, tc::k_tc_rowgemm<Prob>, pb, status);
    return;
  }
  if (r16)
    tc::k_tc_rowgemm16<Prob><<<grid, 256, smem, st>>>(pb, status);
  else
    tc::k_tc_rowgemm<Prob><<<grid, 256, smem, st>>>(pb, status);
}

/* The neighbour-sum row form (tc::k_tc_nbr), persistent, two CTAs per SM; launched like the
 * row form (programmatic dependent launch unless pdl is 0). */
template <class Prob> static void launch_nb(const Prob &pb, int num_sms, int *status, cudaStream_t st, int pdl) {
  const long tps = (pb.s + tc::kNbOut - 1) / tc::kNbOut;
  const long tiles = tps * pb.strips * pb.batches;
  const long cap = 2L * num_sms;
  const int grid = (int)(tiles < cap ? tiles : cap);
  const size_t smem = tc::smem_bytes(pb.kpad, pb.npad);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, tc::k_tc_nbr<Prob>, pb, status);
}

/* First point of each leaf box for the sections whose shifted target leaves its box
 * (sc >= P/2): reference fmmfft.c:771-803 (far) and :839-954 (near).  For sc > P/2 the value
 * comes from box-1 (local expansion evalmh, window box-2..box with the cotsh offsets); for
 * sc = P/2 it is the mean of that and the in-box value the contraction stored.
 * One warp per box: the lanes take the T far-field terms and the 3b window points (consecutive
 * lanes on consecutive points, so every load is coalesced), then a warp sum.  Block: 8 warps,
 * kFixBoxes boxes per warp, all of one section (grid y). */
constexpr int kFixBoxes = 8;
template <typename R>
__global__ void __launch_bounds__(256) k_leaf_fix(const R *__restrict__ psi_n, const R *__restrict__ xt,
                                                  const R *__restrict__ evalmh, const R *__restrict__ cot,
                                                  R *__restrict__ u, long M, long s, int log2s, int T, int b,
                                                  int P) {
  const int sc = P / 2 + blockIdx.y; /* sc in [P/2, P-1] */
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  { /* transform blockIdx.z of a batch */
    const long tr = blockIdx.z;
    psi_n += tr * 2 * (P - 1) * s * T, xt += tr * 2 * P * M, u += tr * 2 * (P - 1) * M;
  }
  const R *eh = evalmh + (long)(sc - 1) * T;
  const R *ct = cot + (long)(sc - 1) * 4 * b;
  const long i0 = ((long)blockIdx.x * 8 + warp) * kFixBoxes;
  for (int t = 0; t < kFixBoxes; ++t) {
    const long idx = i0 + t;
    if (idx >= 2 * s) break; /* warp-uniform */
    const long ri = idx >> log2s, bx = idx & (s - 1);
    const long pl = 2L * (sc - 1) + ri;
    const R *pp = psi_n + (pl * s + ((bx - 1) & (s - 1))) * T;
    const R *xs = xt + (pl + 2) * M;
    R acc = 0;
    for (int k = lane; k < T; k += 32) acc = fma(pp[k], eh[k], acc);
    for (int q = lane; q < 3 * b; q += 32) acc = fma(xs[(bx * b - 2 * b + q) & (M - 1)], ct[q], acc);
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      R *dst = u + pl * M + bx * b;
      if (2 * sc > P)
        *dst = acc;
      else
        *dst = R(0.5) * (*dst + acc);
    }
  }
}

/* Section sc = P/2 after the tensor-core leaf: the first point of each box is the mean of the
 * in-box value and the value from box-1's expansion, which the contraction left in fixbuf
 * ([2][s]; reference fmmfft.c:771-803, :839-954). */
template <typename R>
__global__ void k_leaf_mid(R *__restrict__ u, const float *__restrict__ fixbuf, long M, long s, int log2s, int b,
                           int P) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 2 * s) return;
  const long ri = idx >> log2s, bx = idx & (s - 1), tr = blockIdx.y;
  R *dst = u + (tr * 2 * (P - 1) + 2L * (P / 2 - 1) + ri) * M + bx * b;
  *dst = R(0.5) * (*dst + (R)fixbuf[tr * 2 * s + idx]);
}

/* Leaf stage, direct form (b a multiple of 8): far field (L2T) plus near field of one re/im
 * plane of one section for NB consecutive leaf boxes (reference fmmfft.c:751-954).
 *
 * Each thread computes 8 consecutive targets j0..j0+7 of one box:
 *   u[j] = sum_k psi[box][k] E_sc[k][j] + sum_{q < 3b} x[(box-1) b + q] cot_sc[q + b - j],
 * the near-field coefficients of the 8 targets are a sliding window of the Toeplitz row, so
 * per 8 window points the thread loads 8 x values and 16 cot values (vector loads from shared
 * memory) for 64 FMAs.  The first point of each box for sc >= P/2 (target shifted into the
 * previous box) is evaluated from box-1's local expansion (evalmh) and the window box-2..box,
 * and for sc = P/2 averaged with the in-box value, as the reference does (:771-803, :839-954).
 * Block: 256 threads, grid (boxes / NB, 2 (P-1) planes). */

/* 16-byte vector of R (float4 / double2) for the shared-memory staging copies. */
template <typename R> struct vec16;
template <> struct vec16<float> { using T = float4; };
template <> struct vec16<double> { using T = double2; };

/* Shared-memory row pitch for n values: a multiple of 4 whose quarter is odd, so that rows of
 * consecutive boxes start in different 16-byte bank groups. */
__host__ __device__ __forceinline__ long skew_pitch(long n) {
  long p = (n + 3) & ~3L;
  return ((p >> 2) & 1) ? p : p + 4;
}

template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 1) k_leaf(const R *__restrict__ psi_n, const R *__restrict__ xt,
                                              const R *__restrict__ evalmT, const R *__restrict__ evalmh,
                                              const R *__restrict__ cot, R *__restrict__ u, long M,
                                              long s, int T, int b, int P, int NB, int e_in_smem) {
  using V = typename vec16<R>::T;
  constexpr int VW = 16 / sizeof(R); /* values per 16-byte vector */
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long xp = skew_pitch(b), tp = skew_pitch(T);
  R *xw = reinterpret_cast<R *>(smem_raw); /* boxes B0-2 .. B0+NB, one row of pitch xp each */
  R *ps = xw + (long)(NB + 3) * xp;        /* psi of boxes B0-1 .. B0+NB-1, pitch tp */
  R *ct = ps + (((long)(NB + 1) * tp + 7) & ~7L); /* 4b */
  R *cts = ct + 4 * b;                     /* 4b: cts[e] = ct[e + 1] (FP32 pairs of odd offset) */
  R *eh = cts + 4 * b;                     /* T (rounded up to 8) */
  R *Es = eh + ((T + 7) & ~7);             /* T b when e_in_smem */
  { /* transform blockIdx.z of a batch */
    const long tr = blockIdx.z;
    psi_n += tr * 2 * (P - 1) * s * T, xt += tr * 2 * P * M, u += tr * 2 * (P - 1) * M;
  }
  const int pl = blockIdx.y, sc = pl / 2 + 1;
  const long B0 = (long)blockIdx.x * NB;
  const R *xs = xt + (long)(pl + 2) * M;
  const R *pp = psi_n + (long)pl * s * T;
  const R *E = evalmT + (long)(sc - 1) * T * b;
  const R *cg = cot + (long)(sc - 1) * 4 * b;
  const bool shifted = 2 * sc >= P;
  /* staging, 16 bytes per load where rows allow (b is a power of two >= 8) */
  {
    const int lv = __ffs(b / VW) - 1; /* vectors per x row = b / VW, a power of two */
    const int nx = (NB + 3) * (b / VW);
    for (int e0 = threadIdx.x; e0 < nx; e0 += 4 * blockDim.x) { /* 4 loads in flight */
      V v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * blockDim.x, row = e >> lv, c = e & ((b / VW) - 1);
        if (e < nx) v[u] = *reinterpret_cast<const V *>(xs + ((B0 - 2 + row) & (s - 1)) * b + c * VW);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * blockDim.x, row = e >> lv, c = e & ((b / VW) - 1);
        if (e < nx) *reinterpret_cast<V *>(xw + (long)row * xp + c * VW) = v[u];
      }
    }
  }
  if (T % VW == 0) {
    const int tv = T / VW, np_ = (NB + 1) * tv;
    for (int e0 = threadIdx.x; e0 < np_; e0 += 4 * blockDim.x) { /* 4 loads in flight */
      V v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * blockDim.x, bx = e / tv, c = e - bx * tv;
        if (e < np_) v[u] = *reinterpret_cast<const V *>(pp + ((B0 - 1 + bx) & (s - 1)) * T + c * VW);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * blockDim.x, bx = e / tv, c = e - bx * tv;
        if (e < np_) *reinterpret_cast<V *>(ps + (long)bx * tp + c * VW) = v[u];
      }
    }
  } else {
    for (int e = threadIdx.x; e < (NB + 1) * T; e += blockDim.x) {
      const int bx = e / T, k = e - bx * T; /* 32-bit division */
      ps[(long)bx * tp + k] = pp[((B0 - 1 + bx) & (s - 1)) * T + k];
    }
  }
  for (int e = threadIdx.x; e < 4 * b / VW; e += blockDim.x)
    reinterpret_cast<V *>(ct)[e] = reinterpret_cast<const V *>(cg)[e];
  for (int e = threadIdx.x; e < 4 * b; e += blockDim.x) cts[e] = e + 1 < 4 * b ? cg[e + 1] : R(0);
  if (shifted)
    for (int e = threadIdx.x; e < T; e += blockDim.x) eh[e] = evalmh[(long)(sc - 1) * T + e];
  if (e_in_smem)
    for (long e = threadIdx.x; e < (long)T * b / VW; e += blockDim.x)
      reinterpret_cast<V *>(Es)[e] = reinterpret_cast<const V *>(E)[e];
  __syncthreads();
  const R *Eu = e_in_smem ? Es : E;
  const int G = b >> 3; /* threads per box */
  for (int w = threadIdx.x; w < NB * G; w += blockDim.x) {
    const int bi = w / G, j0 = (w - bi * G) * 8;
    R acc[8];
    const R *pr = ps + (long)(bi + 1) * tp;
    if constexpr (sizeof(R) == 4) {
      /* far field, targets paired: acc[2h], acc[2h+1] in one f32x2 FMA */
      float2 a2[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) a2[h] = make_float2(0.f, 0.f);
      for (int k = 0; k < T; ++k) {
        R e8[8];
        ld8<R>(Eu + (long)k * b + j0, e8);
        const float2 a = make_float2(pr[k], pr[k]);
#pragma unroll
        for (int h = 0; h < 4; ++h) a2[h] = ffma2(a, make_float2(e8[2 * h], e8[2 * h + 1]), a2[h]);
      }
#pragma unroll
      for (int h = 0; h < 4; ++h) acc[2 * h] = a2[h].x, acc[2 * h + 1] = a2[h].y;
    } else {
#pragma unroll
      for (int t = 0; t < 8; ++t) acc[t] = R(0);
      for (int k = 0; k < T; ++k) {
        R e8[8];
        ld8<R>(Eu + (long)k * b + j0, e8);
        const R a = pr[k];
#pragma unroll
        for (int t = 0; t < 8; ++t) acc[t] = fma(a, e8[t], acc[t]);
      }
    }
    /* near field over boxes box-1 .. box+1; each box's part is summed separately before it
     * joins the total (long windows, b up to 2048, keep their FP32 rounding small) */
#pragma unroll 1
    for (int seg = 0; seg < 3; ++seg) {
      const R *xr = xw + (long)(bi + 1 + seg) * xp; /* xw row i holds box B0 - 2 + i */
      R part[8];
      if constexpr (sizeof(R) == 4) {
        /* window points paired: even and odd points of target t accumulate in the two lanes
         * of p2[t]; their weights (w[m], w[m+1]), m = 2p - t + 8, are an aligned pair of ct
         * for even t and of the shifted copy cts for odd t */
        float2 p2[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) p2[t] = make_float2(0.f, 0.f);
        for (int q = 0; q < b; q += 8) {
          R x8[8], w16[16], ws16[16];
          const int cq = seg * b + q + b - j0; /* cot index of (point q, target j0) */
          ld8<R>(xr + q, x8);
          ld8<R>(ct + (cq - 8), w16);
          ld8<R>(ct + cq, w16 + 8);
          ld8<R>(cts + (cq - 8), ws16);
          ld8<R>(cts + cq, ws16 + 8);
#pragma unroll
          for (int pi = 0; pi < 4; ++pi) {
            const float2 xv = make_float2(x8[2 * pi], x8[2 * pi + 1]);
#pragma unroll
            for (int t = 0; t < 8; ++t) {
              const int m = 2 * pi - t + 8;
              const float2 wv = (t & 1) ? make_float2(ws16[m - 1], ws16[m]) : make_float2(w16[m], w16[m + 1]);
              p2[t] = ffma2(xv, wv, p2[t]);
            }
          }
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) part[t] = p2[t].x + p2[t].y;
      } else {
#pragma unroll
        for (int t = 0; t < 8; ++t) part[t] = R(0);
        for (int q = 0; q < b; q += 8) {
          R x8[8], w16[16];
          const int cq = seg * b + q + b - j0; /* cot index of (point q, target j0) */
          ld8<R>(xr + q, x8);
          ld8<R>(ct + (cq - 8), w16);
          ld8<R>(ct + cq, w16 + 8);
#pragma unroll
          for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int t = 0; t < 8; ++t) part[t] = fma(x8[i], w16[i - t + 8], part[t]);
        }
      }
#pragma unroll
      for (int t = 0; t < 8; ++t) acc[t] += part[t];
    }
    if (j0 == 0 && shifted) {
      R far = R(0), near = R(0);
      const R *pq = ps + (long)bi * tp; /* box - 1 */
      for (int k = 0; k < T; ++k) far = fma(pq[k], eh[k], far);
      for (int seg = 0; seg < 3; ++seg) { /* window box-2 .. box */
        const R *xq = xw + (long)(bi + seg) * xp;
        R part = R(0);
        for (int q = 0; q < b; ++q) part = fma(xq[q], ct[seg * b + q], part);
        near += part;
      }
      const R v = far + near;
      acc[0] = (2 * sc > P) ? v : R(0.5) * (acc[0] + v);
    }
    R *dst = u + (long)pl * M + (B0 + bi) * b + j0;
    if constexpr (sizeof(R) == 4) { /* 32-byte aligned: b and j0 are multiples of 8 */
      *reinterpret_cast<float4 *>(dst) = make_float4(acc[0], acc[1], acc[2], acc[3]);
      *reinterpret_cast<float4 *>(dst + 4) = make_float4(acc[4], acc[5], acc[6], acc[7]);
    } else {
#pragma unroll
      for (int t = 0; t < 8; ++t) dst[t] = acc[t];
    }
  }
}

/* ======================================================================== shared-memory FFT */

/* Forward DFT of 8 values in registers (split into two 4-point DFTs). */
template <typename C> __device__ __forceinline__ void dft4(C &a, C &b, C &c, C &d) {
  C t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), u = csub(b, d), t3;
  t3.x = u.y, t3.y = -u.x; /* -i (b - d) */
  a = cadd(t0, t2), b = cadd(t1, t3), c = csub(t0, t2), d = csub(t1, t3);
}
template <typename C> __device__ __forceinline__ void dft8(C *v) {
  using R = decltype(v[0].x);
  const R h = R(0.70710678118654752440084436210484904);
  dft4(v[0], v[2], v[4], v[6]);
  dft4(v[1], v[3], v[5], v[7]);
  C o1 = v[3], o2 = v[5], o3 = v[7], w;
  /* o_k * exp(-2 pi i k / 8), k = 1, 2, 3 */
  w.x = h * (o1.x + o1.y), w.y = h * (o1.y - o1.x), o1 = w;
  w.x = o2.y, w.y = -o2.x, o2 = w;
  w.x = h * (o3.y - o3.x), w.y = -h * (o3.x + o3.y), o3 = w;
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
  v[0] = cadd(e0, o0), v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1), v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2), v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3), v[7] = csub(e3, o3);
}

/* W independent forward DFTs of length L held in shared memory as buf[i*W + w].  Stockham
 * stages of radix 8 (each thread: 8 values, twiddles, an 8-point DFT in registers), after one
 * radix-2 or radix-4 stage when log2 L is not a multiple of 3; ping-pongs between buf and alt
 * and returns the buffer that holds the result.  Twiddle exp(-2 pi i t / L) = tw[t * tws]. */
template <typename C>
__device__ C *smem_fft(C *buf, C *alt, int L, int W, const C *__restrict__ tw, long tws) {
  int lg = __ffs(L) - 1, Ns = 1;
  if (lg % 3 == 1) { /* one radix-2 stage */
    const int half = L / 2;
    for (int e = threadIdx.x; e < half * W; e += blockDim.x) {
      int j = e / W, w = e - j * W;
      C v0 = buf[j * W + w], v1 = buf[(j + half) * W + w];
      alt[(2 * j) * W + w] = cadd(v0, v1);
      alt[(2 * j + 1) * W + w] = csub(v0, v1);
    }
    __syncthreads();
    C *t = buf;
    buf = alt, alt = t;
    Ns = 2;
  } else if (lg % 3 == 2) { /* one radix-4 stage */
    const int q4 = L / 4;
    for (int e = threadIdx.x; e < q4 * W; e += blockDim.x) {
      int j = e / W, w = e - j * W;
      C a = buf[j * W + w], b = buf[(j + q4) * W + w], c = buf[(j + 2 * q4) * W + w],
        d = buf[(j + 3 * q4) * W + w];
      dft4(a, b, c, d);
      alt[(4 * j) * W + w] = a;
      alt[(4 * j + 1) * W + w] = b;
      alt[(4 * j + 2) * W + w] = c;
      alt[(4 * j + 3) * W + w] = d;
    }
    __syncthreads();
    C *t = buf;
    buf = alt, alt = t;
    Ns = 4;
  }
  const int q8 = L / 8;
  for (; Ns < L; Ns *= 8) {
    for (int e = threadIdx.x; e < q8 * W; e += blockDim.x) {
      int j = e / W, w = e - j * W;
      int k = j % Ns;
      C v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = buf[(j + r * q8) * W + w];
      if (Ns > 1) {
        const long ts = (long)k * (L / (Ns * 8)) * tws;
#pragma unroll
        for (int r = 1; r < 8; ++r) v[r] = cmul(v[r], tw[r * ts]);
      }
      dft8(v);
      const int o = (j / Ns) * Ns * 8 + k;
#pragma unroll
      for (int r = 0; r < 8; ++r) alt[(o + r * Ns) * W + w] = v[r];
    }
    __syncthreads();
    C *t = buf;
    buf = alt, alt = t;
  }
  return buf;
}

/* One FFT pass over `nseq` sequences of length L:
 *   element i of sequence g (g = batch*per + w) is read from in[ibase(g) + i*istride],
 *   transformed, optionally multiplied by exp(-2 pi i * post(g) * kout / M) (4-step twiddle),
 *   and written to out[obase(g) + kout*ostride].
 * Sequences come in groups of W per block; `per` sequences per batch row (row = block of M). */
struct FftPass {
  int L, W, per;     /* per: sequences per row */
  long M;            /* row length */
  long iseq, istr;   /* input: seq stride, element stride (within a row) */
  long oseq, ostr;   /* output */
  int twiddle_post;  /* apply exp(-2 pi i * w_global * k / M) */
  long tws;          /* twiddle stride into twM for length-L DFTs: M / L */
  int conj_out;
  /* register pass only (k_fft_reg): row strides of input and output, and the post-twiddle
   * exp(-2 pi i e / T) of exponent e = (g i twmul) & twmask, T = twmask + 1, read from twP as
   * twP[e] (twbits = 0) or as twP[e & lo] * twP[lo + 1 + (e >> twbits)], lo = 2^twbits - 1 */
  long irow, orow;
  unsigned twmul, twmask;
  int twbits;
};

/* FMM-FFT passes: rows of M (or of W rows of M), post-twiddle table exp(-2 pi i t / M). */
static FftPass fmm_pass(FftPass fp) {
  fp.irow = fp.orow = fp.M;
  fp.twmul = 1, fp.twmask = (unsigned)(fp.M - 1), fp.twbits = 0;
  return fp;
}

template <typename R>
__global__ void k_fft_pass(const typename cplx<R>::T *__restrict__ in,
                           typename cplx<R>::T *__restrict__ out,
                           const typename cplx<R>::T *__restrict__ twM, FftPass fp, const OutTab ot = OutTab{}) {
  using C = typename cplx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  C *alt = buf + (long)fp.L * fp.W;
  C *twl = alt + (long)fp.L * fp.W; /* exp(-2 pi i t / L), t < L: the DFT twiddles, in shared memory */
  for (int t = threadIdx.x; t < fp.L; t += blockDim.x) twl[t] = twM[(long)t * fp.tws];
  const long row = blockIdx.y;
  const long g0 = (long)blockIdx.x * fp.W; /* first sequence of this block within the row */
  const C *src = in + row * fp.M;
  C *dst = ot.rpp ? reinterpret_cast<C *>(ot.p[row / ot.rpp]) + (row % ot.rpp) * fp.M : out + row * fp.M;
  const int LW = fp.L * fp.W;
  if (fp.istr == 1) {
    for (int e = threadIdx.x; e < LW; e += blockDim.x) {
      int i = e % fp.L, w = e / fp.L;
      buf[i * fp.W + w] = src[(g0 + w) * fp.iseq + i];
    }
  } else {
    for (int e = threadIdx.x; e < LW; e += blockDim.x) {
      int w = e % fp.W, i = e / fp.W;
      buf[i * fp.W + w] = src[(g0 + w) * fp.iseq + (long)i * fp.istr];
    }
  }
  __syncthreads();
  C *res = smem_fft<C>(buf, alt, fp.L, fp.W, twl, 1);
  if (fp.ostr == 1) {
    for (int e = threadIdx.x; e < LW; e += blockDim.x) {
      int i = e % fp.L, w = e / fp.L;
      C v = res[i * fp.W + w];
      if (fp.twiddle_post) v = cmul(v, twM[((g0 + w) * i) & (fp.M - 1)]);
      if (fp.conj_out) v.y = -v.y;
      dst[(g0 + w) * fp.oseq + i] = v;
    }
  } else {
    for (int e = threadIdx.x; e < LW; e += blockDim.x) {
      int w = e % fp.W, i = e / fp.W;
      C v = res[i * fp.W + w];
      if (fp.twiddle_post) v = cmul(v, twM[((g0 + w) * i) & (fp.M - 1)]);
      if (fp.conj_out) v.y = -v.y;
      dst[(g0 + w) * fp.oseq + (long)i * fp.ostr] = v;
    }
  }
}

/* Register-resident Stockham pass: one thread per radix-8 butterfly column (L/8 threads per
 * sequence, W sequences per block) keeps its 8 values in registers through every stage; the
 * stages exchange through ONE shared buffer laid out per sequence, element i of sequence w at
 * w*LP + fft_swz(i, kw) (pitch LP of fft_lp, an XOR swizzle within 16-element rows), which
 * keeps every exchange of both thread orders free of bank conflicts at the FMM-FFT's shapes
 * (L = 512 with W = 8; the combine's L = P with W = 32 / 16).  The first
 * stage reads global memory directly and the last stage writes it directly.  Thread order:
 * along the sequence (TIN) when the input is contiguous in i, across sequences otherwise, so
 * that a warp's loads are coalesced either way; when the output wants the other order
 * (TOUT != TIN) the result goes once through the shared buffer.  The 4-step twiddle of output
 * i = t + r L/8 of sequence g factors as exp(-2 pi i g t / M) exp(-2 pi i g (L/8) r / M): one
 * gather per thread and 8 W steps in shared memory.  Shared: fft_smem_elems(L, W) elements
 * (more for compensated twiddles); needs 16 <= L and W*L/8 <= 512; offsets within a row fit 32
 * bits (M <= 2^26). */
/* Exchange-buffer layout.  A half-warp's 16 8-byte accesses are conflict-free when they fall on
 * 16 distinct slots (element index mod 16).  Across sequences (thread order w-fastest) the
 * pitch LP = L + 16/W puts W sequences 16/W slots apart, and for W = 8 the XOR of bit 0 by
 * w bit 2 separates the pairs {c, c+8} that a radix-8 store's two threads of one sequence hit;
 * along a sequence the row swizzle h(R) = (R & 7) ^ ((R & 4) << 1) of row R = i / 16 spreads
 * the stride-8 stores 8t + r (rows t/2) and the stage-8 stores (rows R, R + 4) over both
 * halves of the row.  The swizzle permutes within each 16-element row, so indices stay in
 * [w LP, w LP + L). */
__host__ __device__ __forceinline__ int fft_lp(int L, int W) {
  return L + (W >= 16 ? 1 : W == 1 ? 0 : 16 / W);
}
__device__ __forceinline__ int fft_swz(int i, int kw) {
  const int R = i >> 4;
  return i ^ (R & 7) ^ ((R & 4) << 1) ^ kw;
}
/* Shared elements of a register pass: exchange buffer, stage twiddles (L - Ns0 <= L used, the
 * region kept at L + L/16 + 1), 4-step twiddle steps [w][9]. */
__host__ __device__ __forceinline__ size_t fft_smem_elems(int L, int W) {
  return (size_t)W * fft_lp(L, W) + L + L / 16 + 1 + 9 * (size_t)W;
}

/* Input of a register pass: element t + r q (r < 8) of sequence g of row `row` into v[r]. */
template <typename R> struct StridedLd { /* in + row irow + g iseq + i istr */
  const typename cplx<R>::T *__restrict__ in;
  long irow, iseq;
  unsigned istr;
  __device__ __forceinline__ void operator()(long row, unsigned g, int t, int q,
                                             typename cplx<R>::T (&v)[8]) const {
    const typename cplx<R>::T *sp = in + row * irow + g * iseq + t * istr;
    const unsigned qs = (unsigned)q * istr;
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = sp[r * qs];
  }
};

/* The combine's input: element sc of column m is x_0[m] for sc = 0, else
 * c_sc (u_sc[m] - i S_sc / M) from the planar far+near field u (re, im planes per section). */
template <typename R> struct CombineLd {
  const R *__restrict__ xt, *__restrict__ u;
  const typename cplx<R>::T *__restrict__ ssum, *__restrict__ pretw;
  long M;
  R invM;
  int P;
  const typename cplx<R>::T *__restrict__ pretw_lo; /* compensated pre-twiddle (FP32), or null */
  long m0; /* first column (a shard's own columns of its strip) */
  /* row = transform of a batch: its sections, fields and section sums */
  __device__ __forceinline__ void operator()(long row, unsigned mc, int t, int q,
                                             typename cplx<R>::T (&v)[8]) const {
    const long m = m0 + mc;
    const R *xt = this->xt + row * 2 * P * M, *u = this->u + row * 2 * (P - 1) * M;
    const typename cplx<R>::T *ssum = this->ssum + row * P;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int sc = t + r * q;
      if (sc == 0) {
        v[r].x = xt[m], v[r].y = xt[M + m];
      } else {
        const typename cplx<R>::T S = ssum[sc];
        typename cplx<R>::T a;
        a.x = u[(2L * (sc - 1)) * M + m] + S.y * invM;
        a.y = u[(2L * (sc - 1) + 1) * M + m] - S.x * invM;
        if constexpr (sizeof(R) == 4) {
          if (pretw_lo) {
            v[r] = cmul_comp(a, pretw[sc], pretw_lo[sc]);
            continue;
          }
        }
        v[r] = cmul(pretw[sc], a);
      }
    }
  }
};

/* COMP (FP32): compensated twiddles.  twD_lo / twP_lo hold the FP32 rounding of each table
 * entry's remainder; the stage twiddles are applied with cmul_comp from a second shared table,
 * and the 4-step post-twiddle of output i of sequence g is read directly as twP[(g i) mod T]
 * (hi and lo; single-level tables, twbits = 0) instead of as a product of two rounded factors.
 * Shared memory: L + L/16 + 1 more elements.
 * LGT != 0: a build for L = 2^LGT only (fp.L must equal it), so that the stage loop unrolls and
 * every exchange index is folded at compile time; LGT = 0 serves any L. */
template <typename R, bool TIN, bool TOUT, class Ld = StridedLd<R>, bool COMP = false, int LGT = 0>
__global__ void __launch_bounds__(512, sizeof(R) == 4 ? 3 : 1)
    k_fft_reg(const Ld ld, typename cplx<R>::T *__restrict__ out,
              const typename cplx<R>::T *__restrict__ twD, const typename cplx<R>::T *__restrict__ twP,
              FftPass fp, const typename cplx<R>::T *__restrict__ twD_lo = nullptr,
              const typename cplx<R>::T *__restrict__ twP_lo = nullptr, const OutTab ot = OutTab{}) {
  using C = typename cplx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = LGT ? 1 << LGT : fp.L, W = fp.W, q = L >> 3;
  const int lq = LGT ? LGT - 3 : __ffs(q) - 1, lW = __ffs(W) - 1;
  const int LP = fft_lp(L, W);
  C *buf = reinterpret_cast<C *>(smem_raw);
  /* stage twiddles, stage-major: for the stage of span Ns (Ns0, 8 Ns0, ..., L/8; Ns0 the first
   * stage's radix), exp(-2 pi i r k / (8 Ns)) at (Ns - Ns0) + 7 k + r - 1 (k < Ns, 1 <= r < 8):
   * a thread's 7 twiddles are consecutive and a half-warp's threads 7 apart */
  C *twl = buf + W * LP;
  C *twq = twl + L + L / 16 + 1; /* 4-step twiddle steps exp(-2 pi i g q r / M), [w][9] */
  C *twl_lo = twq + 9 * W;       /* COMP: the remainders of twl */
  const int tid = threadIdx.x;
  const unsigned g0 = blockIdx.x * (unsigned)W;
  /* post-twiddle exp(-2 pi i e / T) for e = g * i */
  auto post = [&](unsigned gi) -> C {
    const unsigned e = (gi * fp.twmul) & fp.twmask;
    if (fp.twbits == 0) return twP[e];
    const unsigned lo = (1u << fp.twbits) - 1;
    return cmul(twP[lo + 1 + (e >> fp.twbits)], twP[e & lo]);
  };
  const int lg = LGT ? LGT : __ffs(L) - 1;
  const int ns0 = lg % 3 == 0 ? 8 : lg % 3 == 2 ? 4 : 2;
  for (int Ns = ns0; Ns <= q; Ns <<= 3)
    for (int m = tid; m < 7 * Ns; m += blockDim.x) {
      const int k = m / 7, r = m - 7 * k + 1;
      const long e = (long)(r * k * (q / Ns)) * fp.tws; /* r k L / (8 Ns) of L */
      twl[Ns - ns0 + m] = twD[e];
      if constexpr (COMP) twl_lo[Ns - ns0 + m] = twD_lo[e];
    }
  if (fp.twiddle_post && !COMP)
    for (int m = tid; m < 8 * W; m += blockDim.x)
      twq[(m >> 3) * 9 + (m & 7)] = post((g0 + (m >> 3)) * (unsigned)q * (unsigned)(m & 7));
  /* COMP: x times exp(-2 pi i e / T), e = g i twmul mod T, from the hi / lo tables */
  auto post_comp = [&](C x, unsigned gi) -> C {
    if constexpr (COMP) {
      const unsigned e = (gi * fp.twmul) & fp.twmask;
      return cmul_comp(x, twP[e], twP_lo[e]);
    } else {
      return x;
    }
  };
  int t, w;
  if (TIN) t = tid & (q - 1), w = tid >> lq;
  else w = tid & (W - 1), t = tid >> lW;
  const unsigned ostr = (unsigned)fp.ostr;
  const long row = blockIdx.y;
  C v[8];
  ld(row, g0 + w, t, q, v);
  C *bw = buf + w * LP;
  const int kw = W == 8 ? (w >> 2) & 1 : 0;
  int Ns, lNs;
  if (lg % 3 == 0) { /* radix-8 first stage: outputs 8t + r */
    dft8(v);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      bw[fft_swz(8 * t + r, kw)] = v[r];
    }
    Ns = 8, lNs = 3;
  } else if (lg % 3 == 2) { /* radix 4: butterflies t (v0,2,4,6) and t+q (v1,3,5,7) */
    dft4(v[0], v[2], v[4], v[6]);
    dft4(v[1], v[3], v[5], v[7]);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      bw[fft_swz(4 * t + r, kw)] = v[2 * r];
      bw[fft_swz(4 * (t + q) + r, kw)] = v[2 * r + 1];
    }
    Ns = 4, lNs = 2;
  } else { /* radix 2: butterflies t + m q, inputs v[m], v[m+4] */
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int i = 2 * (t + m * q);
      bw[fft_swz(i, kw)] = cadd(v[m], v[m + 4]);
      bw[fft_swz(i + 1, kw)] = csub(v[m], v[m + 4]);
    }
    Ns = 2, lNs = 1;
  }
  /* the stages after the first; their count is a constant in an L-specific build */
  const int nst = LGT ? (LGT - (LGT % 3 == 0 ? 3 : LGT % 3)) / 3 : (lg - lNs) / 3;
#pragma unroll
  for (int si = 0; si < nst; ++si) {
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = bw[fft_swz(t + r * q, kw)];
    const int k = t & (Ns - 1);
    const int tb = Ns - ns0 + 7 * k - 1;
#pragma unroll
    for (int r = 1; r < 8; ++r) {
      if constexpr (COMP)
        v[r] = cmul_comp(v[r], twl[tb + r], twl_lo[tb + r]);
      else
        v[r] = cmul(v[r], twl[tb + r]);
    }
    dft8(v);
    if (si == nst - 1) break; /* v[r] = output t + r q */
    __syncthreads();
    const int o = ((t >> lNs) << (lNs + 3)) + k;
#pragma unroll
    for (int r = 0; r < 8; ++r) bw[fft_swz(o + (r << lNs), kw)] = v[r];
    Ns <<= 3, lNs += 3;
  }
  C *dp = ot.rpp ? reinterpret_cast<C *>(ot.p[row / ot.rpp]) + (row % ot.rpp) * fp.orow : out + row * fp.orow;
  if (TOUT == TIN) {
    const unsigned g = g0 + w;
    C *op = dp + g * fp.oseq + t * ostr;
    const unsigned qs = (unsigned)q * ostr;
    C a;
    if (fp.twiddle_post && !COMP) a = post(g * (unsigned)t);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      C x = v[r];
      if (fp.twiddle_post) {
        if constexpr (COMP)
          x = post_comp(x, g * (unsigned)(t + r * q));
        else
          x = cmul(x, cmul(a, twq[w * 9 + r]));
      }
      if (fp.conj_out) x.y = -x.y;
      op[r * qs] = x;
    }
  } else {
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; ++r) bw[fft_swz(t + r * q, kw)] = v[r];
    __syncthreads();
    int t2, w2;
    if (TOUT) t2 = tid & (q - 1), w2 = tid >> lq;
    else w2 = tid & (W - 1), t2 = tid >> lW;
    const unsigned g = g0 + w2;
    const C *b2 = buf + w2 * LP;
    const int kw2 = W == 8 ? (w2 >> 2) & 1 : 0;
    C *op = dp + g * fp.oseq + t2 * ostr;
    const unsigned qs = (unsigned)q * ostr;
    C a;
    if (fp.twiddle_post && !COMP) a = post(g * (unsigned)t2);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = t2 + r * q;
      C x = b2[fft_swz(i, kw2)];
      if (fp.twiddle_post) {
        if constexpr (COMP)
          x = post_comp(x, g * (unsigned)i);
        else
          x = cmul(x, cmul(a, twq[w2 * 9 + r]));
      }
      if (fp.conj_out) x.y = -x.y;
      op[r * qs] = x;
    }
  }
}

/* Launch one FFT pass: the register kernel when the shape allows it, else the shared-memory
 * pass.  per = sequences per row; W_old = sequences per block of the shared-memory pass. */
template <typename R>
static void launch_fft_pass(const typename cplx<R>::T *in, typename cplx<R>::T *out,
                            const typename cplx<R>::T *twM, FftPass fp, long per, long rows,
                            int W_old, int reg_threads, cudaStream_t st,
                            const typename cplx<R>::T *twM_lo = nullptr, const OutTab *ot = nullptr) {
  using C = typename cplx<R>::T;
  const OutTab O = ot ? *ot : OutTab{}; /* the last pass of a pointer-table execute */
  const int L = fp.L;
  const bool tin = fp.istr == 1, tout = fp.ostr == 1;
  if (L >= 16 && L <= 8 * reg_threads && !(tout && !tin)) {
    int W = reg_threads / (L / 8);
    if (W > 16) W = 16;
    if (W > per) W = (int)per;
    if (W < 1) W = 1;
    if (tin || W >= 4) {
      fp.W = W;
      const StridedLd<R> sld{in, fp.M, fp.iseq, (unsigned)fp.istr};
      const int thr = W * (L / 8);
      const size_t sm = sizeof(C) * fft_smem_elems(L, W);
      dim3 g((unsigned)(per / W), (unsigned)rows);
      if constexpr (sizeof(R) == 4) {
        if (twM_lo) { /* compensated twiddles */
          const size_t smc = sm + sizeof(C) * (size_t)(L + L / 16 + 1);
          if (tin && tout)
            k_fft_reg<R, true, true, StridedLd<R>, true><<<g, thr, smc, st>>>(sld, out, twM, twM, fmm_pass(fp),
                                                                              twM_lo, twM_lo, O);
          else if (tin)
            k_fft_reg<R, true, false, StridedLd<R>, true><<<g, thr, smc, st>>>(sld, out, twM, twM, fmm_pass(fp),
                                                                               twM_lo, twM_lo, O);
          else
            k_fft_reg<R, false, false, StridedLd<R>, true><<<g, thr, smc, st>>>(sld, out, twM, twM, fmm_pass(fp),
                                                                                twM_lo, twM_lo, O);
          return;
        }
      }
      if (L == 512) { /* the size-2^18 FFTs' two passes: a build for L = 512 */
        if (tin && tout)
          k_fft_reg<R, true, true, StridedLd<R>, false, 9><<<g, thr, sm, st>>>(sld, out, twM, twM, fmm_pass(fp),
                                                                               nullptr, nullptr, O);
        else if (tin)
          k_fft_reg<R, true, false, StridedLd<R>, false, 9><<<g, thr, sm, st>>>(sld, out, twM, twM, fmm_pass(fp),
                                                                                nullptr, nullptr, O);
        else
          k_fft_reg<R, false, false, StridedLd<R>, false, 9><<<g, thr, sm, st>>>(sld, out, twM, twM, fmm_pass(fp),
                                                                                 nullptr, nullptr, O);
        return;
      }
      if (tin && tout)
        k_fft_reg<R, true, true><<<g, thr, sm, st>>>(sld, out, twM, twM, fmm_pass(fp), nullptr, nullptr, O);
      else if (tin)
        k_fft_reg<R, true, false><<<g, thr, sm, st>>>(sld, out, twM, twM, fmm_pass(fp), nullptr, nullptr, O);
      else
        k_fft_reg<R, false, false><<<g, thr, sm, st>>>(sld, out, twM, twM, fmm_pass(fp), nullptr, nullptr, O);
      return;
    }
  }
  fp.W = W_old;
  dim3 g((unsigned)(per / W_old), (unsigned)rows);
  k_fft_pass<R><<<g, 256, sizeof(C) * (size_t)L * (2 * W_old + 1), st>>>(in, out, twM, fp, O);
}

/* ======================================================================== combine */

/* For TMc points m and every section: w_0 = x_0[m], w_sc = c_sc (u_sc[m] - (i/M) Ssum_sc),
 * z_r[m] = sum_sc exp(-2 pi i sc r / P) w_sc[m] (a length-P DFT), written to z[r][m]. */
template <typename R>
__global__ void k_combine(const R *__restrict__ xt, const R *__restrict__ u,
                          const typename cplx<R>::T *__restrict__ ssum,
                          const typename cplx<R>::T *__restrict__ pretw,
                          const typename cplx<R>::T *__restrict__ twP,
                          typename cplx<R>::T *__restrict__ z, long M, int P, int TMc) {
  using C = typename cplx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw); /* [P][TMc] */
  C *alt = buf + (long)P * TMc;
  const long m0 = (long)blockIdx.x * TMc;
  const R invM = R(1) / R(M);
  { /* transform blockIdx.y of a batch */
    const long tr = blockIdx.y;
    xt += tr * 2 * P * M, u += tr * 2 * (P - 1) * M, ssum += tr * P, z += tr * P * M;
  }
  for (int e = threadIdx.x; e < P * TMc; e += blockDim.x) {
    int mm = e % TMc, sc = e / TMc;
    C w;
    if (sc == 0) {
      w.x = xt[m0 + mm];
      w.y = xt[M + m0 + mm];
    } else {
      C v;
      C S = ssum[sc];
      v.x = u[(2L * (sc - 1)) * M + m0 + mm] + S.y * invM; /* u - i S / M */
      v.y = u[(2L * (sc - 1) + 1) * M + m0 + mm] - S.x * invM;
      w = cmul(pretw[sc], v);
    }
    buf[sc * TMc + mm] = w;
  }
  __syncthreads();
  C *res = smem_fft<C>(buf, alt, P, TMc, twP, 1);
  for (int e = threadIdx.x; e < P * TMc; e += blockDim.x) {
    int mm = e % TMc, r = e / TMc;
    z[(long)r * M + m0 + mm] = res[r * TMc + mm];
  }
}

/* Bin 0 of every output block, y[r M], equals sum_n x[n] exp(-2 pi i n r / P), i.e. the
 * length-P DFT of the section sums that stage 2 already holds.  Through the FMM that bin is
 * reached via the cot kernel's zero-frequency eigenvalue -cot(pi sc / P) (about 20 for
 * sc = 1, P = 64), which the pre-twiddle c_sc then cancels; in FP32 the amplified rounding
 * makes these P bins the least accurate of the transform.  FP32 plans with >= 10 terms
 * therefore evaluate them from this identity, in FP64. */
template <typename R>
__global__ void k_block_dc(const typename cplx<R>::T *__restrict__ ssum,
                           typename cplx<R>::T *__restrict__ y, long M, int P, int conj_out,
                           const OutTab yt, int r0 = 0, int nrows = 0) {
  /* one warp per output bin r; lane l sums sc = l, l + 32, ...; FP64 warp reduction.  A shard of
   * a sharded transform writes its own rows: bins r0 .. r0 + nrows - 1 at y + (r - r0) M. */
  using C = typename cplx<R>::T;
  const int rl = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (rl >= (nrows ? nrows : P)) return;
  const int r = r0 + rl;
  ssum += (long)blockIdx.y * P; /* transform of a batch */
  y = yt.rpp ? reinterpret_cast<typename cplx<R>::T *>(yt.p[blockIdx.y]) : y + (long)blockIdx.y * P * M;
  double re = 0, im = 0;
  for (int sc = lane; sc < P; sc += 32) {
    double sn, cs;
    sincospi(-2.0 * (double)((long)sc * r % P) / (double)P, &sn, &cs);
    C v = ssum[sc];
    re += (double)v.x * cs - (double)v.y * sn;
    im += (double)v.x * sn + (double)v.y * cs;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if (lane == 0) {
    C out;
    out.x = (R)re;
    out.y = (R)(conj_out ? -im : im);
    y[(long)rl * M] = out;
  }
}

/* ======================================================================== coarse tree */

/* The coarse levels of the tree (few boxes: every level whose row count per transform is below
 * a threshold, at most 2^kCoarseMaxLevel boxes per plane) in one launch instead of one launch per
 * level: the upward M2M for parent levels Lm .. 2, the top flip, and the downward M2L + L2L for
 * child levels 3 .. Ll.  Every expansion plane (section, re/im, transform) is independent of the
 * others at every level (its neighbours wrap within the plane), so one block takes one plane
 * through all of these levels.  The plane's coarse levels stay in shared memory: phi of the
 * levels above Lm (made by the per-level kernels) is read from global memory once, every level
 * computed here is kept in shared memory for the levels after it and written to global memory
 * once (the per-level kernels after this one and the debug views read it there), so a level
 * costs one block barrier and no global round trip.  The levels' operators are copied with
 * cp.async into two alternating buffers, the next level's while the current one computes (one
 * buffer, copied after the barrier, when two do not fit).  Same operators, layouts and outputs
 * as the per-level launches (reference fmmfft.c:476-515 upward, :620-749 top and downward).
 * Compute: one warp per output row, lane = output column (N / 32 columns per lane); the K sum
 * accumulates per 32-column block, then into the total (two-level FP32 accumulation, as in the
 * row kernels).  Launched as a programmatic dependent launch: the first operator is staged
 * before the wait for the kernel that made its input. */
template <typename R> struct CoarseArgs {
  R *phi, *psi;
  const R *bm2m, *btop, *bm2l;
  long S1; /* planes / 2, all transforms of the execute */
  int T, Lm, Ll; /* coarse M2M parent levels Lm..2 (none when Lm < 2); M2L child levels 3..Ll */
  int dbuf;      /* two operator buffers */
};
constexpr int kCoarseMaxLevel = 6; /* coarse M2M parents hold at most 2^6 boxes per plane */
constexpr int kCoarseWarps = 32;   /* a block: one warp per row */
constexpr int kCoarseTop = kCoarseMaxLevel + 1; /* highest level a block holds (M2M input, M2L) */

__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

/* Issue the copy of a level's operator B (K x N, row-major) into the shared array Bs with
 * cp.async, in 16-byte pieces where the size and address allow, else one element per copy;
 * nothing waits here. */
template <typename R>
__device__ __forceinline__ void coarse_stage_b(int K, int N, const R *__restrict__ B, R *__restrict__ Bs) {
  const int n = K * N;
  const uint32_t sb = (uint32_t)__cvta_generic_to_shared(Bs);
  if (((size_t)n * sizeof(R)) % 16 == 0 && ((uintptr_t)B & 15) == 0 && (sb & 15) == 0) {
    constexpr int per = 16 / sizeof(R);
    for (int e = threadIdx.x * per; e < n; e += blockDim.x * per)
      tc::cp_async16(sb + (uint32_t)(e * sizeof(R)), B + e);
  } else {
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      if constexpr (sizeof(R) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" : : "r"(sb + (uint32_t)(e * 8)), "l"(B + e) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" : : "r"(sb + (uint32_t)(e * 4)), "l"(B + e) : "memory");
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

/* Floats (elements) of a plane's levels 2..L: (2^(L+1) - 4) rows of T. */
__host__ __device__ constexpr long coarse_lvl_rows(int L) { return (2L << L) - 4; }

/* Shared memory of the coarse kernel: one or two operator buffers (the largest operator, the
 * M2L one, 5T x 2T), the plane's phi and psi levels 2..kCoarseTop and the split-K partial sums
 * (at most 32 rows x parts of 2T). */
template <typename R> static size_t coarse_smem(long T, int dbuf) {
  return sizeof(R) * ((dbuf ? 20 : 10) * (size_t)T * T + 2 * (size_t)coarse_lvl_rows(kCoarseTop) * T +
                      (size_t)kCoarseWarps * 4 * T);
}

/* Rows [0, rows) of one level: out[r][n] = sum_k A(r, k) Bs[k][n].  Row r's A is up to three
 * contiguous pieces of shared memory, segs(r, p, o) filling piece pointers p[] and their first K
 * index o[] (o[0] = 0, pieces in K order, o[3] = K).  A level with fewer rows than warps splits
 * each row's K range over S = warps / rows warps (S <= 8); their partial sums go to `red` and are
 * added in a fixed order (so a plane's bits do not depend on anything else).  Lane = output
 * column (NJ columns per lane, N <= 32 NJ).  Outputs go to the shared level Os and to global
 * memory Og.  Ends with the outputs written by the threads that wrote them (the caller's next
 * barrier publishes them). */
template <typename R, int NJ, class Segs>
__device__ __forceinline__ void coarse_level(int rows, int K, int N, const R *__restrict__ Bs, R *__restrict__ Os,
                                             R *__restrict__ Og, R *__restrict__ red, Segs segs) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int S = kCoarseWarps / rows;
  S = S < 1 ? 1 : (S > 8 ? 8 : S);
  const int kper = (K + S - 1) / S;
  for (int it = warp; it < rows * S; it += kCoarseWarps) {
    const int r = it / S, part = it - r * S;
    const int k0 = part * kper, k1 = k0 + kper < K ? k0 + kper : K;
    const R *pc[3];
    int o[4];
    segs(r, pc, o);
    R acc[NJ];
#pragma unroll
    for (int j = 0; j < NJ; ++j) acc[j] = R(0);
    for (int q = 0; q < 3; ++q) {
      const int lo = k0 > o[q] ? k0 : o[q], hi = k1 < o[q + 1] ? k1 : o[q + 1];
      const R *ap = pc[q];
#pragma unroll 4
      for (int k = lo; k < hi; ++k) {
        const R av = ap[k - o[q]];
        const R *bk = Bs + k * N + lane;
#pragma unroll
        for (int j = 0; j < NJ; ++j)
          if (NJ == 1 || lane + 32 * j < N) acc[j] = fma(av, bk[32 * j], acc[j]);
      }
    }
    if (S == 1) {
#pragma unroll
      for (int j = 0; j < NJ; ++j)
        if (lane + 32 * j < N) Os[r * N + lane + 32 * j] = acc[j], Og[r * N + lane + 32 * j] = acc[j];
    } else {
#pragma unroll
      for (int j = 0; j < NJ; ++j)
        if (lane + 32 * j < N) red[it * N + lane + 32 * j] = acc[j];
    }
  }
  if (S > 1) {
    __syncthreads();
    for (int e = threadIdx.x; e < rows * N; e += blockDim.x) {
      const int r = e / N, c = e - r * N;
      R v = red[(r * S) * N + c];
      for (int part = 1; part < S; ++part) v += red[(r * S + part) * N + c];
      Os[e] = v;
      Og[e] = v;
    }
  }
}

/* the same with the lane's column count chosen from N */
template <typename R, class Segs>
__device__ __forceinline__ void coarse_level_n(int rows, int K, int N, const R *Bs, R *Os, R *Og, R *red, Segs segs) {
  if (N <= 32) coarse_level<R, 1>(rows, K, N, Bs, Os, Og, red, segs);
  else if (N <= 64) coarse_level<R, 2>(rows, K, N, Bs, Os, Og, red, segs);
  else coarse_level<R, 4>(rows, K, N, Bs, Os, Og, red, segs);
}

template <typename R> __global__ void __launch_bounds__(32 * kCoarseWarps) k_coarse(CoarseArgs<R> a) {
  extern __shared__ __align__(16) unsigned char coarse_raw[];
  const int T = a.T;
  R *Bs[2];
  Bs[0] = reinterpret_cast<R *>(coarse_raw);
  Bs[1] = a.dbuf ? Bs[0] + 10L * T * T : Bs[0];
  R *Ph = Bs[0] + (a.dbuf ? 20L : 10L) * T * T; /* phi levels 2..kCoarseTop of this plane */
  R *Ps = Ph + coarse_lvl_rows(kCoarseTop) * T; /* psi levels 2..kCoarseTop */
  R *red = Ps + coarse_lvl_rows(kCoarseTop) * T; /* split-K partial sums: 32 x 4T */
  const long S1 = a.S1, pl = blockIdx.x;
  /* level l of this block's plane, in global and in shared memory */
  auto lv = [&](R *base, int l) { return base + lvl_off(l, S1, T) + pl * (1L << l) * T; };
  auto sl = [&](R *base, int l) { return base + ((1L << l) - 4) * T; };
  /* the levels in order: M2M parents Lm..2, the top flip, M2L children 3..Ll */
  const int nm = a.Lm >= 2 ? a.Lm - 1 : 0, nlev = nm + 1 + (a.Ll >= 3 ? a.Ll - 2 : 0);
  auto stage_op = [&](int i, R *dst) {
    if (i < nm) coarse_stage_b<R>(2 * T, T, a.bm2m + (long)(a.Lm - i - 2) * 2 * T * T, dst);
    else if (i == nm) coarse_stage_b<R>(T, T, a.btop, dst);
    else coarse_stage_b<R>(5 * T, 2 * T, a.bm2l + (long)(i - nm - 1) * 10 * T * T, dst);
  };
  tc::pdl_trigger();
  stage_op(0, Bs[0]); /* a plan constant */
  tc::pdl_wait();
  { /* phi of the levels this block does not make: Lm+1 .. Ltop (only Lm+1 when the M2M runs
     * here; the top flip and M2L read levels 2..Ll) */
    const int lo = a.Lm >= 2 ? a.Lm + 1 : 2;
    const int hi = a.Ll > lo ? a.Ll : lo;
    for (int l = lo; l <= hi; ++l) {
      const R *g = lv(a.phi, l);
      R *d = sl(Ph, l);
      const int n = (1 << l) * T;
      for (int e = threadIdx.x; e < n; e += blockDim.x) d[e] = g[e];
    }
  }
  for (int i = 0; i < nlev; ++i) {
    R *B = Bs[i & 1];
    if (a.dbuf) {
      cp_async_wait0(); /* this thread's copies of level i's operator */
      __syncthreads();  /* everyone's; the level before is written and done with the other buffer */
      if (i + 1 < nlev) stage_op(i + 1, Bs[(i + 1) & 1]);
    } else {
      if (i > 0) {
        __syncthreads(); /* the level before is done with the buffer */
        stage_op(i, B);
      }
      cp_async_wait0();
      __syncthreads();
    }
    if (i < nm) { /* M2M: parent level L from child pairs of L + 1 */
      const int L = a.Lm - i;
      const R *child = sl(Ph, L + 1);
      coarse_level_n<R>(1 << L, 2 * T, T, B, sl(Ph, L), lv(a.phi, L), red, [=](int r, const R **p, int *o) {
        p[0] = child + r * 2 * T, p[1] = p[2] = p[0];
        o[0] = 0, o[1] = o[2] = o[3] = 2 * T;
      });
    } else if (i == nm) { /* top flip: psi_2[c] = topflp . phi_2[(c + 2) mod 4] */
      const R *phi2 = sl(Ph, 2);
      coarse_level_n<R>(4, T, T, B, sl(Ps, 2), lv(a.psi, 2), red, [=](int r, const R **p, int *o) {
        p[0] = phi2 + ((r + 2) & 3) * T, p[1] = p[2] = p[0];
        o[0] = 0, o[1] = o[2] = o[3] = T;
      });
    } else { /* M2L + L2L: child level l, one row per parent box: psi of the parent, then the
              * child pairs 2r-2, 2r-1 and 2r+2, 2r+3 (wrapping; a pair never straddles the end) */
      const int l = i - nm + 2;
      const R *psi_par = sl(Ps, l - 1), *phi = sl(Ph, l);
      const int mask = (1 << l) - 1;
      coarse_level_n<R>(1 << (l - 1), 5 * T, 2 * T, B, sl(Ps, l), lv(a.psi, l), red,
                        [=](int r, const R **p, int *o) {
                          p[0] = psi_par + r * T;
                          p[1] = phi + ((2 * r - 2) & mask) * T;
                          p[2] = phi + ((2 * r + 2) & mask) * T;
                          o[0] = 0, o[1] = T, o[2] = 3 * T, o[3] = 5 * T;
                        });
    }
  }
  cp_async_wait0();
}

/* Self-test of the bounded device waits: the same wait routine as the tensor-core kernels
 * (tc::t_wait on an mbarrier, with tensor memory held), made to wait for an event that never
 * comes (an mbarrier nobody arrives on) with a short limit.  The wait gives up, records the error
 * in `status`, the tensor memory is freed and the kernel returns: the host then sees
 * FMMFFT_ERR_TIMEOUT and the context stays usable. */
__global__ void __launch_bounds__(64) k_selftest_wait(unsigned long long limit_ns, int *status) {
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  {
    if (threadIdx.x < 32) tc::tmem_alloc(&tmem_slot, 32);
    if (threadIdx.x == 0) {
      tc::mbar_init(&bar, 1);
      tc::fence_mbar_init();
      abort_flag = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (threadIdx.x == 0) tc::t_wait(&bar, 0, &abort_flag, status, limit_ns);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (threadIdx.x < 32) tc::tmem_dealloc(tmem_slot, 32);
  }
}

/* ======================================================================== host orchestration */

template <typename R> static int upload(R **dst, const double *src, size_t n, char *err, size_t errlen) {
  R *h = (R *)malloc(sizeof(R) * (n ? n : 1));
  if (!h) return 2;
  for (size_t i = 0; i < n; ++i) h[i] = (R)src[i];
  cudaError_t e = cudaMemcpy(*dst, h, sizeof(R) * n, cudaMemcpyHostToDevice);
  free(h);
  if (e != cudaSuccess) {
    snprintf(err, errlen, "cudaMemcpy: %s", cudaGetErrorString(e));
    return 3;
  }
  return 0;
}

static inline size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

/* The FP32 remainders of FP64 values, v - (float)v rounded to FP32, into dst (device). */
template <typename P_> static int upload_lo(P_ *dst, const double *src, size_t n, char *err, size_t errlen) {
  float *h = (float *)malloc(sizeof(float) * (n ? n : 1));
  if (!h) return 2;
  for (size_t i = 0; i < n; ++i) h[i] = (float)(src[i] - (double)(float)src[i]);
  cudaError_t e = cudaMemcpy(dst, h, sizeof(float) * n, cudaMemcpyHostToDevice);
  free(h);
  if (e != cudaSuccess) {
    snprintf(err, errlen, "cudaMemcpy: %s", cudaGetErrorString(e));
    return 3;
  }
  return 0;
}
static inline long pow2_floor(long v) {
  long p = 1;
  while (p * 2 <= v) p *= 2;
  return p;
}

/* Round to TF32 (nearest, ties away from zero), as cvt.rna.tf32.f32 does. */
static float tf32_rna_host(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) {
    u += 0x1000u;
    u &= 0xffffe000u;
  }
  float r;
  memcpy(&r, &u, 4);
  return r;
}

/* FP32 -> BF16 bits, round to nearest even (finite values): the upper 16 bits after adding half a
 * BF16 unit minus one plus the lowest kept bit; and BF16 bits -> FP32. */
static uint16_t bf16_rne_host(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
static float bf16_to_float_host(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

/* Uploads one operator, given as FP64 [npad][kpad] K-major values, split into TF32 hi and lo:
 * as two [npad][kpad] arrays (dhi, dlo) and, when dws is given, as the warp-specialised
 * kernel's block (hi rows 0..npad-1, lo rows npad..2 npad-1, core-matrix layout). */
/* Splits operator v ([npad][kpad], row n = output column n, zero padded) into TF32 hi / lo and
 * uploads the images the kernels copy into shared memory as they are:
 *   dimg   the row forms' (k_tc_rowgemm, k_tc_nbr): hi rows then lo rows, K-major core
 *          matrices with K extent kpad (element (n, k) at byte core_off(n, k, kpad)); 2 kpad npad;
 *   dimg16 the 16-lane form's (k_tc_rowgemm16): the same with K extent kp16 = round16(kpad) and
 *          element (n, k) holding v(perm16(n), perm16(k)), zero for perm16(k) >= kpad; 2 kp16 npad;
 *   dws    the warp-specialised form's (ws_b_index layout; BF16 hi / lo for BF16x3 plans).
 * Null images are skipped. */
static int tc_put(float *dimg, float *dimg16, float *dws, const double *v, int kpad, int npad, char *err,
                  size_t errlen, int bf16 = 0) {
  const long cnt = (long)kpad * npad;
  const int kp16 = tc::round16(kpad);
  const long cnt16 = (long)kp16 * npad;
  const size_t wsn = tc::ws_b_floats(kpad, npad);
  float *h = (float *)calloc((size_t)4 * cnt + 2 * cnt16 + wsn + 1, sizeof(float));
  if (!h) return 2;
  float *img = h + 2 * cnt, *img16 = img + 2 * cnt, *w = img16 + 2 * cnt16;
  uint16_t *wb = (uint16_t *)w; /* BF16 block: wsn 16-bit values */
  for (long i = 0; i < cnt; ++i) {
    float f = (float)v[i];
    float hi = tf32_rna_host(f);
    h[i] = hi;
    h[cnt + i] = tf32_rna_host(f - hi);
    const int n = (int)(i / kpad), k = (int)(i % kpad);
    const long o = (long)(tc::core_off(n, k, kpad) >> 2);
    img[o] = h[i];
    img[cnt + o] = h[cnt + i];
    if (bf16) {
      const uint16_t bh = bf16_rne_host(f);
      const float fh = bf16_to_float_host(bh);
      wb[tc::ws_b_index_bf16(n, k, kpad)] = bh;
      wb[tc::ws_b_index_bf16(npad + n, k, kpad)] = bf16_rne_host(f - fh);
    } else {
      w[tc::ws_b_index(n, k, kpad)] = h[i];
      w[tc::ws_b_index(npad + n, k, kpad)] = h[cnt + i];
    }
  }
  for (int n = 0; n < npad; ++n)
    for (int k = 0; k < kp16; ++k) {
      const int ks = tc::perm16(k);
      const long o = (long)(tc::core_off(n, k, kp16) >> 2), src = (long)tc::perm16(n) * kpad + ks;
      img16[o] = ks < kpad ? h[src] : 0.f;
      img16[cnt16 + o] = ks < kpad ? h[cnt + src] : 0.f;
    }
  cudaError_t e = cudaSuccess;
  if (dimg) e = cudaMemcpy(dimg, img, sizeof(float) * 2 * cnt, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && dimg16) e = cudaMemcpy(dimg16, img16, sizeof(float) * 2 * cnt16, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && dws)
    e = cudaMemcpy(dws, w, (bf16 ? 2 : 4) * wsn, cudaMemcpyHostToDevice);
  free(h);
  if (e != cudaSuccess) {
    snprintf(err, errlen, "cudaMemcpy: %s", cudaGetErrorString(e));
    return 3;
  }
  return 0;
}

/* B operands of the tensor-core stages, K-major: B[n][k] multiplies A column k into output n. */
template <typename R> static int tc_upload_ops(Dev<R> *d, const fmm_ops64 *o, char *err, size_t errlen) {
  const long T = o->T, b = o->b, P = o->P, n = o->n, S1 = P - 1;
  long cap = (long)d->kp_s2m * d->np_s2m;
  if (d->tc_m2m_stride > cap) cap = d->tc_m2m_stride;
  if (d->tc_m2l_stride > cap) cap = d->tc_m2l_stride;
  if (d->tc_leaf_stride > cap) cap = d->tc_leaf_stride;
  if (d->tc_lnb_stride > cap) cap = d->tc_lnb_stride;
  double *v = (double *)malloc(sizeof(double) * cap);
  if (!v) return 2;
  int rc = 0;
  if (d->ok_s2m) {
    const int kp = d->kp_s2m, np = d->np_s2m;
    for (long i = 0; i < (long)kp * np; ++i) v[i] = 0;
    for (long nn = 0; nn < T; ++nn)
      for (long k = 0; k < b; ++k) v[nn * kp + k] = o->initch[k * T + nn];
    rc |= tc_put(d->tc_s2m[0], d->tc_s2m[1], d->ws_s2m, v, kp, np, err, errlen, d->bf16);
  }
  if (d->ok_m2m)
    for (long L = 2; L <= n - 1; ++L) {
      const int kp = d->kp_m2m, np = d->np_m2m;
      const double *ops = o->levops + (L - 2) * FMM_NLEVOPS * T * T;
      for (long i = 0; i < (long)kp * np; ++i) v[i] = 0;
      for (long t = 0; t < T; ++t)
        for (long k = 0; k < T; ++k) {
          v[t * kp + k] = ops[FMM_SHFTFN * T * T + t * T + k];
          v[t * kp + T + k] = ops[FMM_SHFTFP * T * T + t * T + k];
        }
      rc |= tc_put(d->tc_m2m[0] + (L - 2) * 2 * d->tc_m2m_stride, d->tc_m2m[1] + (L - 2) * d->tc_m2m_stride16,
                   d->ws_m2m + (L - 2) * d->ws_m2m_stride, v, kp, np, err, errlen, d->bf16);
    }
  if (d->ok_m2l)
    for (long l = 3; l <= n; ++l) {
      const int kp = d->kp_m2l, np = d->np_m2l;
      const double *ops = o->levops + (l - 3) * FMM_NLEVOPS * T * T;
      for (long i = 0; i < (long)kp * np; ++i) v[i] = 0;
#define OPT(which, t, k) ops[(which) * T * T + (t) * T + (k)]
      for (long t = 0; t < T; ++t)
        for (long k = 0; k < T; ++k) {
          v[t * kp + 0 * T + k] = OPT(FMM_SHFTLP, t, k);       /* left child  <- psi parent */
          v[(T + t) * kp + 0 * T + k] = OPT(FMM_SHFTLN, t, k); /* right child <- psi parent */
          v[t * kp + 1 * T + k] = OPT(FMM_FLIP2P, t, k);       /* left  <- phi[2B-2] */
          v[(T + t) * kp + 1 * T + k] = OPT(FMM_FLIP3P, t, k); /* right <- phi[2B-2] */
          v[(T + t) * kp + 2 * T + k] = OPT(FMM_FLIP2P, t, k); /* right <- phi[2B-1] */
          v[t * kp + 3 * T + k] = OPT(FMM_FLIP2N, t, k);       /* left  <- phi[2B+2] */
          v[t * kp + 4 * T + k] = OPT(FMM_FLIP3N, t, k);       /* left  <- phi[2B+3] */
          v[(T + t) * kp + 4 * T + k] = OPT(FMM_FLIP2N, t, k); /* right <- phi[2B+3] */
        }
#undef OPT
      rc |= tc_put(d->tc_m2l[0] + (l - 3) * 2 * d->tc_m2l_stride, d->tc_m2l[1] + (l - 3) * d->tc_m2l_stride16,
                   d->ws_m2l + (l - 3) * d->ws_m2l_stride, v, kp, np, err, errlen, d->bf16);
    }
  /* The two near-field weights of largest magnitude, source offsets d = 0 and d = -1 from the
   * target (|w| up to ~P / pi), are left out of both leaf operators and applied in FP32 when the
   * kernels store the leaf's outputs: split into TF32 parts and summed in the tensor core's FP32
   * accumulator they set the leaf's rounding error (4 x that of FP32 products); without them the
   * remaining terms are O(1) and the leaf's error is that of the FP32 stores' two FMAs. */
  float *w01 = (d->ok_lnb || d->ok_leaf) ? (float *)malloc(sizeof(float) * 2 * S1) : nullptr;
  if ((d->ok_lnb || d->ok_leaf) && !w01) rc = 2;
  if (w01)
    for (long sc = 1; sc < P; ++sc) {
      const double *ct = o->cot + (sc - 1) * 4 * b;
      w01[2 * (sc - 1)] = (float)ct[2 * b], w01[2 * (sc - 1) + 1] = (float)ct[2 * b - 1];
    }
  if (d->ok_leaf && w01)
    for (long sc = 1; sc < P; ++sc) {
      const int kp = d->kp_leaf, np = d->np_leaf;
      const double *ct = o->cot + (sc - 1) * 4 * b;
      for (long i = 0; i < (long)kp * np; ++i) v[i] = 0;
      for (long j = 0; j < b; ++j) {
        for (long k = 0; k < T; ++k) v[j * kp + k] = o->evalm[(j * S1 + (sc - 1)) * T + k];
        for (long q = 0; q < 3 * b; ++q) v[j * kp + T + q] = ct[q + b - j];
        v[j * kp + T + j + b] = 0, v[j * kp + T + j + b - 1] = 0; /* d = 0, -1: in FP32 */
      }
      if (2 * sc >= P) { /* column b: the next box's half-shifted first point (TcLeaf) */
        for (long k = 0; k < T; ++k) v[b * kp + k] = o->evalmh[(sc - P / 2) * T + k];
        for (long q = 0; q < 3 * b; ++q) v[b * kp + T + q] = ct[q];
      }
      rc |= tc_put(d->tc_leaf[0] + (sc - 1) * 2 * d->tc_leaf_stride, d->tc_leaf[1] + (sc - 1) * d->tc_leaf_stride16,
                   d->ws_leaf + (sc - 1) * d->ws_leaf_stride, v, kp, np, err, errlen, d->bf16);
    }
  if (d->ok_lnb && w01) /* neighbour-sum form (TcLeafNb): x_B's weights for boxes B, B+1, B-1 */
    for (long sc = 1; sc < P; ++sc) {
      const int kp = d->kp_lnb, np = d->np_lnb;
      const double *ct = o->cot + (sc - 1) * 4 * b;
      for (long i = 0; i < (long)kp * np; ++i) v[i] = 0;
      for (long j = 0; j < b; ++j) {
        for (long k = 0; k < T; ++k) v[j * kp + k] = o->evalm[(j * S1 + (sc - 1)) * T + k];
        for (long q = 0; q < b; ++q) {
          v[j * kp + T + q] = ct[q + 2 * b - j];           /* window middle: box B */
          v[(b + j) * kp + T + q] = ct[q + b - j];         /* window start of box B+1 */
          v[(2 * b + j) * kp + T + q] = ct[q + 3 * b - j]; /* window end of box B-1 */
        }
      }
      for (long j = 0; j < b; ++j) {
        v[j * kp + T + j] = 0;                        /* d = 0 */
        if (j > 0) v[j * kp + T + j - 1] = 0;         /* d = -1 within box B */
      }
      v[b * kp + T + b - 1] = 0;                      /* d = -1: the last point of B, first target of B+1 */
      if (2 * sc >= P) { /* H(B), and x_B's parts of H(B+1) and H(B-1) */
        for (long k = 0; k < T; ++k) v[3 * b * kp + k] = o->evalmh[(sc - P / 2) * T + k];
        for (long q = 0; q < b; ++q) {
          v[3 * b * kp + T + q] = ct[b + q];
          v[(3 * b + 1) * kp + T + q] = ct[q];
          v[(3 * b + 2) * kp + T + q] = ct[2 * b + q];
        }
      }
      rc |= tc_put(d->tc_lnb[0] + (sc - 1) * 2 * d->tc_lnb_stride, nullptr, nullptr, v, kp, np, err, errlen, 0);
    }
  if (w01) {
    if (!rc && cudaMemcpy(d->lnb_w01, w01, sizeof(float) * 2 * S1, cudaMemcpyHostToDevice) != cudaSuccess) rc = 3;
    free(w01);
  }
  free(v);
  return rc;
}

constexpr long kCoarseRows = 4096; /* default: tree levels with fewer rows form the coarse tree */

/* Coarse-tree settings of a plan: threshold (FMMFFT_COARSE_ROWS overrides, 0 turns the
 * one-launch coarse tree off) and whether the kernel's shared memory fits.  The choice depends on
 * the plan only, so a transform gives the same bits alone, in a batch or in a server mix. */
template <typename R> static void coarse_setup(Dev<R> *d) {
  d->coarse_rows = kCoarseRows;
  if (const char *ev = getenv("FMMFFT_COARSE_ROWS")) d->coarse_rows = atol(ev), d->env_set |= KNOB_COARSE;
  /* two operator buffers where they fit beside the plane's levels, else one */
  d->coarse_dbuf = coarse_smem<R>(d->T, 1) <= (size_t)200 * 1024;
  const size_t sm = coarse_smem<R>(d->T, d->coarse_dbuf);
  int nb = 0;
  if (sm <= (size_t)200 * 1024) {
    /* the attribute is the kernel's, not the plan's: always the full allowance, so that a plan
     * with fewer terms made later does not shrink what an earlier plan's launch needs */
    cudaFuncSetAttribute(k_coarse<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_coarse<R>, 32 * kCoarseWarps, sm);
  }
  d->coarse_grid = nb;
  if (d->coarse_grid < 1) d->coarse_rows = 0; /* operator too large for shared memory */
}

template <typename R>
static int dev_create(const fmm_ops64 *o, int precision, int nb, Dev<R> **out, char *err, size_t errlen,
                      size_t *dry_bytes = nullptr) {
  using C = typename cplx<R>::T;
  Dev<R> *d = new (std::nothrow) Dev<R>();
  if (!d) return 2;
  memset((void *)d, 0, sizeof(*d));
  const long M = o->M, P = o->P, T = o->T, b = o->b, s = o->s, n = o->n, S1 = P - 1;
  d->M = M, d->P = P, d->T = T, d->b = b, d->s = s, d->n = n, d->N = M * P, d->S1 = S1;
  d->precision = precision;
  d->nbmax = nb, d->last_nbt = 1;
  d->tileM = P >= 2048 ? 1 : 2048 / P;
  if (d->tileM > M) d->tileM = M;
  d->ntile = M / d->tileM;
  /* size-M FFT split */
  const long LMAX = sizeof(R) == 4 ? 4096 : 2048;
  if (M <= LMAX) {
    d->M1 = M, d->M2 = 1;
  } else {
    long lg = 0;
    while ((1L << lg) < M) ++lg;
    d->M2 = 1L << ((lg + 1) / 2);
    d->M1 = M / d->M2;
  }
  const long nlev = n - 2 > 0 ? n - 2 : 0;
  const long lvtot = 2 * S1 * T * ((2L << n) - 4);
  /* tensor-core operator shapes (precision FMMFFT_F32_TC only) */
  const int tc = ((precision == 2 || precision == 3) && sizeof(R) == 4);
  d->bf16 = precision == 3 && sizeof(R) == 4;
  auto up8 = [](long v) { return (int)((v + 7) / 8 * 8); };
  auto up16 = [](long v) { return (int)((v + 15) / 16 * 16); };
  d->tc = tc;
  d->kp_s2m = up8(b), d->np_s2m = up16(T);
  d->kp_m2m = up8(2 * T), d->np_m2m = up16(T);
  d->kp_m2l = up8(5 * T), d->np_m2l = up16(2 * T);
  d->kp_leaf = up8(T + 3 * b), d->np_leaf = up16(b + 1); /* + the half-shifted column */
  d->kp_lnb = up8(T + b), d->np_lnb = up16(3 * b + 3);    /* three blocks + three half-shift columns */
  auto fits = [&](int kp, int np) {
    return tc && (T % 4 == 0) && (b % 4 == 0) && np <= 256 && kp <= 256 &&
           tc::smem16_bytes(kp, np) <= (size_t)110 * 1024 && tc::tmem_cols(tc::round16(kp), np) <= 256 &&
           tc::ws_fits(kp, np);
  };
  d->ok_s2m = fits(d->kp_s2m, d->np_s2m);
  d->ok_m2m = fits(d->kp_m2m, d->np_m2m) && nlev > 0;
  d->ok_m2l = fits(d->kp_m2l, d->np_m2l) && nlev > 0;
  /* The leaf's near-field weights are near-singular (|w| ~ P/pi against O(1) sums), and the
   * tensor core's FP32 accumulation over those cancelling sums lifts the transform's rel-L2 from
   * 2.3e-7 (leaf on the CUDA cores) to 6.5e-7 at b = 32 (3.8e-7 at b = 8, 1.8e-7 at b = 16; the
   * same with three TF32 parts per operand, so the split is not the cause), within the 1e-6 bar,
   * for a 1.5x faster leaf.  FMMFFT_TC_STAGES without bit 8 keeps it on the CUDA cores. */
  d->ok_leaf = fits(d->kp_leaf, d->np_leaf);
  /* FMMFFT_LEAF_FORM=row keeps the leaf on the window-row form (TcLeaf) */
  d->ok_lnb = tc && !d->bf16 && T % 4 == 0 && b % 8 == 0 && b <= 32 && d->kp_lnb <= 256 &&
              d->np_lnb <= 128 && tc::smem_bytes(d->kp_lnb, d->np_lnb) <= (size_t)110 * 1024 &&
              tc::nb_tmem_cols(d->kp_lnb, d->np_lnb) <= 256;
  if (const char *ev = getenv("FMMFFT_LEAF_FORM")) d->ok_lnb &= strcmp(ev, "row") != 0;
  d->tc_min_rows = kTcMinRows;
  if (const char *ev = getenv("FMMFFT_TC_MIN_ROWS")) d->tc_min_rows = atol(ev), d->env_set |= KNOB_TCMIN;
  /* FMMFFT_TC_FORM=pipelined routes the tree stages that fit to the warp-specialised kernel
   * (4xTF32, rel-L2 2.4e-7 at N = 2^24, P = 64, 24 terms, against 2.7e-7); the row form stays
   * the default because it is faster there (M2L 0.47 ms against 0.58 ms on a B200) */
  d->tc_form = -1;
  /* per-stage default forms: the 16-lane row form (3) for S2M, M2M and M2L (measured at cfg2
   * with the operators staged by bulk copy: M2L 0.218 ms against 0.240 on the 32-lane form) */
  d->form_m2l = 3;
  if (const char *ev = getenv("FMMFFT_TC_FORM"))
    d->tc_form = strcmp(ev, "row") == 0 ? 0 : strcmp(ev, "row16") == 0 ? 3 : strcmp(ev, "ws") == 0 ? 4 : -1,
    d->env_set |= KNOB_FORM;
  d->pdl = 1;
  if (const char *ev = getenv("FMMFFT_PDL")) d->pdl = atoi(ev) != 0;
  coarse_setup(d);
  /* FMMFFT_FUSE_S2M=0 keeps S2M a separate stage (on the tensor cores for FP32 TC plans) */
  d->fuse_s2m = 1;
  if (const char *ev = getenv("FMMFFT_FUSE_S2M")) d->fuse_s2m = atoi(ev) != 0, d->env_set |= KNOB_FUSE;
  /* compensated twiddles in the FP32 FFT passes: off by default.  Measured on a B200 (N = 2^20
   * .. 2^22, split-TF32 plans): rel-L2 5.2e-7 against 5.6e-7, for FFT pass 1 taking 0.19 ms
   * instead of 0.09 ms at N = 2^24 (the post-twiddle is then gathered per element).
   * FMMFFT_COMP_TWIDDLES=1 turns them on. */
  d->comp_tw = 0;
  if (const char *ev = getenv("FMMFFT_COMP_TWIDDLES")) d->comp_tw = sizeof(R) == 4 && atoi(ev) != 0;
  d->fft_threads = 512;
  if (const char *ev = getenv("FMMFFT_FFT_THREADS")) {
    const int v = atoi(ev);
    if (v >= 32 && v <= 512 && (v & (v - 1)) == 0) d->fft_threads = v, d->env_set |= KNOB_FFT;
  }
  /* FMMFFT_TC_STAGES: bit mask of the stages routed to the tensor cores (1 S2M, 2 M2M, 4 M2L,
   * 8 leaf); default all */
  if (const char *ev = getenv("FMMFFT_TC_STAGES")) {
    long m = atol(ev);
    d->ok_s2m &= (m & 1) != 0, d->ok_m2m &= (m & 2) != 0, d->ok_m2l &= (m & 4) != 0, d->ok_leaf &= (m & 8) != 0;
    d->ok_lnb &= (m & 8) != 0;
  }
  const long sz_s2m = d->ok_s2m ? (long)d->kp_s2m * d->np_s2m : 0;
  d->tc_s2m_stride16 = 2L * tc::round16(d->kp_s2m) * d->np_s2m;
  d->tc_m2m_stride16 = 2L * tc::round16(d->kp_m2m) * d->np_m2m;
  d->tc_m2l_stride16 = 2L * tc::round16(d->kp_m2l) * d->np_m2l;
  d->tc_leaf_stride16 = 2L * tc::round16(d->kp_leaf) * d->np_leaf;
  d->tc_m2m_stride = (long)d->kp_m2m * d->np_m2m;
  d->tc_m2l_stride = (long)d->kp_m2l * d->np_m2l;
  d->tc_leaf_stride = (long)d->kp_leaf * d->np_leaf;
  d->tc_lnb_stride = (long)d->kp_lnb * d->np_lnb;
  const long sz_lnb = d->ok_lnb ? S1 * d->tc_lnb_stride : 0;
  const long sz_m2m = d->ok_m2m ? nlev * d->tc_m2m_stride : 0;
  const long sz_m2l = d->ok_m2l ? nlev * d->tc_m2l_stride : 0;
  const long sz_leaf = d->ok_leaf ? S1 * d->tc_leaf_stride : 0;
  /* in floats; a BF16 block is half as many (its element count is even) */
  const long wdiv = d->bf16 ? 2 : 1;
  d->ws_m2m_stride = (long)tc::ws_b_floats(d->kp_m2m, d->np_m2m) / wdiv;
  d->ws_m2l_stride = (long)tc::ws_b_floats(d->kp_m2l, d->np_m2l) / wdiv;
  d->ws_leaf_stride = (long)tc::ws_b_floats(d->kp_leaf, d->np_leaf) / wdiv;
  const long ws_s2m_n = d->ok_s2m ? (long)tc::ws_b_floats(d->kp_s2m, d->np_s2m) / wdiv : 0;
  const long ws_m2m_n = d->ok_m2m ? nlev * d->ws_m2m_stride : 0;
  const long ws_m2l_n = d->ok_m2l ? nlev * d->ws_m2l_stride : 0;
  const long ws_leaf_n = d->ok_leaf ? S1 * d->ws_leaf_stride : 0;
  size_t off = 0;
#define CARVE(field, count, type)          \
  size_t off_##field = off;                \
  off = align_up(off + sizeof(type) * (size_t)(count));
  CARVE(initch, b * T, R)
  CARVE(btop, T * T, R)
  CARVE(bm2m, (nlev ? nlev : 1) * 2 * T * T, R)
  CARVE(bm2l, (nlev ? nlev : 1) * 10 * T * T, R)
  CARVE(evalmT, S1 * T * b, R)
  CARVE(evalmh, S1 * T, R)
  CARVE(cot, S1 * 4 * b, R)
  CARVE(pretw, P, C)
  CARVE(twP, P, C)
  CARVE(twM, M, C)
  CARVE(pretwlo, d->comp_tw ? P : 0, C)
  CARVE(twPlo, d->comp_tw ? P : 0, C)
  CARVE(twMlo, d->comp_tw ? M : 0, C)
  CARVE(xt, nb * 2 * P * M, R)
  CARVE(part, nb * d->ntile * P, C)
  CARVE(ssum, nb * P, C)
  CARVE(phi, nb * lvtot, R)
  CARVE(psi, nb * lvtot, R)
  CARVE(u, nb * 2 * S1 * M, R)
  CARVE(z, nb * P * M, C)
  CARVE(tmp, nb * P * M, C)
  CARVE(status, 1, int)
  CARVE(sync, 64, unsigned)
  CARVE(tcs2m, 2 * sz_s2m, float)
  CARVE(tcm2m, 2 * sz_m2m, float)
  CARVE(tcm2l, 2 * sz_m2l, float)
  CARVE(tcleaf, 2 * sz_leaf, float)
  CARVE(tclnb, 2 * sz_lnb, float)
  CARVE(tcs2m16, d->ok_s2m ? d->tc_s2m_stride16 : 0, float)
  CARVE(tcm2m16, d->ok_m2m ? nlev * d->tc_m2m_stride16 : 0, float)
  CARVE(tcm2l16, d->ok_m2l ? nlev * d->tc_m2l_stride16 : 0, float)
  CARVE(tcleaf16, d->ok_leaf ? S1 * d->tc_leaf_stride16 : 0, float)
  CARVE(leaffix, (d->ok_leaf || d->ok_lnb) ? nb * 2 * s : 0, float)
  CARVE(lnbw, (d->ok_lnb || d->ok_leaf) ? 2 * S1 : 0, float)
  CARVE(wss2m, ws_s2m_n, float)
  CARVE(wsm2m, ws_m2m_n, float)
  CARVE(wsm2l, ws_m2l_n, float)
  CARVE(wsleaf, ws_leaf_n, float)
#undef CARVE
  if (dry_bytes) {
    *dry_bytes = off;
    delete d;
    return 0;
  }
  void *pool = NULL;
  cudaError_t ce = cudaMalloc(&pool, off);
  if (ce != cudaSuccess) {
    snprintf(err, errlen, "cudaMalloc(%zu): %s", off, cudaGetErrorString(ce));
    delete d;
    return 2;
  }
  d->pool = pool;
  d->bytes = off;
  char *base = (char *)pool;
  d->initch = (R *)(base + off_initch);
  d->btop = (R *)(base + off_btop);
  d->bm2m = (R *)(base + off_bm2m);
  d->bm2l = (R *)(base + off_bm2l);
  d->evalmT = (R *)(base + off_evalmT);
  d->evalmh = (R *)(base + off_evalmh);
  d->cot = (R *)(base + off_cot);
  d->pretw = (C *)(base + off_pretw);
  d->twP = (C *)(base + off_twP);
  d->twM = (C *)(base + off_twM);
  d->pretw_lo = (C *)(base + off_pretwlo);
  d->twP_lo = (C *)(base + off_twPlo);
  d->twM_lo = (C *)(base + off_twMlo);
  d->xt = (R *)(base + off_xt);
  d->part = (C *)(base + off_part);
  d->ssum = (C *)(base + off_ssum);
  d->phi = (R *)(base + off_phi);
  d->psi = (R *)(base + off_psi);
  d->z = (C *)(base + off_z);
  d->tmp = (C *)(base + off_tmp);
  d->u = (R *)(base + off_u);
  d->status = (int *)(base + off_status);
  d->sync = (unsigned *)(base + off_sync);
  d->tc_s2m[0] = (float *)(base + off_tcs2m), d->tc_s2m[1] = (float *)(base + off_tcs2m16);
  d->tc_m2m[0] = (float *)(base + off_tcm2m), d->tc_m2m[1] = (float *)(base + off_tcm2m16);
  d->tc_m2l[0] = (float *)(base + off_tcm2l), d->tc_m2l[1] = (float *)(base + off_tcm2l16);
  d->tc_leaf[0] = (float *)(base + off_tcleaf), d->tc_leaf[1] = (float *)(base + off_tcleaf16);
  d->tc_lnb[0] = (float *)(base + off_tclnb), d->tc_lnb[1] = nullptr;
  d->leaf_fix = (float *)(base + off_leaffix);
  d->lnb_w01 = (float *)(base + off_lnbw);
  d->ws_s2m = (float *)(base + off_wss2m);
  d->ws_m2m = (float *)(base + off_wsm2m);
  d->ws_m2l = (float *)(base + off_wsm2l);
  d->ws_leaf = (float *)(base + off_wsleaf);
  cudaMemset(d->status, 0, sizeof(int));
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&d->num_sms, cudaDevAttrMultiProcessorCount, dev);
  }

  /* ---- operator layouts (FP64 on the host, rounded once to R) ---- */
  int rc = 0;
  size_t hn = (size_t)(10 * T * T);
  if ((size_t)(S1 * T * b) > hn) hn = (size_t)(S1 * T * b);
  if ((size_t)(2 * P) > hn) hn = (size_t)(2 * P);
  double *h = (double *)malloc(sizeof(double) * (hn + 16));
  if (!h) return 2;
  rc |= upload<R>(&d->initch, o->initch, b * T, err, errlen);
  for (long k = 0; k < T; ++k)
    for (long t = 0; t < T; ++t) h[k * T + t] = o->topflp[t * T + k];
  rc |= upload<R>(&d->btop, h, T * T, err, errlen);
  for (long L = 2; L <= n - 1; ++L) { /* M2M parent level L uses shftfn/fp index L-2 */
    const double *ops = o->levops + (L - 2) * FMM_NLEVOPS * T * T;
    for (long k = 0; k < T; ++k)
      for (long t = 0; t < T; ++t) {
        h[k * T + t] = ops[FMM_SHFTFN * T * T + t * T + k];
        h[(T + k) * T + t] = ops[FMM_SHFTFP * T * T + t * T + k];
      }
    R *dst = d->bm2m + (L - 2) * 2 * T * T;
    rc |= upload<R>(&dst, h, 2 * T * T, err, errlen);
  }
  for (long l = 3; l <= n; ++l) { /* M2L+L2L child level l uses index l-3 */
    const double *ops = o->levops + (l - 3) * FMM_NLEVOPS * T * T;
#define OPT(which, t, k) ops[(which) * T * T + (t) * T + (k)]
    const long N2 = 2 * T;
    for (long i = 0; i < 10 * T * T; ++i) h[i] = 0;
    for (long k = 0; k < T; ++k)
      for (long t = 0; t < T; ++t) {
        h[(0 * T + k) * N2 + t] = OPT(FMM_SHFTLP, t, k);     /* psi parent -> left */
        h[(0 * T + k) * N2 + T + t] = OPT(FMM_SHFTLN, t, k); /* psi parent -> right */
        h[(1 * T + k) * N2 + t] = OPT(FMM_FLIP2P, t, k);     /* phi[2B-2] -> left  (c-2) */
        h[(1 * T + k) * N2 + T + t] = OPT(FMM_FLIP3P, t, k); /* phi[2B-2] -> right (c-3) */
        h[(2 * T + k) * N2 + T + t] = OPT(FMM_FLIP2P, t, k); /* phi[2B-1] -> right (c-2) */
        h[(3 * T + k) * N2 + t] = OPT(FMM_FLIP2N, t, k);     /* phi[2B+2] -> left  (c+2) */
        h[(4 * T + k) * N2 + t] = OPT(FMM_FLIP3N, t, k);     /* phi[2B+3] -> left  (c+3) */
        h[(4 * T + k) * N2 + T + t] = OPT(FMM_FLIP2N, t, k); /* phi[2B+3] -> right (c+2) */
      }
#undef OPT
    R *dst = d->bm2l + (l - 3) * 10 * T * T;
    rc |= upload<R>(&dst, h, 10 * T * T, err, errlen);
  }
  for (long sc = 1; sc < P; ++sc)
    for (long k = 0; k < T; ++k)
      for (long j = 0; j < b; ++j) h[((sc - 1) * T + k) * b + j] = o->evalm[(j * S1 + (sc - 1)) * T + k];
  rc |= upload<R>(&d->evalmT, h, S1 * T * b, err, errlen);
  for (long i = 0; i < S1 * T; ++i) h[i] = 0;
  for (long sc = P / 2; sc < P; ++sc)
    for (long k = 0; k < T; ++k) h[(sc - 1) * T + k] = o->evalmh[(sc - P / 2) * T + k];
  rc |= upload<R>(&d->evalmh, h, S1 * T, err, errlen);
  rc |= upload<R>(&d->cot, o->cot, S1 * 4 * b, err, errlen);
  const double PI = 3.14159265358979323846264338327950288;
  h[0] = 0, h[1] = 0;
  for (long sc = 1; sc < P; ++sc) {
    h[2 * sc] = -cos(PI * sc / P) * sin(PI * sc / P);
    h[2 * sc + 1] = sin(PI * sc / P) * sin(PI * sc / P);
  }
  rc |= upload<R>((R **)&d->pretw, h, 2 * P, err, errlen);
  if (d->comp_tw) rc |= upload_lo(d->pretw_lo, h, 2 * P, err, errlen);
  for (long k = 0; k < P; ++k) h[2 * k] = cos(2 * PI * k / P), h[2 * k + 1] = -sin(2 * PI * k / P);
  rc |= upload<R>((R **)&d->twP, h, 2 * P, err, errlen);
  if (d->comp_tw) rc |= upload_lo(d->twP_lo, h, 2 * P, err, errlen);
  free(h);
  double *hm = (double *)malloc(sizeof(double) * 2 * (size_t)M);
  if (!hm) return 2;
  for (long k = 0; k < M; ++k) {
    double a = 2 * PI * (double)k / (double)M;
    hm[2 * k] = cos(a), hm[2 * k + 1] = -sin(a);
  }
  rc |= upload<R>((R **)&d->twM, hm, 2 * M, err, errlen);
  if (d->comp_tw) rc |= upload_lo(d->twM_lo, hm, 2 * M, err, errlen);
  free(hm);
  if (tc && !rc) rc = tc_upload_ops(d, o, err, errlen);
  if (rc) {
    cudaFree(pool);
    delete d;
    return rc;
  }
  if (cudaStreamCreateWithFlags(&d->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError(); /* no side stream: the sums run in line */
    if (d->side) cudaStreamDestroy(d->side);
    if (d->ev_fork) cudaEventDestroy(d->ev_fork);
    d->side = nullptr, d->ev_fork = d->ev_join = nullptr;
  }
  *out = d;
  return 0;
}

/* Frees a plan's device state. */
template <typename R> static void dev_release(Dev<R> *d) {
  if (!d) return;
  if (d->side) cudaStreamDestroy(d->side);
  if (d->ev_fork) cudaEventDestroy(d->ev_fork);
  if (d->ev_join) cudaEventDestroy(d->ev_join);
  cudaFree(d->pool);
  delete d;
}

/* Parts of one execute (a shard of a sharded transform runs its plan's stages in pieces, with
 * exchanges between them); a null control runs the whole transform. */
struct ExecCtl {
  unsigned mask;                        /* stages to run: bit 1 << ST_* */
  long m2m_stop, m2l_from;              /* lowest M2M parent level, first M2L child level (0: own) */
  int no_coarse;                        /* every tree level on its own, no coarse-tree kernel */
  long sum_t0, sum_nt;                  /* section sums over tiles [sum_t0, sum_t0 + sum_nt) */
  void *sum_out;                        /* ... into this P-vector (null: the plan's) */
  long comb_m0, comb_cols, comb_ostride; /* combine of columns [m0, m0 + cols) into rows of ostride */
  void *comb_out;
  double comb_invM;                     /* 1 / M of the whole transform */
};

template <typename R>
static int dev_execute(Dev<R> *d, const void *vin, void *vout, cudaStream_t st, int inverse,
                       int nbt, char *err, size_t errlen, const void *const *ins = nullptr,
                       void *const *outs = nullptr, const ExecCtl *ctl = nullptr) {
  using C = typename cplx<R>::T;
  auto run = [&](int stg) { return !ctl || ((ctl->mask >> stg) & 1u); };
  /* ins / outs (both or neither): transform tr reads ins[tr] and writes outs[tr] instead of
   * vin + tr N and vout + tr N */
  InTab xin{};
  if (ins)
    for (int i = 0; i < nbt; ++i) xin.p[i] = ins[i];
  xin.n = ins ? nbt : 0;
  auto out_tab = [&](long rows) { /* the last pass's output rows, `rows` of them in all */
    OutTab o{};
    if (outs) {
      for (int i = 0; i < nbt; ++i) o.p[i] = outs[i];
      o.rpp = (int)(rows / nbt);
    }
    return o;
  };
  const long M = d->M, P = d->P, T = d->T, b = d->b, s = d->s, n = d->n, S1 = d->S1;
  /* nbt transforms of this shape, inputs and outputs N apart: every tree stage runs over the
   * rows of all of them at once (the expansion planes of transform tr follow those of tr - 1
   * within each level), the other stages take the transform as a grid dimension */
  if (nbt < 1 || nbt > d->nbmax) {
    snprintf(err, errlen, "execute of %d transforms on a plan that holds %d", nbt, d->nbmax);
    return 1;
  }
  d->last_nbt = nbt;
  const long S1e = (long)nbt * S1;
  const C *x = (const C *)vin;
  C *y = (C *)vout;
  Prof &pf = d->prof;
  const int slot = (pf.on && pf.count < pf.cap) ? pf.count++ : -1;
  int cur = -1;
  auto stage = [&](int id) {
    if (slot >= 0)
      for (int k = cur + 1; k <= id; ++k) cudaEventRecord(pf.ev[slot * (ST_COUNT + 1) + k], st);
    cur = id;
  };
  for (int k = 0; k < ST_COUNT; ++k) pf.launches[k] = 0;
  /* 1-2: sections and their sums */
  stage(ST_SECTIONS);
  /* S2M fused into the sections pass when tiles hold whole leaf boxes */
  const bool s2m_fused = d->tileM % b == 0 && T % 4 == 0 && d->fuse_s2m;
  if (run(ST_SECTIONS)) {
    int TMt = (int)d->tileM;
    size_t sm = sizeof(C) * TMt * (P + 1) + (s2m_fused ? sizeof(R) * b * T : 0);
    k_sections<R><<<dim3((unsigned)d->ntile, (unsigned)nbt), 256, sm, st>>>(
        x, d->xt, d->part, M, (int)P, TMt, inverse, d->initch,
        s2m_fused ? d->phi + lvl_off(n, S1e, T) : nullptr, (int)b, (int)T, xin);
    pf.launches[ST_SECTIONS]++;
  }
  stage(ST_SUMS);
  bool sums_forked = false;
  if (run(ST_SUMS)) { /* a shard sums its own tiles only */
    const long t0 = ctl ? ctl->sum_t0 : 0, nt = ctl ? ctl->sum_nt : d->ntile;
    C *out = (ctl && ctl->sum_out) ? (C *)ctl->sum_out : d->ssum;
    cudaStream_t ss = st;
    if (!ctl && d->side) { /* off the critical path until the combine */
      cudaEventRecord(d->ev_fork, st);
      cudaStreamWaitEvent(d->side, d->ev_fork, 0);
      ss = d->side, sums_forked = true;
    }
    k_sum_sections<R><<<dim3((unsigned)P, (unsigned)nbt), 256, 0, ss>>>(d->part + t0 * P, nt, (int)P, out);
    if (sums_forked) cudaEventRecord(d->ev_join, ss);
    pf.launches[ST_SUMS]++;
  }
  /* 3: S2M at level n (done in stage 1 when fused) */
  stage(ST_S2M);
  if (!s2m_fused && run(ST_S2M)) {
    bool done = false;
    if constexpr (sizeof(R) == 4) {
      if (d->tc && d->ok_s2m && 2 * S1 * s >= d->tc_min_rows) {
        TcS2M q{};
        q.rows = 2 * S1 * s, q.batches = nbt, q.nchunks = 1, q.clen[0] = (int)b, q.coff[0] = 0;
        q.P = (int)P;
        q.kpad = d->kp_s2m, q.npad = d->np_s2m, q.nout = (int)T;
        q.bimg = d->tc_s2m[0], q.bimg16 = d->tc_s2m[1], q.bimg_stride = q.bimg16_stride = 0;
        q.wsb = d->ws_s2m, q.wsb_stride = 0;
        q.xt = d->xt, q.out = d->phi + lvl_off(n, S1e, T), q.M = M, q.b = (int)b, q.T = (int)T;
        launch_tc(q, d->num_sms, d->status, st, d->tc_form < 0 ? 3 : d->tc_form, d->pdl, d->bf16);
        done = true;
      }
    }
    if (!done) {
      ProbS2M<R> pb{d->xt, d->initch, d->phi + lvl_off(n, S1e, T), 2 * S1 * s, M, (int)b, (int)T, (int)P};
      launch_rowgemm<R>(pb, pb.rows, (int)T, nbt, st);
    }
    pf.launches[ST_S2M]++;
  }
  /* coarse tree: levels below the row threshold run in one cooperative launch (stage 5) */
  long thr = d->coarse_rows;
  if (d->tc && d->tc_min_rows < thr) thr = d->tc_min_rows; /* never take a level off the TCs */
  /* routing by the row counts of ONE transform, so that a transform takes the same kernels (and
   * gives the same bits) alone and in a batch */
  const bool coarse = !(ctl && ctl->no_coarse) && d->coarse_grid >= 1 && thr > 2 * S1 * 4;
  long Lm = 1, Ll = 2;
  if (coarse) { /* and at most 2^kCoarseMaxLevel boxes per plane (one block runs a plane) */
    for (long L = 2; L <= n - 1 && L <= kCoarseMaxLevel; ++L)
      if (2 * S1 * (1L << L) < thr) Lm = L;
    for (long l = 3; l <= n && l - 1 <= kCoarseMaxLevel; ++l)
      if (2 * S1 * (1L << (l - 1)) < thr) Ll = l;
  }
  /* 4: M2M, parent level L = n-1 .. 2 (.. Lm+1 with the coarse tree) */
  stage(ST_M2M);
  const long m2m_stop = (ctl && ctl->m2m_stop) ? ctl->m2m_stop : (coarse ? Lm + 1 : 2);
  for (long L = n - 1; run(ST_M2M) && L >= m2m_stop; --L) {
    bool done = false;
    if constexpr (sizeof(R) == 4) {
      if (d->tc && d->ok_m2m && 2 * S1 * (1L << L) >= d->tc_min_rows) {
        TcM2M q{};
        q.rows = 2 * S1e * (1L << L), q.batches = 1, q.nchunks = 1, q.clen[0] = (int)(2 * T), q.coff[0] = 0;
        q.kpad = d->kp_m2m, q.npad = d->np_m2m, q.nout = (int)T;
        q.bimg = d->tc_m2m[0] + (L - 2) * 2 * d->tc_m2m_stride, q.bimg16 = d->tc_m2m[1] + (L - 2) * d->tc_m2m_stride16;
        q.bimg_stride = q.bimg16_stride = 0, q.wsb = d->ws_m2m + (L - 2) * d->ws_m2m_stride, q.wsb_stride = 0;
        q.child = d->phi + lvl_off(L + 1, S1e, T), q.out = d->phi + lvl_off(L, S1e, T), q.T = (int)T;
        launch_tc(q, d->num_sms, d->status, st, d->tc_form < 0 ? 3 : d->tc_form, d->pdl, d->bf16);
        done = true;
      }
    }
    if (!done) {
      ProbM2M<R> pb{d->phi + lvl_off(L + 1, S1e, T), d->bm2m + (L - 2) * 2 * T * T,
                    d->phi + lvl_off(L, S1e, T), 2 * S1e * (1L << L), (int)(2 * T), (int)T};
      launch_rowgemm<R>(pb, pb.rows, (int)T, 1, st);
    }
    pf.launches[ST_M2M]++;
  }
  /* 5: top flip, or the whole coarse tree (M2M Lm..2, top flip, M2L 3..Ll) */
  stage(ST_TOP);
  if (!run(ST_TOP)) {
  } else if (coarse) {
    CoarseArgs<R> ca{d->phi, d->psi, d->bm2m, d->btop, d->bm2l, S1e, (int)T, (int)Lm, (int)Ll, d->coarse_dbuf};
    /* one block per expansion plane of every transform of the execute; a programmatic dependent
     * launch (it stages its first operator before waiting for the level below) */
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(2 * S1e));
    cfg.blockDim = dim3(32 * kCoarseWarps);
    cfg.dynamicSmemBytes = coarse_smem<R>(T, d->coarse_dbuf);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = d->pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k_coarse<R>, ca);
    pf.launches[ST_TOP]++;
  } else {
    ProbTop<R> pb{d->phi + lvl_off(2, S1e, T), d->btop, d->psi + lvl_off(2, S1e, T), 2 * S1e * 4,
                  (int)T, (int)T};
    launch_rowgemm<R>(pb, pb.rows, (int)T, 1, st);
    pf.launches[ST_TOP]++;
  }
  /* 6: M2L + L2L, child level l = 3..n (Ll+1..n with the coarse tree; rows = parent boxes) */
  stage(ST_M2L);
  const long m2l_from = (ctl && ctl->m2l_from) ? ctl->m2l_from : (coarse ? Ll + 1 : 3);
  for (long l = m2l_from; run(ST_M2L) && l <= n; ++l) {
    bool done = false;
    if constexpr (sizeof(R) == 4) {
      if (d->tc && d->ok_m2l && 2 * S1 * (1L << (l - 1)) >= d->tc_min_rows) {
        TcM2L q{};
        q.rows = 2 * S1e * (1L << (l - 1)), q.batches = 1, q.nchunks = 3;
        q.clen[0] = (int)T, q.clen[1] = (int)(2 * T), q.clen[2] = (int)(2 * T);
        q.coff[0] = 0, q.coff[1] = (int)T, q.coff[2] = (int)(3 * T);
        q.kpad = d->kp_m2l, q.npad = d->np_m2l, q.nout = (int)(2 * T);
        q.bimg = d->tc_m2l[0] + (l - 3) * 2 * d->tc_m2l_stride, q.bimg16 = d->tc_m2l[1] + (l - 3) * d->tc_m2l_stride16;
        q.bimg_stride = q.bimg16_stride = 0, q.wsb = d->ws_m2l + (l - 3) * d->ws_m2l_stride, q.wsb_stride = 0;
        q.psi_par = d->psi + lvl_off(l - 1, S1e, T), q.phi = d->phi + lvl_off(l, S1e, T);
        q.out = d->psi + lvl_off(l, S1e, T), q.T = (int)T, q.lpar = (int)(l - 1);
        launch_tc(q, d->num_sms, d->status, st, d->tc_form < 0 ? d->form_m2l : d->tc_form, d->pdl, d->bf16);
        done = true;
      }
    }
    if (!done) {
      ProbM2L<R> pb{d->psi + lvl_off(l - 1, S1e, T), d->phi + lvl_off(l, S1e, T),
                    d->bm2l + (l - 3) * 10 * T * T, d->psi + lvl_off(l, S1e, T),
                    2 * S1e * (1L << (l - 1)), (int)(5 * T), (int)(2 * T), (int)T, (int)(l - 1)};
      launch_rowgemm<R>(pb, pb.rows, (int)(2 * T), 1, st);
    }
    pf.launches[ST_M2L]++;
  }
  /* 7: leaf far + near field per section, then the half-shifted first points */
  stage(ST_LEAF);
  if (run(ST_LEAF)) {
    ProbLeaf<R> pb{};
    pb.psi_n = d->psi + lvl_off(n, S1e, T);
    pb.xt = d->xt;
    pb.evalmT = d->evalmT;
    pb.cot = d->cot;
    pb.u = d->u;
    pb.rows = 2 * s, pb.M = M, pb.s = s;
    pb.K = (int)(T + 3 * b), pb.N = (int)b, pb.T = (int)T, pb.b = (int)b;
    bool done = false;
    if constexpr (sizeof(R) == 4) {
      const bool tc_leaf_rows = d->tc && 2 * s >= (d->tc_min_rows < 256 ? d->tc_min_rows : 256);
      if (tc_leaf_rows && d->ok_lnb && d->tc_form < 0) { /* neighbour-sum form */
        TcLeafNb q{};
        q.rows = 2 * s * nbt, q.batches = (int)S1, q.nchunks = 2;
        q.clen[0] = (int)T, q.clen[1] = (int)b, q.coff[0] = 0, q.coff[1] = (int)T;
        q.kpad = d->kp_lnb, q.npad = d->np_lnb, q.nout = (int)b;
        q.bimg = d->tc_lnb[0], q.bimg_stride = 2 * d->tc_lnb_stride, q.bimg16 = nullptr, q.bimg16_stride = 0;
        q.w01 = d->lnb_w01;
        q.fixbuf = d->leaf_fix, q.P = (int)P;
        q.psi_n = pb.psi_n, q.xt = d->xt, q.u = d->u, q.M = M, q.s = s, q.T = (int)T, q.b = (int)b;
        q.log2s = (int)n, q.strips = 2L * nbt;
        launch_nb(q, d->num_sms, d->status, st, d->pdl);
        done = true;
      } else if (tc_leaf_rows && d->ok_leaf) {
        TcLeaf q{};
        q.rows = 2 * s * nbt, q.batches = (int)S1, q.nchunks = 4;
        q.clen[0] = (int)T, q.clen[1] = q.clen[2] = q.clen[3] = (int)b;
        q.coff[0] = 0, q.coff[1] = (int)T, q.coff[2] = (int)(T + b), q.coff[3] = (int)(T + 2 * b);
        q.kpad = d->kp_leaf, q.npad = d->np_leaf, q.nout = (int)b;
        q.bimg = d->tc_leaf[0], q.bimg_stride = 2 * d->tc_leaf_stride, q.w01 = d->lnb_w01;
        q.bimg16 = d->tc_leaf[1], q.bimg16_stride = d->tc_leaf_stride16;
        q.wsb = d->ws_leaf, q.wsb_stride = d->ws_leaf_stride;
        q.fixbuf = d->leaf_fix, q.P = (int)P;
        q.psi_n = pb.psi_n, q.xt = d->xt, q.u = d->u, q.M = M, q.s = s, q.T = (int)T, q.b = (int)b;
        q.log2s = (int)n;
        launch_tc(q, d->num_sms, d->status, st, d->tc_form < 0 ? 0 : d->tc_form, d->pdl, d->bf16);
        done = true;
      }
    }
    if (!done && b % 8 == 0) {
      /* direct form; it also evaluates the half-shifted first points */
      /* boxes per block: two 8-target groups per thread for FP32, one for FP64 */
      int NB = (int)((sizeof(R) == 4 ? 512 : 256) / (b / 8));
      if (NB < 1) NB = 1;
      if (NB > s) NB = (int)s;
      const int e_in_smem = (size_t)T * b * sizeof(R) <= 16384;
      size_t sm = sizeof(R) * ((size_t)(NB + 3) * skew_pitch(b) +
                               (((size_t)(NB + 1) * skew_pitch(T) + 7) & ~(size_t)7) + 8 * b +
                               ((T + 7) & ~7) + (e_in_smem ? (size_t)T * b : 0));
      dim3 g((unsigned)(s / NB), (unsigned)(2 * S1), (unsigned)nbt);
      k_leaf<R><<<g, 256, sm, st>>>(pb.psi_n, d->xt, d->evalmT, d->evalmh, d->cot, d->u, M, s,
                                    (int)T, (int)b, (int)P, NB, e_in_smem);
      pf.launches[ST_LEAF]++;
    } else if (!done) {
      for (int tr = 0; tr < nbt; ++tr) { /* one launch per transform of the batch */
        ProbLeaf<R> pt = pb;
        pt.psi_n += (long)tr * 2 * S1 * s * T, pt.xt += (long)tr * 2 * P * M, pt.u += (long)tr * 2 * S1 * M;
        launch_rowgemm<R>(pt, pt.rows, (int)b, (int)S1, st);
        pf.launches[ST_LEAF]++;
      }
      stage(ST_LEAFFIX);
      pf.launches[ST_LEAFFIX]++;
      dim3 g((unsigned)((2 * s + 8 * kFixBoxes - 1) / (8 * kFixBoxes)), (unsigned)(P - P / 2), (unsigned)nbt);
      k_leaf_fix<R><<<g, 256, 0, st>>>(pb.psi_n, d->xt, d->evalmh, d->cot, d->u, M, s, (int)n, (int)T,
                                       (int)b, (int)P);
    } else { /* tensor-core leaf: it stored the half-shifted points; section P/2 averages them */
      pf.launches[ST_LEAF]++;
      stage(ST_LEAFFIX);
      pf.launches[ST_LEAFFIX]++;
      k_leaf_mid<R><<<dim3((unsigned)((2 * s + 255) / 256), (unsigned)nbt), 256, 0, st>>>(
          d->u, d->leaf_fix, M, s, (int)n, (int)b, (int)P);
    }
  }
  /* 8: combine -> z[P][M] */
  stage(ST_COMBINE);
  /* a shard combines its own columns [m0, m0 + cols) of its strip into rows of ostride */
  const long cm0 = ctl ? ctl->comb_m0 : 0, ccols = ctl ? ctl->comb_cols : M, costr = ctl ? ctl->comb_ostride : M;
  C *const cz = ctl ? (C *)ctl->comb_out : d->z;
  const R cinvM = ctl ? (R)ctl->comb_invM : R(1) / R(M);
  if (ctl && run(ST_COMBINE) && !(P >= 16 && P * M < (1L << 32))) {
    snprintf(err, errlen, "a column window of the combine needs P >= 16");
    return 1;
  }
  if (sums_forked) cudaStreamWaitEvent(st, d->ev_join, 0); /* the combine reads the sums */
  if (!run(ST_COMBINE)) {
  } else if (P >= 16 && P * M < (1L << 32)) {
    pf.launches[ST_COMBINE]++;
    /* register Stockham over sections, Wc columns per block, the pre-twiddle in the loader */
    int Wc = 512 / (int)(P / 8);
    if (Wc > 32) Wc = 32;
    if (Wc > M) Wc = (int)M;
    FftPass fp{};
    fp.L = (int)P, fp.W = Wc, fp.per = (int)(M < (1L << 30) ? M : (1L << 30)), fp.M = M;
    fp.irow = 0, fp.orow = P * costr, fp.oseq = 1, fp.ostr = costr, fp.tws = 1; /* row = transform */
    fp.twiddle_post = 0, fp.conj_out = 0, fp.twmul = 1, fp.twmask = 0, fp.twbits = 0;
    const CombineLd<R> cl{d->xt, d->u, d->ssum, d->pretw, M, cinvM, (int)P,
                          d->comp_tw ? d->pretw_lo : nullptr, cm0};
    const int thr = Wc * (int)(P / 8);
    const size_t sm = sizeof(C) * fft_smem_elems((int)P, Wc);
    if (d->comp_tw && sizeof(R) == 4)
      k_fft_reg<R, false, false, CombineLd<R>, true>
          <<<dim3((unsigned)(ccols / Wc), (unsigned)nbt), thr, sm + sizeof(C) * (size_t)(P + P / 16 + 1), st>>>(
              cl, cz, d->twP, d->twP, fp, d->twP_lo, d->twP_lo);
    else if (P == 64) /* a build for 64 sections */
      k_fft_reg<R, false, false, CombineLd<R>, false, 6><<<dim3((unsigned)(ccols / Wc), (unsigned)nbt), thr, sm, st>>>(
          cl, cz, d->twP, d->twP, fp);
    else
      k_fft_reg<R, false, false, CombineLd<R>><<<dim3((unsigned)(ccols / Wc), (unsigned)nbt), thr, sm, st>>>(
          cl, cz, d->twP, d->twP, fp);
  } else {
    pf.launches[ST_COMBINE]++;
    int TMc = (int)(P >= 1024 ? 1 : (1024 / P < 32 ? 1024 / P : 32));
    if (TMc > M) TMc = (int)M;
    size_t sm = 2 * sizeof(C) * (size_t)P * TMc;
    k_combine<R><<<dim3((unsigned)(M / TMc), (unsigned)nbt), 256, sm, st>>>(d->xt, d->u, d->ssum, d->pretw,
                                                                             d->twP, d->z, M, (int)P, TMc);
  }
  /* 9: size-M FFTs, z -> y */
  stage(ST_FFT1);
  if (run(ST_FFT1)) {
    const long SMEM = 96 * 1024;
    if (d->M2 == 1) {
      int W = (int)pow2_floor(SMEM / (long)(2 * sizeof(C) * M));
      if (W > P) W = (int)P;
      /* W rows of one sequence each: treat them as one "row" of W sequences */
      FftPass fp{(int)M, W, W, M * W, M, 1, M, 1, 0, 1, inverse};
      if (M >= 16 && M <= 8L * d->fft_threads) { /* register kernel: its own W, rows = P / W */
        int Wr = d->fft_threads / (int)(M / 8);
        if (Wr > 16) Wr = 16;
        if (Wr > P) Wr = (int)P;
        if (Wr < 1) Wr = 1;
        fp.M = M * Wr;
        const OutTab ot = out_tab(nbt * P / Wr);
        launch_fft_pass<R>(d->z, y, d->twM, fp, Wr, nbt * P / Wr, W, d->fft_threads, st,
                           d->comp_tw ? d->twM_lo : nullptr, &ot);
      } else {
        const OutTab ot = out_tab(nbt * P / W);
        launch_fft_pass<R>(d->z, y, d->twM, fp, W, nbt * P / W, W, d->fft_threads, st,
                           d->comp_tw ? d->twM_lo : nullptr, &ot);
      }
      pf.launches[ST_FFT1]++;
    } else {
      const long M1 = d->M1, M2 = d->M2;
      /* pass 1: for each m1, DFT over m2 (stride M1), twiddle, store tmp[k2*M1 + m1] */
      int W1 = (int)pow2_floor(SMEM / (long)(2 * sizeof(C) * M2));
      if (W1 > 16) W1 = 16;
      if (W1 > M1) W1 = (int)M1;
      FftPass f1{(int)M2, W1, (int)M1, M, 1, M1, 1, M1, 1, M / M2, 0};
      launch_fft_pass<R>(d->z, d->tmp, d->twM, f1, M1, nbt * P, W1, d->fft_threads, st,
                         d->comp_tw ? d->twM_lo : nullptr);
      pf.launches[ST_FFT1]++;
      stage(ST_FFT2);
      /* pass 2: for each k2, DFT over m1 (contiguous), store y[k2 + M2*k1] */
      int W2 = (int)pow2_floor(SMEM / (long)(2 * sizeof(C) * M1));
      if (W2 > 16) W2 = 16;
      if (W2 > M2) W2 = (int)M2;
      FftPass f2{(int)M1, W2, (int)M2, M, M1, 1, 1, M2, 0, M / M1, inverse};
      const OutTab ot = out_tab(nbt * P);
      launch_fft_pass<R>(d->tmp, y, d->twM, f2, M2, nbt * P, W2, d->fft_threads, st,
                         d->comp_tw ? d->twM_lo : nullptr, &ot);
      pf.launches[ST_FFT2]++;
    }
  }
  stage(ST_DC);
  /* below 10 terms the FMM's own truncation at these bins exceeds FP32 resolution (3e-8 at
   * 10 terms, 5e-6 at 8), and the reference's value is the FMM one, so it is kept */
  if (sizeof(R) == 4 && T >= 10 && run(ST_DC)) {
    k_block_dc<R><<<dim3((unsigned)((P + 3) / 4), (unsigned)nbt), 128, 0, st>>>(d->ssum, y, M, (int)P, inverse,
                                                                                    out_tab(nbt));
    pf.launches[ST_DC]++;
  }
  if (slot >= 0) cudaEventRecord(pf.ev[slot * (ST_COUNT + 1) + ST_COUNT], st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(err, errlen, "kernel launch: %s", cudaGetErrorString(e));
    return 3;
  }
  return 0;
}

/* ======================================================================== autotuner */
/* The plan's stage choices that do not change what is computed, only which kernels compute it
 * and how: FFT block size, coarse-tree threshold (the one-launch coarse levels), the row count
 * from which tree stages run on the tensor cores, and S2M fused into the sections pass.  On the
 * first plan of each (N, P, terms, b, precision) in a process the autotuner times the
 * candidates on one transform (coordinate descent: each knob over its values with the others at
 * their best so far; each candidate the fastest of 5 executes after 2 warm-ups, in place on the
 * plan's own workspace) and caches the winner; every later plan of that key, batched or not,
 * takes the cached choice, so
 * transforms of one shape give the same bits alone, in a batch or in a server mix.  Knobs an
 * environment switch fixed are not tuned.  FP64 plans keep the defaults. */
struct TuneKey { /* the capacity is not part of it: a batch must take its transforms' choice */
  long N, P, T, b;
  int prec;
};
struct TuneVal {
  int fft_threads, fuse_s2m;
  long coarse_rows, tc_min_rows;
  int tc_form;
};
static std::mutex g_tune_mu;
static TuneKey g_tune_key[256];
static TuneVal g_tune_val[256];
static int g_ntune;

template <typename R> static void tune_apply(Dev<R> *d, const TuneVal &v) {
  if (!(d->env_set & KNOB_FFT)) d->fft_threads = v.fft_threads;
  if (!(d->env_set & KNOB_FUSE)) d->fuse_s2m = v.fuse_s2m;
  if (!(d->env_set & KNOB_COARSE)) d->coarse_rows = v.coarse_rows;
  if (!(d->env_set & KNOB_TCMIN)) d->tc_min_rows = v.tc_min_rows;
  if (!(d->env_set & KNOB_FORM)) d->tc_form = v.tc_form;
  d->tuned = 1;
}

template <typename R>
static int dev_autotune(Dev<R> *d, char *err, size_t errlen) {
  using C = typename cplx<R>::T;
  TuneKey key;
  memset(&key, 0, sizeof key);
  key.N = d->N, key.P = d->P, key.T = d->T, key.b = d->b, key.prec = d->precision;
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    for (int i = 0; i < g_ntune; ++i)
      if (!memcmp(&g_tune_key[i], &key, sizeof key)) {
        tune_apply(d, g_tune_val[i]);
        return 0;
      }
  }
  cudaStream_t st;
  FMM_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0), cudaEventCreate(&e1);
  const int nbt = 1; /* one transform: the choice is per transform, whatever the capacity */
  FMM_CUDA_TRY(cudaMemsetAsync(d->z, 0, sizeof(C) * (size_t)d->N * nbt, st));
  int rc = 0;
  auto measure = [&]() -> float {
    float best = 1e30f;
    for (int it = 0; it < 7 && !rc; ++it) {
      cudaEventRecord(e0, st);
      rc = dev_execute(d, d->z, d->z, st, 0, nbt, err, errlen);
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (it >= 2 && ms < best) best = ms;
    }
    return best;
  };
  TuneVal cur;
  memset(&cur, 0, sizeof cur);
  cur.fft_threads = d->fft_threads, cur.fuse_s2m = d->fuse_s2m, cur.coarse_rows = d->coarse_rows;
  cur.tc_min_rows = d->tc_min_rows, cur.tc_form = d->tc_form;
  float best = measure();
  auto knob = [&](unsigned bit, auto set, const long *vals, int nv) {
    if (d->env_set & bit) return;
    TuneVal keep = cur;
    for (int i = 0; i < nv && !rc; ++i) {
      TuneVal c = cur;
      set(c, vals[i]);
      if (!memcmp(&c, &cur, sizeof c)) continue;
      tune_apply(d, c);
      const float t = measure();
      if (t < best * 0.98f) best = t, keep = c; /* a 2% margin: noise does not flip the choice */
    }
    cur = keep;
    tune_apply(d, cur);
  };
  if (d->tc && !d->bf16) { /* tensor-core kernel: per-stage row forms, 16-lane everywhere, warp-specialised */
    const long v[] = {-1, 3, 4};
    knob(KNOB_FORM, [](TuneVal &c, long x) { c.tc_form = (int)x; }, v, 3);
  }
  if (d->tc) {
    const long v[] = {1024, 4096, 16384};
    knob(KNOB_TCMIN, [](TuneVal &c, long x) { c.tc_min_rows = x; }, v, 3);
  }
  if (d->coarse_grid >= 1) {
    const long v[] = {0, 2048, 4096, 8192, 16384};
    knob(KNOB_COARSE, [](TuneVal &c, long x) { c.coarse_rows = x; }, v, 4);
  }
  if (d->tileM % d->b == 0 && d->T % 4 == 0) {
    const long v[] = {0, 1};
    knob(KNOB_FUSE, [](TuneVal &c, long x) { c.fuse_s2m = (int)x; }, v, 2);
  }
  {
    const long v[] = {256, 512};
    knob(KNOB_FFT, [](TuneVal &c, long x) { c.fft_threads = (int)x; }, v, 2);
  }
  cudaEventDestroy(e0), cudaEventDestroy(e1);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(g_tune_mu);
  if (g_ntune < 256) g_tune_key[g_ntune] = key, g_tune_val[g_ntune] = cur, ++g_ntune;
  return 0;
}

/* ======================================================================== C interface */

/* Opt a kernel in to the largest dynamic shared memory the device allows next to its static
 * shared memory. */
template <typename K> static void allow_dyn_smem(K *kernel, int maxopt) {
  cudaFuncAttributes a;
  if (cudaFuncGetAttributes(&a, kernel) != cudaSuccess) return;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       maxopt - (int)a.sharedSizeBytes);
}

/* cudaFuncSetAttribute acts on the current device only, so the opt-in is made once per device
 * (plans and allocation-free calls may run on several GPUs of one process). */
#define FMMK_MAXDEV 64
static int set_smem_limits(void) {
  static volatile int done[FMMK_MAXDEV];
  int maxopt = 0, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 3;
  if (dev < FMMK_MAXDEV && done[dev]) return 0;
  cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int lim = maxopt > 0 ? maxopt : 48 * 1024;
  cudaFuncSetAttribute(k_fft_pass<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_pass<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, false, false, CombineLd<float>>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, false, false, CombineLd<float>, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, true, true, StridedLd<float>, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, true, false, StridedLd<float>, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, false, false, StridedLd<float>, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<double, false, false, CombineLd<double>>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<double, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<double, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<double, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, true, true, StridedLd<float>, false, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, true, false, StridedLd<float>, false, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, false, false, StridedLd<float>, false, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<double, true, true, StridedLd<double>, false, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<double, true, false, StridedLd<double>, false, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<double, false, false, StridedLd<double>, false, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<float, false, false, CombineLd<float>, false, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_reg<double, false, false, CombineLd<double>, false, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_combine<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_combine<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_sections<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_sections<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_leaf<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_leaf<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  allow_dyn_smem(tc::k_tc_rowgemm<TcS2M>, lim);
  allow_dyn_smem(tc::k_tc_rowgemm<TcM2M>, lim);
  allow_dyn_smem(tc::k_tc_rowgemm<TcM2L>, lim);
  allow_dyn_smem(tc::k_tc_rowgemm<TcLeaf>, lim);
  allow_dyn_smem(tc::k_tc_nbr<TcLeafNb>, lim);
  allow_dyn_smem(tc::k_tc_rowgemm16<TcS2M>, lim);
  allow_dyn_smem(tc::k_tc_rowgemm16<TcM2M>, lim);
  allow_dyn_smem(tc::k_tc_rowgemm16<TcM2L>, lim);
  allow_dyn_smem(tc::k_tc_rowgemm16<TcLeaf>, lim);
  allow_dyn_smem(tc::k_tc_ws<TcS2M>, lim);
  allow_dyn_smem(tc::k_tc_ws<TcM2M>, lim);
  allow_dyn_smem(tc::k_tc_ws<TcM2L>, lim);
  allow_dyn_smem(tc::k_tc_ws<TcLeaf>, lim);
  allow_dyn_smem(tc::k_tc_ws<TcS2M, true>, lim);
  allow_dyn_smem(tc::k_tc_ws<TcM2M, true>, lim);
  allow_dyn_smem(tc::k_tc_ws<TcM2L, true>, lim);
  allow_dyn_smem(tc::k_tc_ws<TcLeaf, true>, lim);
  if (dev < FMMK_MAXDEV) done[dev] = 1;
  return 0;
}

extern "C" int fmmk_device_ok(char *err, size_t errlen) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    snprintf(err, errlen, "no CUDA device: %s", cudaGetErrorString(e));
    return 4;
  }
  int dev = 0, major = 0, minor = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  if (major != 10 || minor != 0) {
    snprintf(err, errlen, "device is sm_%d%d; this library is built for sm_100a only", major, minor);
    return 4;
  }
  return 0;
}

extern "C" int fmmk_create(const fmm_ops64 *ops, int precision, fmmk_state **out,
                           size_t *device_bytes, char *err, size_t errlen) {
  return fmmk_create_n(ops, precision, 1, out, device_bytes, err, errlen);
}

extern "C" int fmmk_create_n(const fmm_ops64 *ops, int precision, int nb, fmmk_state **out,
                             size_t *device_bytes, char *err, size_t errlen) {
  if (nb < 1 || nb > FMMK_MAX_BATCH) {
    snprintf(err, errlen, "batch capacity %d outside 1..%d", nb, FMMK_MAX_BATCH);
    return 1;
  }
  int rc = fmmk_device_ok(err, errlen);
  if (rc) return rc;
  set_smem_limits();
  fmmk_state *st = (fmmk_state *)calloc(1, sizeof(fmmk_state));
  if (!st) return 2;
  st->precision = precision;
  if (precision == 0) {
    Dev<double> *d = NULL;
    rc = dev_create<double>(ops, precision, nb, &d, err, errlen);
    st->dev = d;
    if (!rc && device_bytes) *device_bytes = d->bytes;
  } else {
    Dev<float> *d = NULL;
    rc = dev_create<float>(ops, precision, nb, &d, err, errlen);
    st->dev = d;
    if (!rc && device_bytes) *device_bytes = d->bytes;
    const char *ev = getenv("FMMFFT_AUTOTUNE");
    if (!rc && !(ev && atoi(ev) == 0)) {
      rc = dev_autotune<float>(d, err, errlen);
      if (rc) dev_release(d);
    }
  }
  if (rc) {
    free(st);
    return rc;
  }
  *out = st;
  return 0;
}

/* Device bytes a plan of this shape, precision and batch capacity holds, without allocating. */
extern "C" int fmmk_plan_bytes(long M, long P, long T, long b, int precision, int nb, size_t *bytes,
                               char *err, size_t errlen) {
  fmm_ops64 o;
  memset(&o, 0, sizeof o);
  o.M = M, o.P = P, o.T = T, o.b = b, o.s = M / b;
  o.n = 0;
  while ((1L << (o.n + 1)) <= o.s) ++o.n;
  if (precision == 0) {
    Dev<double> *d = NULL;
    return dev_create<double>(&o, precision, nb, &d, err, errlen, bytes);
  }
  Dev<float> *d = NULL;
  return dev_create<float>(&o, precision, nb, &d, err, errlen, bytes);
}

extern "C" void fmmk_destroy(fmmk_state *st) {
  if (!st) return;
  if (st->refine) {
    fmmk_destroy(st->refine->f64);
    cudaFree(st->refine->a);
    free(st->refine);
  }
  for (int i = 0; i < FMMK_GRAPHS; ++i)
    if (st->graphs[i].exec) cudaGraphExecDestroy(st->graphs[i].exec);
  host_pipe_free(st->pipe);
  if (st->precision == 0) {
    Dev<double> *d = (Dev<double> *)st->dev;
    dev_release(d);
  } else {
    Dev<float> *d = (Dev<float> *)st->dev;
    dev_release(d);
  }
  free(st);
}

extern "C" int fmmk_execute_n(fmmk_state *st, const void *d_in, void *d_out, void *stream,
                              int inverse, int nbt, char *err, size_t errlen) {
  cudaStream_t s = (cudaStream_t)stream;
  if (st->precision == 0)
    return dev_execute<double>((Dev<double> *)st->dev, d_in, d_out, s, inverse, nbt, err, errlen);
  return dev_execute<float>((Dev<float> *)st->dev, d_in, d_out, s, inverse, nbt, err, errlen);
}

extern "C" int fmmk_execute_ptrs(fmmk_state *st, int nbt, const void *const *ins, void *const *outs,
                                 void *stream, char *err, size_t errlen) {
  cudaStream_t s = (cudaStream_t)stream;
  if (nbt > kMaxIo) {
    snprintf(err, errlen, "execute of %d transforms: a pointer table holds at most %d", nbt, kMaxIo);
    return 1;
  }
  if (st->precision == 0)
    return dev_execute<double>((Dev<double> *)st->dev, ins[0], outs[0], s, 0, nbt, err, errlen, ins, outs);
  return dev_execute<float>((Dev<float> *)st->dev, ins[0], outs[0], s, 0, nbt, err, errlen, ins, outs);
}

extern "C" int fmmk_execute(fmmk_state *st, const void *d_in, void *d_out, void *stream,
                            int inverse, char *err, size_t errlen) {
  return fmmk_execute_n(st, d_in, d_out, stream, inverse, 1, err, errlen);
}

extern "C" int fmmk_execute_host(fmmk_state *st, const void *h_in, void *h_out, void *stream,
                                 char *err, size_t errlen) {
  cudaStream_t s = (cudaStream_t)stream;
  long N;
  size_t esz;
  void *work;
  if (st->precision == 0) {
    Dev<double> *d = (Dev<double> *)st->dev;
    N = d->N, esz = sizeof(double2), work = d->z;
  } else {
    Dev<float> *d = (Dev<float> *)st->dev;
    N = d->N, esz = sizeof(float2), work = d->z;
  }
  /* the input is staged into the plan's z buffer ([P][M] complex, dead until the combine) and
   * the transform runs in place on that copy; the result is copied back from it */
  FMM_CUDA_TRY(cudaMemcpyAsync(work, h_in, esz * (size_t)N, cudaMemcpyHostToDevice, s));
  /* in-place execute on the staged copy: stage 1 consumes z before z is rewritten */
  int rc = fmmk_execute(st, work, work, stream, 0, err, errlen);
  if (rc) return rc;
  FMM_CUDA_TRY(cudaMemcpyAsync(h_out, work, esz * (size_t)N, cudaMemcpyDeviceToHost, s));
  FMM_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

/* n transforms of host arrays h_in[i] -> h_out[i] (each N complex), pipelined: transform i is
 * copied into staging buffer i mod 3 on the copy-in stream, executed in place there on `stream`
 * and copied back on the copy-out stream, so that with pinned host memory the three overlap
 * across consecutive transforms (PCIe carries both directions at once).  The buffers (3 N
 * complex on the device) and the two copy streams are made on the first call and kept with the
 * plan.  Each transform's bits are those of fmmk_execute.  Returns when every output is in host
 * memory, with `stream` ordered after the last copy-out. */
extern "C" int fmmk_execute_host_many(fmmk_state *st, int n, const void *const *h_in, void *const *h_out,
                                      void *stream, char *err, size_t errlen) {
  cudaStream_t s = (cudaStream_t)stream;
  const long N = st->precision == 0 ? ((Dev<double> *)st->dev)->N : ((Dev<float> *)st->dev)->N;
  const size_t bytes = (st->precision == 0 ? sizeof(double2) : sizeof(float2)) * (size_t)N;
  if (!st->pipe) {
    HostPipe *hp = (HostPipe *)calloc(1, sizeof(HostPipe));
    if (!hp) return 2;
    cudaError_t e = cudaStreamCreateWithFlags(&hp->cin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&hp->cout, cudaStreamNonBlocking);
    for (int i = 0; i < FMMK_HOST_SLOTS && e == cudaSuccess; ++i) {
      e = cudaMalloc(&hp->buf[i], bytes);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&hp->in_done[i], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&hp->ex_done[i], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&hp->out_done[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
      snprintf(err, errlen, "execute_host_many staging: %s", cudaGetErrorString(e));
      host_pipe_free(hp);
      cudaGetLastError();
      return e == cudaErrorMemoryAllocation ? 2 : 3;
    }
    st->pipe = hp;
  }
  HostPipe *hp = st->pipe;
  /* the caller's stream may hold work the staging buffers' last users are ordered after */
  FMM_CUDA_TRY(cudaEventRecord(hp->out_done[0], s));
  FMM_CUDA_TRY(cudaStreamWaitEvent(hp->cin, hp->out_done[0], 0));
  for (int i = 0; i < n; ++i) {
    const int k = i % FMMK_HOST_SLOTS;
    void *buf = hp->buf[k];
    if (i >= FMMK_HOST_SLOTS) /* buffer k's previous transform has been copied out */
      FMM_CUDA_TRY(cudaStreamWaitEvent(hp->cin, hp->out_done[k], 0));
    FMM_CUDA_TRY(cudaMemcpyAsync(buf, h_in[i], bytes, cudaMemcpyHostToDevice, hp->cin));
    FMM_CUDA_TRY(cudaEventRecord(hp->in_done[k], hp->cin));
    FMM_CUDA_TRY(cudaStreamWaitEvent(s, hp->in_done[k], 0));
    int rc = fmmk_execute(st, buf, buf, stream, 0, err, errlen);
    if (rc) {
      cudaStreamSynchronize(hp->cin);
      cudaStreamSynchronize(hp->cout);
      return rc;
    }
    FMM_CUDA_TRY(cudaEventRecord(hp->ex_done[k], s));
    FMM_CUDA_TRY(cudaStreamWaitEvent(hp->cout, hp->ex_done[k], 0));
    FMM_CUDA_TRY(cudaMemcpyAsync(h_out[i], buf, bytes, cudaMemcpyDeviceToHost, hp->cout));
    FMM_CUDA_TRY(cudaEventRecord(hp->out_done[k], hp->cout));
  }
  /* the caller's stream ends after the last copy-out */
  if (n > 0) FMM_CUDA_TRY(cudaStreamWaitEvent(s, hp->out_done[(n - 1) % FMMK_HOST_SLOTS], 0));
  FMM_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

/* Block-distributed input and output: block r (M complex values, rank r's lq-block `qr` in the
 * reference) at in[r] / out[r], device or host memory.  The blocks are gathered into the plan's
 * z buffer (dead until the combine), transformed in place there and scattered back; host
 * blocks synchronise the stream at the end. */
extern "C" int fmmk_execute_blocks(fmmk_state *st, const void *const *in, void *const *out, int host,
                                   void *stream, char *err, size_t errlen) {
  cudaStream_t s = (cudaStream_t)stream;
  long M, P;
  size_t esz;
  char *work;
  if (st->precision == 0) {
    Dev<double> *d = (Dev<double> *)st->dev;
    M = d->M, P = d->P, esz = sizeof(double2), work = (char *)d->z;
  } else {
    Dev<float> *d = (Dev<float> *)st->dev;
    M = d->M, P = d->P, esz = sizeof(float2), work = (char *)d->z;
  }
  const size_t blk = esz * (size_t)M;
  const cudaMemcpyKind kin = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  const cudaMemcpyKind kout = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  for (long r = 0; r < P; ++r) FMM_CUDA_TRY(cudaMemcpyAsync(work + r * blk, in[r], blk, kin, s));
  int rc = fmmk_execute(st, work, work, stream, 0, err, errlen);
  if (rc) return rc;
  for (long r = 0; r < P; ++r) FMM_CUDA_TRY(cudaMemcpyAsync(out[r], work + r * blk, blk, kout, s));
  if (host) FMM_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

template <typename R>
static int fetch(Dev<R> *d, double *u, double *z, double *phi, double *psi) {
  const long M = d->M, P = d->P, T = d->T, n = d->n, S1 = d->S1;
  cudaDeviceSynchronize();
  auto grab = [](const void *src, size_t count, double *dst) -> int {
    R *h = (R *)malloc(sizeof(R) * count);
    if (!h) return 2;
    if (cudaMemcpy(h, src, sizeof(R) * count, cudaMemcpyDeviceToHost) != cudaSuccess) {
      free(h);
      return 3;
    }
    for (size_t i = 0; i < count; ++i) dst[i] = (double)h[i];
    free(h);
    return 0;
  };
  int rc = 0;
  /* the first transform of the last execute: its planes lead each level's block */
  if (u) rc |= grab(d->u, (size_t)(2 * S1 * M), u);
  if (z) rc |= grab(d->z, (size_t)(2 * P * M), z);
  const long S1e = (long)d->last_nbt * S1;
  for (long l = 2; l <= n; ++l) {
    const size_t cnt = (size_t)(2 * S1 * T * (1L << l));
    if (phi) rc |= grab(d->phi + lvl_off(l, S1e, T), cnt, phi + lvl_off(l, S1, T));
    if (psi) rc |= grab(d->psi + lvl_off(l, S1e, T), cnt, psi + lvl_off(l, S1, T));
  }
  return rc;
}

extern "C" int fmmk_debug_fetch(fmmk_state *st, double *u, double *z, double *phi, double *psi) {
  if (st->precision == 0) return fetch<double>((Dev<double> *)st->dev, u, z, phi, psi);
  return fetch<float>((Dev<float> *)st->dev, u, z, phi, psi);
}

/* ======================================================================== profiling */

template <typename R> static Prof *prof_of(fmmk_state *st) { return &((Dev<R> *)st->dev)->prof; }

extern "C" int fmmk_profile_start(fmmk_state *st, int cap) {
  Prof *pf = st->precision == 0 ? prof_of<double>(st) : prof_of<float>(st);
  if (pf->ev) return 1;
  if (cap < 1) cap = 1;
  pf->ev = (cudaEvent_t *)calloc((size_t)cap * (ST_COUNT + 1), sizeof(cudaEvent_t));
  if (!pf->ev) return 2;
  for (int i = 0; i < cap * (ST_COUNT + 1); ++i)
    if (cudaEventCreate(&pf->ev[i]) != cudaSuccess) return 3;
  pf->cap = cap, pf->count = 0, pf->on = 1;
  return 0;
}

/* Sums, over the executes recorded since start, the device time of each stage (ms) and reports
 * the kernel launches per execute of each stage; frees the events.  Returns the stage count. */
extern "C" int fmmk_profile_stop(fmmk_state *st, double *stage_ms, int *stage_launches, int cap,
                                 int *nexec) {
  Prof *pf = st->precision == 0 ? prof_of<double>(st) : prof_of<float>(st);
  if (!pf->ev) return -1;
  int n = cap < ST_COUNT ? cap : ST_COUNT;
  for (int k = 0; k < n; ++k) stage_ms[k] = 0, stage_launches[k] = pf->launches[k];
  if (pf->count > 0) cudaEventSynchronize(pf->ev[(pf->count - 1) * (ST_COUNT + 1) + ST_COUNT]);
  for (int e = 0; e < pf->count; ++e)
    for (int k = 0; k < n; ++k) {
      float ms = 0;
      cudaEventElapsedTime(&ms, pf->ev[e * (ST_COUNT + 1) + k], pf->ev[e * (ST_COUNT + 1) + k + 1]);
      stage_ms[k] += ms;
    }
  if (nexec) *nexec = pf->count;
  for (int i = 0; i < pf->cap * (ST_COUNT + 1); ++i) cudaEventDestroy(pf->ev[i]);
  free(pf->ev);
  pf->ev = NULL, pf->on = 0, pf->count = 0, pf->cap = 0;
  return ST_COUNT;
}

extern "C" const char *fmmk_stage_name(int i) { return (i >= 0 && i < ST_COUNT) ? kStageNames[i] : ""; }

/* ======================================================================== allocation-free entry */
/* fmmfft_execute_noalloc runs the complex64 FP32 transform with its operator tables and its
 * workspace in this file-scope device array instead of plan memory from cudaMalloc.  Every GPU
 * that loads the library holds the array until process exit.  Its device address is taken once
 * per device with cudaGetSymbolAddress (host code cannot use the symbol itself as a device
 * pointer).  Calls share the array: the tables of the last (N, P, terms, b) stay in it and are
 * reused, and two calls whose kernels overlap on the GPU race on it. */
#define FMMK_NOALLOC_BYTES ((size_t)32 << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[FMMK_NOALLOC_BYTES];

#define FMMK_NOALLOC_MAXDEV 64
#define FMMK_NOALLOC_STAGE_FLOATS ((size_t)2 << 20) /* host staging for the FP32 tables, 8 MiB */
static void *g_noalloc_base[FMMK_NOALLOC_MAXDEV];
static long g_noalloc_key[FMMK_NOALLOC_MAXDEV][4];
static float g_noalloc_stage[FMMK_NOALLOC_STAGE_FLOATS];

/* Operator and workspace layout inside the array: the same arrays, order and rounding as a
 * complex64 plan (dev_create), offsets relative to the array base. */
struct NoallocLayout {
  size_t initch, btop, bm2m, bm2l, evalmT, evalmh, cot, pretw, twP, twM, xt, part, ssum, phi, psi,
      u, z, tmp, sync, end;
};

static NoallocLayout noalloc_layout(const fmm_ops64 *o, long ntile) {
  const long M = o->M, P = o->P, T = o->T, b = o->b, n = o->n, S1 = P - 1;
  const long nlev = n - 2 > 0 ? n - 2 : 0;
  const long lvtot = 2 * S1 * T * ((2L << n) - 4);
  NoallocLayout L;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t at = off;
    off = align_up(off + bytes);
    return at;
  };
  L.initch = take(sizeof(float) * b * T);
  L.btop = take(sizeof(float) * T * T);
  L.bm2m = take(sizeof(float) * (nlev ? nlev : 1) * 2 * T * T);
  L.bm2l = take(sizeof(float) * (nlev ? nlev : 1) * 10 * T * T);
  L.evalmT = take(sizeof(float) * S1 * T * b);
  L.evalmh = take(sizeof(float) * S1 * T);
  L.cot = take(sizeof(float) * S1 * 4 * b);
  L.pretw = take(sizeof(float2) * P);
  L.twP = take(sizeof(float2) * P);
  L.twM = take(sizeof(float2) * M);
  L.xt = take(sizeof(float) * 2 * P * M);
  L.part = take(sizeof(float2) * ntile * P);
  L.ssum = take(sizeof(float2) * P);
  L.phi = take(sizeof(float) * lvtot);
  L.psi = take(sizeof(float) * lvtot);
  L.u = take(sizeof(float) * 2 * S1 * M);
  L.z = take(sizeof(float2) * P * M);
  L.tmp = take(sizeof(float2) * P * M);
  L.sync = take(64 * sizeof(unsigned));
  L.end = off;
  return L;
}

/* FP32 operator tables into g_noalloc_stage at the layout's offsets (same transposes and
 * stacking as dev_create). */
static void noalloc_stage_ops(const fmm_ops64 *o, const NoallocLayout &L) {
  const long M = o->M, P = o->P, T = o->T, b = o->b, n = o->n, S1 = P - 1;
  float *st = g_noalloc_stage;
  memset(st, 0, L.xt);
  float *f;
  f = st + L.initch / 4;
  for (long i = 0; i < b * T; ++i) f[i] = (float)o->initch[i];
  f = st + L.btop / 4;
  for (long k = 0; k < T; ++k)
    for (long t = 0; t < T; ++t) f[k * T + t] = (float)o->topflp[t * T + k];
  for (long Lv = 2; Lv <= n - 1; ++Lv) {
    const double *ops = o->levops + (Lv - 2) * FMM_NLEVOPS * T * T;
    f = st + L.bm2m / 4 + (Lv - 2) * 2 * T * T;
    for (long k = 0; k < T; ++k)
      for (long t = 0; t < T; ++t) {
        f[k * T + t] = (float)ops[FMM_SHFTFN * T * T + t * T + k];
        f[(T + k) * T + t] = (float)ops[FMM_SHFTFP * T * T + t * T + k];
      }
  }
  for (long l = 3; l <= n; ++l) {
    const double *ops = o->levops + (l - 3) * FMM_NLEVOPS * T * T;
    f = st + L.bm2l / 4 + (l - 3) * 10 * T * T;
    const long N2 = 2 * T;
    for (long k = 0; k < T; ++k)
      for (long t = 0; t < T; ++t) {
        f[(0 * T + k) * N2 + t] = (float)ops[FMM_SHFTLP * T * T + t * T + k];
        f[(0 * T + k) * N2 + T + t] = (float)ops[FMM_SHFTLN * T * T + t * T + k];
        f[(1 * T + k) * N2 + t] = (float)ops[FMM_FLIP2P * T * T + t * T + k];
        f[(1 * T + k) * N2 + T + t] = (float)ops[FMM_FLIP3P * T * T + t * T + k];
        f[(2 * T + k) * N2 + T + t] = (float)ops[FMM_FLIP2P * T * T + t * T + k];
        f[(3 * T + k) * N2 + t] = (float)ops[FMM_FLIP2N * T * T + t * T + k];
        f[(4 * T + k) * N2 + t] = (float)ops[FMM_FLIP3N * T * T + t * T + k];
        f[(4 * T + k) * N2 + T + t] = (float)ops[FMM_FLIP2N * T * T + t * T + k];
      }
  }
  f = st + L.evalmT / 4;
  for (long sc = 1; sc < P; ++sc)
    for (long k = 0; k < T; ++k)
      for (long j = 0; j < b; ++j) f[((sc - 1) * T + k) * b + j] = (float)o->evalm[(j * S1 + (sc - 1)) * T + k];
  f = st + L.evalmh / 4;
  for (long sc = P / 2; sc < P; ++sc)
    for (long k = 0; k < T; ++k) f[(sc - 1) * T + k] = (float)o->evalmh[(sc - P / 2) * T + k];
  f = st + L.cot / 4;
  for (long i = 0; i < S1 * 4 * b; ++i) f[i] = (float)o->cot[i];
  const double PI = 3.14159265358979323846264338327950288;
  f = st + L.pretw / 4;
  for (long sc = 1; sc < P; ++sc) {
    f[2 * sc] = (float)(-cos(PI * sc / P) * sin(PI * sc / P));
    f[2 * sc + 1] = (float)(sin(PI * sc / P) * sin(PI * sc / P));
  }
  f = st + L.twP / 4;
  for (long k = 0; k < P; ++k) f[2 * k] = (float)cos(2 * PI * k / P), f[2 * k + 1] = (float)-sin(2 * PI * k / P);
  f = st + L.twM / 4;
  for (long k = 0; k < M; ++k) {
    double a = 2 * PI * (double)k / (double)M;
    f[2 * k] = (float)cos(a), f[2 * k + 1] = (float)-sin(a);
  }
}

/* reuse_ops: the caller knows the tables in the array are for these parameters already. */
extern "C" int fmmk_execute_noalloc(const fmm_ops64 *o, int reuse_ops, const void *d_in,
                                    void *d_out, void *stream, char *err, size_t errlen) {
  int dev = 0;
  FMM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= FMMK_NOALLOC_MAXDEV) {
    snprintf(err, errlen, "device %d outside the %d devices the no-alloc entry tracks", dev,
             FMMK_NOALLOC_MAXDEV);
    return 1;
  }
  if (!g_noalloc_base[dev]) { /* set-up, once per device, with that device current */
    int rc = fmmk_device_ok(err, errlen);
    if (rc) return rc;
    void *p = NULL;
    FMM_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    set_smem_limits();
    g_noalloc_base[dev] = p;
  }
  Dev<float> d;
  memset((void *)&d, 0, sizeof(d));
  d.M = o->M, d.P = o->P, d.T = o->T, d.b = o->b, d.s = o->s, d.n = o->n;
  d.N = o->M * o->P, d.S1 = o->P - 1, d.precision = 1;
  d.fft_threads = 512;
  /* the same stage choices as an FMMFFT_F32 plan (dev_create), including its switches */
  d.fuse_s2m = 1;
  if (const char *ev = getenv("FMMFFT_FUSE_S2M")) d.fuse_s2m = atoi(ev) != 0;
  d.pdl = 1;
  if (const char *ev = getenv("FMMFFT_PDL")) d.pdl = atoi(ev) != 0;
  /* no cooperative coarse-tree kernel here: a timeout of its grid barrier could not be
   * reported by this entry point (sizes it serves never reach the coarse-tree threshold) */
  d.coarse_rows = 0;
  d.tileM = d.P >= 2048 ? 1 : 2048 / d.P;
  if (d.tileM > d.M) d.tileM = d.M;
  d.ntile = d.M / d.tileM;
  if (d.M <= 4096) {
    d.M1 = d.M, d.M2 = 1;
  } else {
    long lg = 0;
    while ((1L << lg) < d.M) ++lg;
    d.M2 = 1L << ((lg + 1) / 2);
    d.M1 = d.M / d.M2;
  }
  NoallocLayout L = noalloc_layout(o, d.ntile);
  if (L.end > FMMK_NOALLOC_BYTES || L.xt / sizeof(float) > FMMK_NOALLOC_STAGE_FLOATS) {
    snprintf(err, errlen,
             "N=%ld P=%ld terms=%ld b=%ld needs %zu bytes of device scratch; the allocation-free "
             "entry point holds at most %zu",
             d.N, d.P, d.T, d.b, L.end, (size_t)FMMK_NOALLOC_BYTES);
    return 1;
  }
  char *base = (char *)g_noalloc_base[dev];
  cudaStream_t st = (cudaStream_t)stream;
  const long key[4] = {o->M, o->P, o->T, o->b};
  int same = reuse_ops && memcmp(key, g_noalloc_key[dev], sizeof key) == 0;
  if (!same) {
    noalloc_stage_ops(o, L);
    FMM_CUDA_TRY(cudaMemcpyAsync(base, g_noalloc_stage, L.xt, cudaMemcpyHostToDevice, st));
    /* no workspace array is read before it is written; zeroing it anyway keeps a fresh
     * configuration independent of what an earlier one left behind */
    FMM_CUDA_TRY(cudaMemsetAsync(base + L.xt, 0, L.end - L.xt, st));
    FMM_CUDA_TRY(cudaStreamSynchronize(st)); /* the host staging array is reused next call */
    memcpy(g_noalloc_key[dev], key, sizeof key);
  }
  d.initch = (float *)(base + L.initch);
  d.btop = (float *)(base + L.btop);
  d.bm2m = (float *)(base + L.bm2m);
  d.bm2l = (float *)(base + L.bm2l);
  d.evalmT = (float *)(base + L.evalmT);
  d.evalmh = (float *)(base + L.evalmh);
  d.cot = (float *)(base + L.cot);
  d.pretw = (float2 *)(base + L.pretw);
  d.twP = (float2 *)(base + L.twP);
  d.twM = (float2 *)(base + L.twM);
  d.xt = (float *)(base + L.xt);
  d.part = (float2 *)(base + L.part);
  d.ssum = (float2 *)(base + L.ssum);
  d.phi = (float *)(base + L.phi);
  d.psi = (float *)(base + L.psi);
  d.u = (float *)(base + L.u);
  d.z = (float2 *)(base + L.z);
  d.tmp = (float2 *)(base + L.tmp);
  d.sync = (unsigned *)(base + L.sync);
  d.status = (int *)(d.sync + 48); /* the coarse-tree barrier records a timeout here */
  d.nbmax = 1;
  return dev_execute<float>(&d, d_in, d_out, st, 0, 1, err, errlen);
}

/* Runs k_selftest_wait against the plan's own status word with a limit of limit_us
 * microseconds, on the legacy stream, and waits for it.  fmmk_check then reports the timeout. */
extern "C" int fmmk_selftest_wait(fmmk_state *st, int which, long limit_us, char *err, size_t errlen) {
  (void)which;
  int *status = st->precision == 0 ? ((Dev<double> *)st->dev)->status : ((Dev<float> *)st->dev)->status;
  k_selftest_wait<<<1, 64>>>((unsigned long long)limit_us * 1000ull, status);
  FMM_CUDA_TRY(cudaGetLastError());
  FMM_CUDA_TRY(cudaDeviceSynchronize());
  return 0;
}

/* The plan's stage choices as text (for benchmark records). */
extern "C" int fmmk_describe(fmmk_state *st, char *buf, size_t len) {
  if (st->precision == 0) {
    Dev<double> *d = (Dev<double> *)st->dev;
    snprintf(buf, len, "fft_threads=%d coarse_rows=%ld fuse_s2m=%d tuned=0", d->fft_threads, d->coarse_rows,
             d->fuse_s2m);
  } else {
    Dev<float> *d = (Dev<float> *)st->dev;
    const char *form = d->tc_form == 0 ? "row" : d->tc_form == 3 ? "row16" : d->tc_form == 4 ? "ws" : "per_stage";
    snprintf(buf, len,
             "fft_threads=%d coarse_rows=%ld tc_min_rows=%ld fuse_s2m=%d tensor_cores=%s tc_form=%s "
             "leaf_form=%s tuned=%d",
             d->fft_threads, d->coarse_rows, d->tc_min_rows, d->fuse_s2m,
             d->tc ? (d->bf16 ? "bf16x3" : "tf32x3") : "none", form,
             !d->tc ? "cuda_cores" : (d->ok_lnb && d->tc_form < 0) ? "neighbour_sum" : d->ok_leaf ? "window_rows" : "cuda_cores",
             d->tuned);
  }
  return 0;
}

/* Reads (and clears) the plan's device status word; synchronises the device. */
extern "C" int fmmk_check(fmmk_state *st) {
  int *status = st->precision == 0 ? ((Dev<double> *)st->dev)->status : ((Dev<float> *)st->dev)->status;
  int h = 0;
  if (cudaDeviceSynchronize() != cudaSuccess) return 3;
  if (cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 3;
  if (h) cudaMemset(status, 0, sizeof(int));
  return h ? 6 : 0;
}

/* ======================================================================== FP64 residual correction */
/* One step of residual correction for complex64 plans (the forward transform F~ in FP32 or
 * split TF32): with y1 = F~ x, the residual r = x - F64^-1 y1 / N is formed in FP64 through the
 * FP64 plan of the same shape (the reference's arithmetic), and y = y1 + F~ r is accumulated in
 * FP64 (complex128 output).  Since r is of the size of F~'s rounding error, F~ r adds only its
 * relative error times that: the result moves from FP32-level agreement with the FP64 FMM
 * output to the square of it, bounded below by the FMM's own truncation at this order. */

__global__ void k_promote(const float2 *__restrict__ a, double2 *__restrict__ o, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    o[i] = make_double2((double)a[i].x, (double)a[i].y);
}

/* r = x - z / N in FP64, rounded once to complex64 */
__global__ void k_residual(const float2 *__restrict__ x, const double2 *__restrict__ z, float2 *__restrict__ r,
                           long n, double invN) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double2 v = z[i];
    r[i] = make_float2((float)((double)x[i].x - v.x * invN), (float)((double)x[i].y - v.y * invN));
  }
}

__global__ void k_accumulate(double2 *__restrict__ o, const float2 *__restrict__ c, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double2 v = o[i];
    o[i] = make_double2(v.x + (double)c[i].x, v.y + (double)c[i].y);
  }
}

/* Makes the FP64 companion plan and scratch of a complex64 plan (once). */
extern "C" int fmmk_refine_enable(fmmk_state *st, const fmm_ops64 *ops, size_t *bytes, char *err, size_t errlen) {
  if (st->precision == 0) {
    snprintf(err, errlen, "residual correction applies to complex64 plans");
    return 1;
  }
  if (st->refine) {
    if (bytes) *bytes = st->refine->bytes;
    return 0;
  }
  Refine *r = (Refine *)calloc(1, sizeof(Refine));
  if (!r) return 2;
  size_t b64 = 0;
  int rc = fmmk_create(ops, 0, &r->f64, &b64, err, errlen);
  if (rc) {
    free(r);
    return rc;
  }
  const long N = ((Dev<float> *)st->dev)->N;
  char *base = NULL;
  const size_t need = align_up(sizeof(float2) * N) * 2 + align_up(sizeof(double2) * N);
  if (cudaMalloc((void **)&base, need) != cudaSuccess) {
    fmmk_destroy(r->f64);
    free(r);
    snprintf(err, errlen, "cudaMalloc(%zu) for the residual pass failed", need);
    return 2;
  }
  r->a = (float2 *)base;
  r->c = (float2 *)(base + align_up(sizeof(float2) * N));
  r->bq = (double2 *)(base + 2 * align_up(sizeof(float2) * N));
  r->bytes = b64 + need;
  st->refine = r;
  if (bytes) *bytes = r->bytes;
  return 0;
}

/* d_in: N complex64, d_out: N complex128 (not overlapping d_in). */
extern "C" int fmmk_execute_refined(fmmk_state *st, const void *d_in, void *d_out, void *stream, char *err,
                                    size_t errlen) {
  Refine *r = st->refine;
  if (!r) {
    snprintf(err, errlen, "residual correction was not enabled on this plan");
    return 1;
  }
  const long N = ((Dev<float> *)st->dev)->N;
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const unsigned grid = (unsigned)(4 * nsm);
  double2 *out = (double2 *)d_out;
  int rc = fmmk_execute(st, d_in, r->a, stream, 0, err, errlen); /* y1 = F~ x */
  if (rc) return rc;
  k_promote<<<grid, 256, 0, s>>>(r->a, out, N);                     /* out = y1 */
  rc = fmmk_execute(r->f64, out, r->bq, stream, 1, err, errlen);      /* bq = N F64^-1 y1 */
  if (rc) return rc;
  k_residual<<<grid, 256, 0, s>>>((const float2 *)d_in, r->bq, r->a, N, 1.0 / (double)N);
  rc = fmmk_execute(st, r->a, r->c, stream, 0, err, errlen);          /* c = F~ r */
  if (rc) return rc;
  k_accumulate<<<grid, 256, 0, s>>>(out, r->c, N);                  /* out = y1 + F~ r */
  FMM_CUDA_TRY(cudaGetLastError());
  return 0;
}

/* ======================================================================== CUDA graphs */

/* Execute through a cached graph: the first call for a given (in, out, direction) captures the
 * plan's launch sequence on a private stream and instantiates it; later calls launch the graph
 * on `stream`.  The least recently used of FMMK_GRAPHS graphs is replaced when full. */
extern "C" int fmmk_execute_graph(fmmk_state *st, const void *d_in, void *d_out, void *stream,
                                  int inverse, char *err, size_t errlen) {
  return fmmk_execute_graph_n(st, d_in, d_out, stream, inverse, 1, err, errlen);
}

extern "C" int fmmk_execute_graph_n(fmmk_state *st, const void *d_in, void *d_out, void *stream,
                                    int inverse, int nbt, char *err, size_t errlen) {
  GraphSlot *hit = NULL, *victim = &st->graphs[0];
  for (int i = 0; i < FMMK_GRAPHS; ++i) {
    GraphSlot *g = &st->graphs[i];
    if (g->exec && g->in == d_in && g->out == d_out && g->inverse == inverse && g->nbt == nbt) hit = g;
    if (!g->exec || (victim->exec && g->last_use < victim->last_use)) victim = g;
  }
  if (!hit) {
    cudaStream_t cap;
    FMM_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      cudaStreamDestroy(cap);
      snprintf(err, errlen, "cudaStreamBeginCapture: %s", cudaGetErrorString(e));
      return 3;
    }
    int rc = fmmk_execute_n(st, d_in, d_out, cap, inverse, nbt, err, errlen);
    cudaGraph_t graph = NULL;
    e = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(cap);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) {
      snprintf(err, errlen, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
      return 3;
    }
    cudaGraphExec_t exec = NULL;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      snprintf(err, errlen, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
      return 3;
    }
    if (victim->exec) cudaGraphExecDestroy(victim->exec);
    victim->in = d_in, victim->out = d_out, victim->inverse = inverse, victim->nbt = nbt, victim->exec = exec;
    hit = victim;
  }
  hit->last_use = ++st->graph_clock;
  FMM_CUDA_TRY(cudaGraphLaunch(hit->exec, (cudaStream_t)stream));
  return 0;
}

/* ======================================================================== batches */

/* Captures n executes into one graph (execute i carries counts[i] transforms of its plan, 1 when
 * counts is NULL): a fork from the capturing stream into nbranch streams, execute i enqueued on
 * branch[i] (all transforms of one plan must share a branch:
 * they share its workspace), and a join.  One cudaGraphLaunch then runs the whole batch, the
 * branches overlapping on the device. */
extern "C" int fmmk_batch_capture(fmmk_state *const *sts, const void *const *ins, void *const *outs,
                                  const int *inverse, const int *counts, const int *branch, int n,
                                  int nbranch, void **exec_out, char *err, size_t errlen) {
  cudaStream_t root;
  FMM_CUDA_TRY(cudaStreamCreateWithFlags(&root, cudaStreamNonBlocking));
  cudaStream_t *br = (cudaStream_t *)calloc((size_t)nbranch, sizeof(cudaStream_t));
  cudaEvent_t *ev = (cudaEvent_t *)calloc((size_t)nbranch + 1, sizeof(cudaEvent_t));
  if (!br || !ev) return 2;
  int rc = 0;
  for (int i = 0; i < nbranch && !rc; ++i)
    if (cudaStreamCreateWithFlags(&br[i], cudaStreamNonBlocking) != cudaSuccess) rc = 3;
  for (int i = 0; i <= nbranch && !rc; ++i)
    if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) rc = 3;
  cudaGraph_t graph = NULL;
  if (!rc && cudaStreamBeginCapture(root, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = 3;
  if (!rc) {
    cudaEventRecord(ev[nbranch], root);
    for (int b = 0; b < nbranch; ++b) cudaStreamWaitEvent(br[b], ev[nbranch], 0);
    for (int i = 0; i < n && !rc; ++i)
      rc = fmmk_execute_n(sts[i], ins[i], outs[i], br[branch[i]], inverse ? inverse[i] : 0,
                          counts ? counts[i] : 1, err, errlen);
    for (int b = 0; b < nbranch; ++b) {
      cudaEventRecord(ev[b], br[b]);
      cudaStreamWaitEvent(root, ev[b], 0);
    }
    cudaError_t e = cudaStreamEndCapture(root, &graph);
    if (!rc && e != cudaSuccess) {
      snprintf(err, errlen, "batch capture: %s", cudaGetErrorString(e));
      rc = 3;
    }
  }
  if (!rc) {
    cudaGraphExec_t exec = NULL;
    cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
      snprintf(err, errlen, "batch instantiate: %s", cudaGetErrorString(e));
      rc = 3;
    } else {
      *exec_out = (void *)exec;
    }
  }
  if (graph) cudaGraphDestroy(graph);
  for (int i = 0; i <= nbranch; ++i)
    if (ev[i]) cudaEventDestroy(ev[i]);
  for (int i = 0; i < nbranch; ++i)
    if (br[i]) cudaStreamDestroy(br[i]);
  cudaStreamDestroy(root);
  free(br), free(ev);
  return rc;
}

extern "C" int fmmk_batch_launch(void *exec, void *stream) {
  return cudaGraphLaunch((cudaGraphExec_t)exec, (cudaStream_t)stream) == cudaSuccess ? 0 : 3;
}
extern "C" void fmmk_batch_free(void *exec) {
  if (exec) cudaGraphExecDestroy((cudaGraphExec_t)exec);
}

/* ======================================================================== plain size-N FFT */

/* A conventional FFT of the whole N-vector on the GPU, the same register Stockham passes as the
 * FMM-FFT's size-M FFTs: one pass (N <= 4096), a 4-step of two passes (N <= 2^21) or a 4-step
 * whose second factor is itself a 4-step (three passes, N <= 2^30).  It stands where the
 * reference's plain FFTW comparators stand (src/fftw_serial.c:53-58, src/fftw_mpi.c:54-58):
 * FMM-FFT against an ordinary FFT of the same length on the same machine.  Forward,
 * unnormalised, out of place (in != out). */
struct fmmk_fft {
  long N;
  int dbl;
  int npass;
  FftPass pass[3];
  long per[3], rows[3];
  int tin[3], tout[3];
  int src[3], dst[3]; /* 0 in, 1 out, 2 tmp */
  void *tmp, *twD, *twP;
  size_t bytes;
};

static FftPass plain_pass(int L, long per, long irow, long iseq, long istr, long orow, long oseq,
                          long ostr, int post, unsigned twmul, long N) {
  FftPass f{};
  f.L = L;
  int W = 512 / (L / 8);
  if (W > 16) W = 16;
  if (W > per) W = (int)per;
  if (W < 1) W = 1;
  f.W = W, f.per = (int)per, f.M = N;
  f.irow = irow, f.iseq = iseq, f.istr = istr;
  f.orow = orow, f.oseq = oseq, f.ostr = ostr;
  f.twiddle_post = post, f.tws = 4096 / L, f.conj_out = 0;
  f.twmul = twmul, f.twmask = (unsigned)(N - 1), f.twbits = N > 4096 ? 12 : 0;
  return f;
}

extern "C" int fmmk_fft_create(long N, int dbl, fmmk_fft **out, size_t *device_bytes, char *err,
                               size_t errlen) {
  int rc = fmmk_device_ok(err, errlen);
  if (rc) return rc;
  int lg = 0;
  while (lg < 62 && (1L << lg) < N) ++lg;
  if (N < 16 || (1L << lg) != N || lg > 30) {
    snprintf(err, errlen, "plain FFT length %ld: a power of two in [16, 2^30] is required", N);
    return 1;
  }
  set_smem_limits();
  fmmk_fft *f = (fmmk_fft *)calloc(1, sizeof(fmmk_fft));
  if (!f) return 2;
  f->N = N, f->dbl = dbl;
  if (lg <= 12) {
    f->npass = 1;
    f->pass[0] = plain_pass((int)N, 1, N, N, 1, N, N, 1, 0, 1, N);
    f->per[0] = 1, f->rows[0] = 1, f->tin[0] = 1, f->tout[0] = 1, f->src[0] = 0, f->dst[0] = 1;
  } else if (lg <= 21) {
    int a = lg / 2 > 9 ? 9 : lg / 2;
    if (a < lg - 12) a = lg - 12;
    const long N2 = 1L << a, N1 = N / N2;
    f->npass = 2;
    /* for each n1: DFT over n2 (stride N1), times exp(-2 pi i n1 k2 / N) -> tmp[k2 N1 + n1] */
    f->pass[0] = plain_pass((int)N2, N1, 0, 1, N1, 0, 1, N1, 1, 1, N);
    f->per[0] = N1, f->rows[0] = 1, f->tin[0] = 0, f->tout[0] = 0, f->src[0] = 0, f->dst[0] = 2;
    /* for each k2: DFT over n1 (contiguous) -> out[k2 + N2 k1] */
    f->pass[1] = plain_pass((int)N1, N2, 0, N1, 1, 0, 1, N2, 0, 1, N);
    f->per[1] = N2, f->rows[1] = 1, f->tin[1] = 1, f->tout[1] = 0, f->src[1] = 2, f->dst[1] = 1;
  } else {
    const int a = lg / 3 > 9 ? 9 : lg / 3;
    const int rest = lg - a;
    const int bb = rest / 2 > 9 ? 9 : rest / 2;
    const long N2 = 1L << a, N1 = N / N2, B = 1L << bb, A = N1 / B;
    f->npass = 3;
    /* pass 1 as in the two-pass case, into out (used as scratch) */
    f->pass[0] = plain_pass((int)N2, N1, 0, 1, N1, 0, 1, N1, 1, 1, N);
    f->per[0] = N1, f->rows[0] = 1, f->tin[0] = 0, f->tout[0] = 0, f->src[0] = 0, f->dst[0] = 1;
    /* row k2 (length N1, n1 = a + A b): for each a, DFT over b (stride A), times
     * exp(-2 pi i a kb / N1) = exp(-2 pi i a kb N2 / N) -> tmp[k2 N1 + kb A + a] */
    f->pass[1] = plain_pass((int)B, A, N1, 1, A, N1, 1, A, 1, (unsigned)N2, N);
    f->per[1] = A, f->rows[1] = N2, f->tin[1] = 0, f->tout[1] = 0, f->src[1] = 1, f->dst[1] = 2;
    /* for each (k2, kb): DFT over a (contiguous) -> out[k2 + N2 (kb + B ka)] */
    f->pass[2] = plain_pass((int)A, B, N1, A, 1, 1, N2, N2 * B, 0, 1, N);
    f->per[2] = B, f->rows[2] = N2, f->tin[2] = 1, f->tout[2] = 0, f->src[2] = 2, f->dst[2] = 1;
  }
  const size_t esz = dbl ? 16 : 8;
  const long nlo = N > 4096 ? 4096 : N, nP = N > 4096 ? 4096 + N / 4096 : N;
  const size_t bt = align_up(esz * (size_t)N), bD = align_up(esz * 4096), bP = align_up(esz * (size_t)nP);
  char *base = NULL;
  if (cudaMalloc((void **)&base, bt + bD + bP) != cudaSuccess) {
    free(f);
    snprintf(err, errlen, "cudaMalloc of %zu bytes failed", bt + bD + bP);
    return 2;
  }
  f->tmp = base, f->twD = base + bt, f->twP = base + bt + bD;
  f->bytes = bt + bD + bP;
  double *h = (double *)malloc(sizeof(double) * 2 * (size_t)(nP > 4096 ? nP : 4096));
  if (!h) {
    cudaFree(base), free(f);
    return 2;
  }
  const double PI = 3.14159265358979323846264338327950288;
  for (long t = 0; t < 4096; ++t) h[2 * t] = cos(2 * PI * t / 4096), h[2 * t + 1] = -sin(2 * PI * t / 4096);
  if (dbl) rc = upload<double>((double **)&f->twD, h, 2 * 4096, err, errlen);
  else rc = upload<float>((float **)&f->twD, h, 2 * 4096, err, errlen);
  for (long t = 0; t < nlo; ++t) h[2 * t] = cos(2 * PI * t / N), h[2 * t + 1] = -sin(2 * PI * t / N);
  for (long t = 0; t < nP - nlo; ++t) {
    const double ang = 2 * PI * (double)(t * nlo) / (double)N;
    h[2 * (nlo + t)] = cos(ang), h[2 * (nlo + t) + 1] = -sin(ang);
  }
  if (!rc) {
    if (dbl) rc = upload<double>((double **)&f->twP, h, 2 * nP, err, errlen);
    else rc = upload<float>((float **)&f->twP, h, 2 * nP, err, errlen);
  }
  free(h);
  if (rc) {
    cudaFree(base), free(f);
    return rc;
  }
  if (device_bytes) *device_bytes = f->bytes;
  *out = f;
  return 0;
}

template <typename R>
static int fft_run(fmmk_fft *f, const void *in, void *out, cudaStream_t st, char *err, size_t errlen) {
  using C = typename cplx<R>::T;
  const C *twD = (const C *)f->twD, *twP = (const C *)f->twP;
  for (int k = 0; k < f->npass; ++k) {
    const FftPass &fp = f->pass[k];
    const C *src = (const C *)(f->src[k] == 0 ? in : (f->src[k] == 1 ? out : f->tmp));
    C *dst = (C *)(f->dst[k] == 1 ? out : f->tmp);
    const int thr = fp.W * (fp.L / 8);
    const size_t sm = sizeof(C) * fft_smem_elems(fp.L, fp.W);
    dim3 g((unsigned)(f->per[k] / fp.W), (unsigned)f->rows[k]);
    const StridedLd<R> sld{src, fp.irow, fp.iseq, (unsigned)fp.istr};
    if (f->tin[k] && f->tout[k])
      k_fft_reg<R, true, true><<<g, thr, sm, st>>>(sld, dst, twD, twP, fp);
    else if (f->tin[k])
      k_fft_reg<R, true, false><<<g, thr, sm, st>>>(sld, dst, twD, twP, fp);
    else
      k_fft_reg<R, false, false><<<g, thr, sm, st>>>(sld, dst, twD, twP, fp);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(err, errlen, "plain FFT launch: %s", cudaGetErrorString(e));
    return 3;
  }
  return 0;
}

extern "C" int fmmk_fft_execute(fmmk_fft *f, const void *in, void *out, void *stream, char *err,
                                size_t errlen) {
  if (in == out) {
    snprintf(err, errlen, "the plain FFT is out of place: input and output must differ");
    return 1;
  }
  cudaStream_t st = (cudaStream_t)stream;
  return f->dbl ? fft_run<double>(f, in, out, st, err, errlen) : fft_run<float>(f, in, out, st, err, errlen);
}

extern "C" size_t fmmk_fft_bytes(const fmmk_fft *f) { return f->bytes; }

extern "C" void fmmk_fft_destroy(fmmk_fft *f) {
  if (!f) return;
  cudaFree(f->tmp);
  free(f);
}

/* ======================================================================== sharded transform */
/* One transform of N = P M points split over G shards (one per GPU in a multi-GPU job), each
 * holding the contiguous block y[g N/G .. (g+1) N/G) of input and output, as the reference's
 * ranks do (src/fmmfft.c:384-978): shard g owns the leaf boxes [g s/G, (g+1) s/G) of every
 * section.  Its plan is an ordinary single-device plan over an EXTENDED strip of s_ext = 2 s/G
 * boxes, its own boxes with H = s/(2G) boxes of halo on either side, built from the operators of
 * the GLOBAL tree (level l of the strip is level l + log2(G/2) of the transform; the leaf and
 * near-field tables are the transform's).  Every box of the strip has its own multipole
 * expansions; the coarse levels come from the other shards: the expansions of the strip's level
 * 3 (global level lc = log2(4G), four own boxes per plane and shard) are all-gathered, each shard
 * runs the global tree above lc on them (a small plan of 2^lc boxes) and takes the local
 * expansions of its strip's 8 level-3 boxes from it.  Below that the strip's own M2L is exact for
 * its own boxes and the box before them, since their interaction lists (2 to 3 boxes away at
 * every level >= 4) stay inside the strip; so are the leaf's fields.  The combine runs over the
 * shard's own columns (all P sections of them are local) into P rows of M/G, one all-to-all
 * gives each shard its P/G rows whole, and a plan of P/G sections of M points runs their FFTs.
 * Exchanges, in order: the halos of x (each shard receives the last N/(2G) points of the shard
 * before it and the first N/(2G) of the one after it), an all-reduce of the P section sums, an
 * all-gather of the coarse expansions, one all-to-all of the combined rows.  The stage kernels
 * are the single-device ones (the reference's halo exchanges per level, :517-618, are replaced
 * by the strip's halo boxes, computed redundantly). */

template <typename R> struct ShardImpl {
  using C = typename cplx<R>::T;
  int G, g, precision;
  long N, P, T, b, M, s, n, lc;
  long s_loc, H, s_ext, n_ext, M_ext, M_loc;
  Dev<R> *loc = nullptr, *crs = nullptr, *fft = nullptr;
  void *mem = nullptr;
  C *x_ext, *sums, *z_send, *z_recv, *y;
  R *phi_send, *phi_all;
  long phi_elems;
};

/* The level-3 expansions of a strip's own boxes (local boxes 2..5 of 8 per plane) into the send
 * buffer, [plane][4][T] */
template <typename R>
__global__ void k_shard_pack(const R *__restrict__ lvl3, R *__restrict__ out, long planes, int T) {
  const long total = planes * 4 * T;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long t = e % T, j = (e / T) % 4, pl = e / (4L * T);
    out[e] = lvl3[(pl * 8 + 2 + j) * T + t];
  }
}
/* The gathered expansions [shard][plane][4][T] into the global level lc, [plane][4G][T] */
template <typename R>
__global__ void k_shard_unpack(const R *__restrict__ all, R *__restrict__ lvl, long planes, int T, int G) {
  const long total = (long)G * planes * 4 * T;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long t = e % T, j = (e / T) % 4, pl = (e / (4L * T)) % planes, gg = e / (4L * T * planes);
    lvl[(pl * 4 * G + 4 * gg + j) * T + t] = all[e];
  }
}
/* The local expansions of the strip's 8 level-3 boxes from the global level lc: strip box k is
 * global box (4 g - 2 + k) mod 4G */
template <typename R>
__global__ void k_shard_inject(const R *__restrict__ glvl, R *__restrict__ lvl3, long planes, int T, int G,
                               int g) {
  const long total = planes * 8 * T;
  const long nb = 4L * G;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long t = e % T, k = (e / T) % 8, pl = e / (8L * T);
    const long gb = ((4L * g - 2 + k) % nb + nb) % nb;
    lvl3[e] = glvl[(pl * nb + gb) * T + t];
  }
}

template <typename R>
static void shard_free(ShardImpl<R> *sh) {
  if (!sh) return;
  Dev<R> *ds[3] = {sh->loc, sh->crs, sh->fft};
  for (Dev<R> *d : ds) dev_release(d);
  cudaFree(sh->mem);
  delete sh;
}

template <typename R>
static int shard_create(const fmm_ops64 *og, int precision, int G, int g, ShardImpl<R> **out, char *err,
                        size_t errlen) {
  using C = typename cplx<R>::T;
  const long M = og->M, P = og->P, T = og->T, b = og->b, s = og->s, n = og->n;
  auto lg2 = [](long v) { long l = 0; while ((1L << l) < v) ++l; return l; };
  if (G < 2 || (G & (G - 1)) || g < 0 || g >= G) {
    snprintf(err, errlen, "shard %d of %d: G must be a power of two >= 2 and 0 <= g < G", g, G);
    return 1;
  }
  const long s_loc = s / G, H = s_loc / 2, s_ext = 2 * s_loc, M_loc = M / G;
  const long tileM = P >= 2048 ? 1 : 2048 / P;
  const int Wc = (int)(512 / (P / 8) > 32 ? 32 : 512 / (P / 8));
  if (P < 16 || P % (2L * G) != 0 || s % G != 0 || s_loc < 8 || (H * b) % tileM != 0 || M_loc % tileM != 0 ||
      M_loc % Wc != 0) {
    snprintf(err, errlen,
             "sharded transform of N = %ld, P = %ld, b = %ld over %d shards: needs P >= 16, P a multiple "
             "of 2G and at least 8 leaf boxes per shard", M * P, P, b, G);
    return 1;
  }
  ShardImpl<R> *sh = new (std::nothrow) ShardImpl<R>();
  if (!sh) return 2;
  sh->G = G, sh->g = g, sh->precision = precision;
  sh->N = M * P, sh->P = P, sh->T = T, sh->b = b, sh->M = M, sh->s = s, sh->n = n;
  sh->s_loc = s_loc, sh->H = H, sh->s_ext = s_ext, sh->n_ext = lg2(s_ext), sh->lc = lg2(4L * G);
  sh->M_ext = s_ext * b, sh->M_loc = M_loc;
  /* the strip: the transform's operators, its levels offset by n - n_ext */
  fmm_ops64 ol = *og;
  ol.M = sh->M_ext, ol.s = s_ext, ol.n = sh->n_ext;
  ol.levops = og->levops + (n - sh->n_ext) * FMM_NLEVOPS * T * T;
  /* the coarse tree: the transform's levels 2..lc as a tree of 4G leaf boxes */
  fmm_ops64 oc = *og;
  oc.s = 4L * G, oc.M = oc.s * b, oc.n = sh->lc;
  /* the shard's rows: P/G sections of M points (only its FFT stage runs) */
  fmm_ops64 of = *og;
  of.P = P / G;
  int rc = dev_create<R>(&ol, precision, 1, &sh->loc, err, errlen);
  if (!rc) rc = dev_create<R>(&oc, precision, 1, &sh->crs, err, errlen);
  if (!rc) rc = dev_create<R>(&of, precision, 1, &sh->fft, err, errlen);
  if (rc) {
    shard_free(sh);
    return rc;
  }
  const long S1 = P - 1, Next = sh->M_ext * P;
  sh->phi_elems = 2 * S1 * 4 * T;
  size_t off = 0;
  auto carve = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes); return o; };
  const size_t o_x = carve(sizeof(C) * Next), o_s = carve(sizeof(C) * P), o_ps = carve(sizeof(R) * sh->phi_elems),
               o_pa = carve(sizeof(R) * sh->phi_elems * G), o_zs = carve(sizeof(C) * (sh->N / G)),
               o_zr = carve(sizeof(C) * (sh->N / G)), o_y = carve(sizeof(C) * (sh->N / G));
  cudaError_t ce = cudaMalloc(&sh->mem, off);
  if (ce != cudaSuccess) {
    snprintf(err, errlen, "cudaMalloc(%zu): %s", off, cudaGetErrorString(ce));
    shard_free(sh);
    return 2;
  }
  char *base = (char *)sh->mem;
  sh->x_ext = (C *)(base + o_x), sh->sums = (C *)(base + o_s), sh->phi_send = (R *)(base + o_ps);
  sh->phi_all = (R *)(base + o_pa), sh->z_send = (C *)(base + o_zs), sh->z_recv = (C *)(base + o_zr);
  sh->y = (C *)(base + o_y);
  *out = sh;
  return 0;
}

/* Phase 0: the strip's sections, its own section sums, S2M and M2M up to its level 3, whose own
 * expansions go to phi_send.  Phase 1 (after the sums were all-reduced and the expansions
 * all-gathered): the coarse tree, the strip's M2L from level 4, the leaf and the combine of its own
 * columns into z_send.  Phase 2 (after the all-to-all into z_recv): the P/G rows' FFTs into y. */
template <typename R>
static int shard_phase(ShardImpl<R> *sh, int phase, cudaStream_t st, char *err, size_t errlen) {
  using C = typename cplx<R>::T;
  const long P = sh->P, T = sh->T, S1 = P - 1, G = sh->G;
  const int blocks = 4 * sh->loc->num_sms;
  int rc = 0;
  if (phase == 0) {
    ExecCtl c{};
    c.mask = (1u << ST_SECTIONS) | (1u << ST_SUMS) | (1u << ST_S2M) | (1u << ST_M2M);
    c.m2m_stop = 3, c.no_coarse = 1;
    c.sum_t0 = sh->H * sh->b / sh->loc->tileM, c.sum_nt = sh->M_loc / sh->loc->tileM, c.sum_out = sh->sums;
    rc = dev_execute<R>(sh->loc, sh->x_ext, sh->y, st, 0, 1, err, errlen, nullptr, nullptr, &c);
    if (!rc)
      k_shard_pack<R><<<blocks, 256, 0, st>>>(sh->loc->phi + lvl_off(3, S1, T), sh->phi_send, 2 * S1, (int)T);
  } else if (phase == 1) {
    FMM_CUDA_TRY(cudaMemcpyAsync(sh->loc->ssum, sh->sums, sizeof(C) * P, cudaMemcpyDeviceToDevice, st));
    k_shard_unpack<R><<<blocks, 256, 0, st>>>(sh->phi_all, sh->crs->phi + lvl_off(sh->lc, S1, T), 2 * S1,
                                              (int)T, (int)G);
    ExecCtl cc{};
    cc.mask = (1u << ST_M2M) | (1u << ST_TOP) | (1u << ST_M2L);
    rc = dev_execute<R>(sh->crs, sh->x_ext, sh->y, st, 0, 1, err, errlen, nullptr, nullptr, &cc);
    if (rc) return rc;
    k_shard_inject<R><<<blocks, 256, 0, st>>>(sh->crs->psi + lvl_off(sh->lc, S1, T),
                                              sh->loc->psi + lvl_off(3, S1, T), 2 * S1, (int)T, (int)G, sh->g);
    ExecCtl c{};
    c.mask = (1u << ST_M2L) | (1u << ST_LEAF) | (1u << ST_COMBINE);
    c.m2l_from = 4, c.no_coarse = 1;
    c.comb_m0 = sh->H * sh->b, c.comb_cols = sh->M_loc, c.comb_ostride = sh->M_loc, c.comb_out = sh->z_send;
    c.comb_invM = 1.0 / (double)sh->M;
    rc = dev_execute<R>(sh->loc, sh->x_ext, sh->y, st, 0, 1, err, errlen, nullptr, nullptr, &c);
  } else if (phase == 2) {
    const long rows = P / G, M = sh->M, Ml = sh->M_loc;
    for (long gg = 0; gg < G; ++gg) /* chunk gg: rows x columns [gg M/G, (gg+1) M/G) */
      FMM_CUDA_TRY(cudaMemcpy2DAsync(sh->fft->z + gg * Ml, sizeof(C) * M, sh->z_recv + gg * rows * Ml,
                                     sizeof(C) * Ml, sizeof(C) * Ml, rows, cudaMemcpyDeviceToDevice, st));
    ExecCtl c{};
    c.mask = 1u << ST_FFT1;
    rc = dev_execute<R>(sh->fft, sh->y, sh->y, st, 0, 1, err, errlen, nullptr, nullptr, &c);
    if (!rc && sizeof(R) == 4 && T >= 10) /* the block-DC bins of the shard's rows, as a plan's */
      k_block_dc<R><<<dim3((unsigned)((rows + 3) / 4), 1), 128, 0, st>>>(sh->sums, sh->y, M, (int)P, 0, OutTab{},
                                                                         (int)(sh->g * rows), (int)rows);
  } else {
    snprintf(err, errlen, "shard phase %d: 0, 1 or 2", phase);
    return 1;
  }
  if (!rc) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      snprintf(err, errlen, "shard phase %d: %s", phase, cudaGetErrorString(e));
      return 3;
    }
  }
  return rc;
}

struct fmmk_shard {
  int precision;
  void *impl;
};

extern "C" int fmmk_shard_create(const fmm_ops64 *o, int precision, int G, int g, fmmk_shard **out, char *err,
                                 size_t errlen) {
  int rc = fmmk_device_ok(err, errlen);
  if (rc) return rc;
  set_smem_limits();
  fmmk_shard *sh = (fmmk_shard *)calloc(1, sizeof(fmmk_shard));
  if (!sh) return 2;
  sh->precision = precision;
  if (precision == 0) {
    ShardImpl<double> *p = nullptr;
    rc = shard_create<double>(o, precision, G, g, &p, err, errlen);
    sh->impl = p;
  } else {
    ShardImpl<float> *p = nullptr;
    rc = shard_create<float>(o, precision, G, g, &p, err, errlen);
    sh->impl = p;
  }
  if (rc) {
    free(sh);
    return rc;
  }
  *out = sh;
  return 0;
}

extern "C" void fmmk_shard_destroy(fmmk_shard *sh) {
  if (!sh) return;
  if (sh->precision == 0) shard_free((ShardImpl<double> *)sh->impl);
  else shard_free((ShardImpl<float> *)sh->impl);
  free(sh);
}

template <typename R> static void shard_bufs(ShardImpl<R> *p, void **ptr, size_t *cnt) {
  ptr[0] = p->x_ext, ptr[1] = p->sums, ptr[2] = p->phi_send, ptr[3] = p->phi_all, ptr[4] = p->z_send;
  ptr[5] = p->z_recv, ptr[6] = p->y;
  cnt[0] = (size_t)(p->M_ext * p->P), cnt[1] = (size_t)(p->H * p->b * p->P), cnt[2] = (size_t)p->phi_elems;
  cnt[3] = (size_t)(p->N / p->G), cnt[4] = (size_t)(p->N / p->G);
}

extern "C" void fmmk_shard_buffers(fmmk_shard *sh, void **ptr, size_t *cnt) {
  if (sh->precision == 0) shard_bufs((ShardImpl<double> *)sh->impl, ptr, cnt);
  else shard_bufs((ShardImpl<float> *)sh->impl, ptr, cnt);
}

extern "C" int fmmk_shard_phase(fmmk_shard *sh, int phase, void *stream, char *err, size_t errlen) {
  cudaStream_t st = (cudaStream_t)stream;
  if (sh->precision == 0) return shard_phase((ShardImpl<double> *)sh->impl, phase, st, err, errlen);
  return shard_phase((ShardImpl<float> *)sh->impl, phase, st, err, errlen);
}
