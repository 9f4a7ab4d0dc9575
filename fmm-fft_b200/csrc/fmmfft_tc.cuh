/*
 * tcgen05 (5th-generation tensor core) form of the FMM tree contractions, sm_100a.
 *
 * Every tree stage is D[r][0..N) = sum_k A(r, k) B[k][0..N) over many rows r (section, re/im
 * plane, box) with a small shared operator B (see fmmfft_kernels.cu).  This kernel runs that
 * contraction on the tensor cores in 3xTF32: each FP32 operand is split into a TF32 "hi" part
 * (round to nearest) and the TF32-rounded residual "lo", and D = A_hi B_hi + A_hi B_lo +
 * A_lo B_hi is accumulated in FP32 in tensor memory (TMEM).  The dropped A_lo B_lo term and the
 * rounding of the residuals leave about 2^-22 relative error per product.
 *
 * Per CTA (256 threads, two CTAs per SM, persistent over 128-row tiles), per K slice of up to
 * 64 columns:
 *   1. every thread loads its part of one tile row from HBM into registers, splits it into TF32
 *      hi and lo, and writes both into the row's TMEM lane (tcgen05.st);
 *   2. one thread issues 3 * slice/8 tcgen05.mma (M = 128, N = Npad, K = 8; A from TMEM, B from
 *      shared memory in the canonical K-major no-swizzle layout) into one TMEM accumulator and
 *      commits them to an mbarrier;
 * then every warp reads its 32 TMEM lanes (= its 32 rows) with tcgen05.ld and stores them.
 * B (hi/lo, pre-split on the host) is staged once per CTA, or once per section for the leaf.
 * Waits on the mbarrier are bounded; on expiry the CTA records an error code and leaves.
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tc {

constexpr int kRows = 128;         /* MMA M, rows per tile */
constexpr long kWaitLimit = 1L << 26; /* try_wait polls before a wait is declared failed */

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

/* K-major, no-swizzle shared-memory matrix descriptor (tcgen05 "matrix descriptor"):
 * start address, leading byte offset (next core matrix along K), stride byte offset (next
 * group of 8 rows), version 1, swizzle mode 0. */
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

/* Instruction descriptor, kind::tf32: D = F32, A = B = TF32, both K-major, M = 128. */
__host__ __device__ constexpr uint32_t make_idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0),
        "r"(0)
      : "memory");
}

/* A from tensor memory (lane = row, one 32-bit column per K element), B from shared memory. */
__device__ __forceinline__ void mma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(d_tmem), "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0),
        "r"(0)
      : "memory");
}

/* 8 consecutive 32-bit TMEM columns of this thread's lane from registers. */
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float *v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
      :
      : "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
      : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  for (long i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_smem_to_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :
               : "r"(smem_addr(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(taddr), "r"(ncols)
               : "memory");
}

/* 8 consecutive 32-bit TMEM columns of this thread's lane. */
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tf32_rna(float a) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return __uint_as_float(r);
}

/* Byte offset of element (row m, column k) in a K-major no-swizzle tile whose K extent is
 * kpad floats: 8-row groups of kpad/4 core matrices, each core matrix 8 rows x 16 bytes. */
__device__ __forceinline__ uint32_t core_off(int m, int k, int kpad) {
  return (uint32_t)((m >> 3) * (kpad * 32) + (k >> 2) * 128 + (m & 7) * 16 + (k & 3) * 4);
}

/* Error codes a CTA records in the plan's device status word. */
enum { kErrWaitTimeout = 1 };

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" : : "r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

constexpr int kSlice = 64; /* K columns of A staged per step */

/* Shared memory the kernel needs for a given padded K and N: B hi and lo. */
__host__ __device__ constexpr size_t smem_bytes(int kpad, int npad) {
  return (size_t)(2 * npad * kpad) * sizeof(float);
}
/* Tensor-memory columns of one CTA: the accumulator (npad, rounded up to 32) plus A hi and A lo
 * of one K slice, as a power of two. */
__host__ __device__ constexpr int tmem_cols(int kpad, int npad) {
  int need = ((npad + 31) / 32) * 32 + 2 * (kpad < kSlice ? kpad : kSlice);
  return need <= 32 ? 32 : need <= 64 ? 64 : need <= 128 ? 128 : need <= 256 ? 256 : 512;
}

/* Generic persistent tcgen05 row contraction.  Prob supplies:
 *   long rows;  int batches;          rows per batch, number of batches
 *   int nchunks; int clen[4]; int coff[4];   A chunk lengths / K offsets (multiples of 4)
 *   int kpad, npad, nout;             padded K (multiple of 8), padded N (x16), stored columns
 *   const float *bhi, *blo; long bstride;   pre-split B, [npad][kpad] per batch
 *   __device__ const float *src(int c, long r, int batch) const;
 *   __device__ float *dst(long r, int batch) const;
 * A never touches shared memory: warp w, lane i owns tile row 32 (w % 4) + i (its TMEM lane)
 * and K columns [32 (w / 4), +32) of each 64-column slice; it loads them (8 float4, all issued
 * before use), splits them into TF32 hi/lo in registers and writes both into its TMEM lane with
 * tcgen05.st.  The MMAs then read A from TMEM and only B (staged once) from shared memory.  The
 * loads of step i+1 are issued before the CTA waits for step i's MMAs.  Two CTAs per SM. */
template <class Prob>
__global__ void __launch_bounds__(256, 2) k_tc_rowgemm(const __grid_constant__ Prob pb, int *status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  /* load map: for slice s, column half h and float4 i, the A chunk (low byte, 0xFF = zero)
   * and the float offset within that chunk's row (high bits) */
  __shared__ int lmap[4][2][8];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kpad = pb.kpad, npad = pb.npad;
  const int ks = kpad < kSlice ? kpad : kSlice;
  const int nslices = (kpad + ks - 1) / ks; /* <= 4: kpad <= 256 */
  float *Bhi = reinterpret_cast<float *>(smem_raw);
  float *Blo = Bhi + npad * kpad;
  const uint32_t ncols = (uint32_t)tmem_cols(kpad, npad);
  if (warp == 0) tmem_alloc(&tmem_slot, ncols);
  if (tid == 0) {
    mbar_init(&mbar, 1);
    fence_mbar_init();
    abort_flag = 0;
  }
  if (tid < 4 * 2 * 8) {
    const int sl = tid >> 4, h = (tid >> 3) & 1, i = tid & 7;
    const int k0 = sl * ks, k = k0 + h * 32 + 4 * i;
    int e = 0xFF;
    if (sl < nslices && h * 32 + 4 * i < ks && k < kpad)
      for (int c = 0; c < pb.nchunks; ++c)
        if (k >= pb.coff[c] && k < pb.coff[c] + pb.clen[c]) e = c | ((k - pb.coff[c]) << 8);
    lmap[sl][h][i] = e;
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t d_cols = (uint32_t)(((npad + 31) / 32) * 32);
  const uint32_t t_ahi = tmem + d_cols, t_alo = tmem + d_cols + (uint32_t)ks;
  const uint32_t idesc = make_idesc_tf32(npad);
  const uint32_t b_sbo = (uint32_t)kpad * 32, lbo = 128;
  const uint32_t bh = smem_addr(Bhi), bl = smem_addr(Blo);
  const int tiles_per_batch = (int)((pb.rows + kRows - 1) / kRows);
  const int ntiles = tiles_per_batch * pb.batches;
  const int quarter = warp & 3, my_half = warp >> 2;
  const int my_m = quarter * 32 + lane;
  const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;

  float4 v[8];
  const float *rowp[4];
  auto load_step = [&](int tile, int slice) {
    if (slice == 0) {
      const int batch = tile / tiles_per_batch;
      const long r = (long)(tile - batch * tiles_per_batch) * kRows + my_m;
      const bool live = r < pb.rows;
#pragma unroll
      for (int c = 0; c < 4; ++c) rowp[c] = (live && c < pb.nchunks) ? pb.src(c, r, batch) : nullptr;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int e = lmap[slice][my_half][i];
      const int c = e & 0xFF;
      v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (c != 0xFF) {
        const float *rp = c == 0 ? rowp[0] : (c == 1 ? rowp[1] : (c == 2 ? rowp[2] : rowp[3]));
        if (rp) v[i] = __ldg(reinterpret_cast<const float4 *>(rp + (e >> 8)));
      }
    }
  };

  int cur_batch = -1;
  uint32_t phase = 0;
  int tile = blockIdx.x, slice = 0;
  if (tile < ntiles) load_step(tile, 0);
  while (tile < ntiles) {
    const int batch = tile / tiles_per_batch;
    const long r0 = (long)(tile - batch * tiles_per_batch) * kRows;
    const int k0 = slice * ks, k1 = k0 + ks;
    if (batch != cur_batch) { /* B of this batch; the previous step's MMAs have completed */
      const float *gbh = pb.bhi + (long)batch * pb.bstride, *gbl = pb.blo + (long)batch * pb.bstride;
      for (int e = tid; e < npad * kpad; e += blockDim.x) {
        int n = e / kpad, k = e - n * kpad;
        uint32_t o = core_off(n, k, kpad) >> 2;
        Bhi[o] = gbh[e];
        Blo[o] = gbl[e];
      }
      fence_smem_to_async();
      cur_batch = batch;
    }
    /* split into TF32 hi / lo and write both into this thread's TMEM lane */
    if (my_half * 32 < ks) {
      float h[32], l[32];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float a[4] = {v[i].x, v[i].y, v[i].z, v[i].w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          h[4 * i + j] = tf32_rna(a[j]);
          l[4 * i + j] = tf32_rna(a[j] - h[4 * i + j]);
        }
      }
      const uint32_t col = (uint32_t)(my_half * 32);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (my_half * 32 + 8 * q >= ks) break;
        tmem_st8(t_ahi + lane_addr + col + 8 * q, h + 8 * q);
        tmem_st8(t_alo + lane_addr + col + 8 * q, l + 8 * q);
      }
    }
    tmem_st_wait();
    fence_before_sync();
    __syncthreads();
    if (warp == 0) { /* lane 0 issues; the rest of warp 0 waits at __syncwarp */
      if (lane == 0) {
        fence_after_sync();
        /* the last slice may extend past kpad: only its real K steps are issued */
        const int ksteps = ((k1 < kpad ? k1 : kpad) - k0) >> 3, kb = k0 >> 3;
#pragma unroll 1
        for (int s = 0; s < 3; ++s) {
          uint32_t ta = (s == 2) ? t_alo : t_ahi;
          /* a K step of 8 TF32 is 256 bytes of B = 16 units of the descriptor's address */
          uint64_t db = make_desc(((s == 1) ? bl : bh) + 256u * kb, lbo, b_sbo);
#pragma unroll 1
          for (int kk = 0; kk < ksteps; ++kk, ta += 8, db += 16)
            mma_tf32_ts(tmem, ta, db, idesc, (k0 | s | kk) != 0);
        }
        mma_commit(&mbar);
      }
      __syncwarp();
    }
    /* next step: its loads go out while the MMAs (and at a tile's end the epilogue) run */
    const bool last_slice = slice == nslices - 1;
    const int ntile = last_slice ? tile + (int)gridDim.x : tile;
    const int nslice = last_slice ? 0 : slice + 1;
    if (ntile < ntiles) load_step(ntile, nslice);
    /* one thread polls the mbarrier; the other warps wait at the CTA barrier */
    if (tid == 0 && !mbar_wait_bounded(&mbar, phase)) {
      atomicExch(status, kErrWaitTimeout);
      abort_flag = 1;
    }
    phase ^= 1;
    __syncthreads();
    fence_after_sync();
    if (abort_flag) break;
    if (last_slice) {
      /* epilogue: this warp's TMEM lanes (= tile rows), columns of half (w / 4) of padded N */
      const long r = r0 + my_m;
      float *dst = (r < pb.rows) ? pb.dst(r, batch) : nullptr;
      const int cw = npad >> 1, cbeg = my_half * cw;
      for (int c0 = cbeg; c0 < cbeg + cw; c0 += 8) {
        float t[8];
        tmem_ld8(tmem + lane_addr + (uint32_t)c0, t);
        if (dst) {
          if (c0 + 8 <= pb.nout) {
            *reinterpret_cast<float4 *>(dst + c0) = make_float4(t[0], t[1], t[2], t[3]);
            *reinterpret_cast<float4 *>(dst + c0 + 4) = make_float4(t[4], t[5], t[6], t[7]);
          } else if (c0 + 4 <= pb.nout) {
            *reinterpret_cast<float4 *>(dst + c0) = make_float4(t[0], t[1], t[2], t[3]);
          }
        }
      }
      fence_before_sync();
      __syncthreads();
    }
    tile = ntile, slice = nslice;
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

}  // namespace tc
