/*
 * tcgen05 (5th-generation tensor core) kernels of the FMM tree and leaf contractions, sm_100a.
 *
 * Every tree stage is D[r][0..N) = sum_k A(r, k) B[k][0..N) over many rows r (section, re/im
 * plane, box) with a small shared operator B (see fmmfft_kernels.cu).  The kernels run that
 * contraction on the tensor cores with each FP32 operand split into a hi part and the rounding of
 * the remainder lo, products accumulated in FP32 in tensor memory (TMEM):
 *
 *   k_tc_rowgemm    row form: A loaded by every thread into registers, split into TF32 hi / lo,
 *                   written into the row's TMEM lane (tcgen05.st); one thread issues the MMAs
 *                   (A from TMEM, B from shared memory), four products (4xTF32); two CTAs per
 *                   SM, persistent over 128-row tiles, 64-column K steps;
 *   k_tc_rowgemm16  the same with the 16x256b TMEM shape (K and N permuted within 16-column
 *                   groups, so a thread moves four consecutive columns with one float4);
 *   k_tc_ws         warp-specialised: producer warps copy A through a shared-memory ring into
 *                   TMEM slots, one thread issues the MMAs (three products), epilogue warps drain
 *                   two accumulators; split TF32 or BF16x3 (the only kernel for BF16x3).
 *
 * The autotuner picks among them per plan shape.  Every mbarrier wait is bounded; on expiry the
 * CTA records an error code, stops and frees its tensor memory.
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tc {

constexpr int kRows = 128;         /* MMA M, rows per tile */

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

/* 16 TMEM lanes x 16 columns from registers (shape 16x256b, two 8-column chunks): thread t
 * writes lanes t/4 and t/4 + 8 at columns 2 (t % 4) and 2 (t % 4) + 1 of each chunk, registers
 * {lane t/4: chunk 0 two columns, lane t/4 + 8: chunk 0, lane t/4: chunk 1, lane t/4 + 8: chunk 1}.
 * The lane field of taddr is the first of the 16 lanes (0 or 16 within the warp's quarter). */
__device__ __forceinline__ void tmem_st16x2(uint32_t taddr, const float *v) {
  asm volatile(
      "tcgen05.st.sync.aligned.16x256b.x2.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
      :
      : "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
      : "memory");
}

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

/* Waits for phase `parity` of `bar` for at most about 2 s (global timer). */
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  unsigned long long t0 = 0;
  for (unsigned it = 0;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 1023) == 1023) {
      unsigned long long now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      if (t0 == 0) t0 = now;
      else if (now - t0 > 2000000000ull) return false;
    }
  }
}

/* Arrives on `bar` and adds `bytes` to the transaction count its current phase waits for. */
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;"
               :
               : "r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
/* Bulk copy (no tensor map) of `bytes` from global memory into this CTA's shared memory,
 * completing on `bar`: both addresses 16-byte aligned, bytes a multiple of 16. */
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :
      : "r"(dst), "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
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

/* 8 consecutive 32-bit TMEM columns of this thread's lane, issued without waiting: the
 * registers hold the values only after tmem_ld_wait(), and reg_fence8 (after the wait) makes
 * every later use of them depend on it. */
__device__ __forceinline__ void tmem_ld8_issue(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void reg_fence8(uint32_t (&r)[8]) {
  asm volatile("" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]));
}

/* 16 lanes x 16 columns (shape 16x256b), issued without waiting (see tmem_ld8_issue). */
__device__ __forceinline__ void tmem_ld16x2_issue(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.16x256b.x2.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr)
      : "memory");
}

/* The same 16 lanes x 16 columns into registers (same register order as tmem_st16x2). */
__device__ __forceinline__ void tmem_ld16x2(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.16x256b.x2.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

/* a rounded to TF32 (10 explicit mantissa bits), to nearest with ties away from zero, as FP32
 * bits with the low 13 bits clear: half a TF32 ulp added to the magnitude bits, then the 13
 * bits dropped (the carry moves into the exponent exactly as IEEE rounding does).  Two
 * integer-pipe instructions instead of a conversion; finite inputs only. */
__device__ __forceinline__ float tf32_rna(float a) {
  return __uint_as_float((__float_as_uint(a) + 0x1000u) & 0xFFFFE000u);
}

/* Byte offset of element (row m, column k) in a K-major no-swizzle tile whose K extent is
 * kpad floats: 8-row groups of kpad/4 core matrices, each core matrix 8 rows x 16 bytes. */
__host__ __device__ __forceinline__ uint32_t core_off(int m, int k, int kpad) {
  return (uint32_t)((m >> 3) * (kpad * 32) + (k >> 2) * 128 + (m & 7) * 16 + (k & 3) * 4);
}

/* Programmatic dependent launch: a kernel launched with programmatic stream serialisation may
 * start while the kernel before it in the stream still runs; griddepcontrol.wait blocks until
 * that kernel has completed and its memory is visible (without the attribute it returns at
 * once), and launch_dependents lets the next such kernel start once every CTA of this one has
 * issued it. */
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

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
  int need = ((2 * npad + 31) / 32) * 32 + 2 * (kpad < kSlice ? kpad : kSlice);
  return need <= 32 ? 32 : need <= 64 ? 64 : need <= 128 ? 128 : need <= 256 ? 256 : 512;
}

/* Generic persistent tcgen05 row contraction.  Prob supplies:
 *   long rows;  int batches;          rows per batch, number of batches
 *   int nchunks; int clen[4]; int coff[4];   A chunk lengths / K offsets (multiples of 4)
 *   int kpad, npad, nout;             padded K (multiple of 8), padded N (x16), stored columns
 *   const float *bimg; long bimg_stride;   B of batch z split into TF32 hi / lo as the kernel's
 *                                     shared-memory image (hi rows then lo rows, core matrices
 *                                     with K extent kpad) at bimg + z bimg_stride
 *   __device__ const float *src(int c, long r, int batch) const;
 *   __device__ float *dst(long r, int batch) const;
 *   __device__ void put8(float *dst, long r, int batch, int c0, const float *t) const;
 *                                     stores output columns c0..c0+7 of row r
 *   static constexpr bool kEpiAlternate;  epilogue chunks dealt alternately to the two halves
 * A never touches shared memory: warp w, lane i owns tile row 32 (w % 4) + i (its TMEM lane)
 * and K columns [32 (w / 4), +32) of each 64-column slice; it loads them (8 float4, all issued
 * before use), splits them into TF32 hi/lo in registers and writes both into its TMEM lane with
 * tcgen05.st.  The MMAs then read A from TMEM and only B (staged once) from shared memory.  The
 * loads of step i+1 are issued before the CTA waits for step i's MMAs.  Two CTAs per SM. */
template <class Prob>
__global__ void __launch_bounds__(256, 2) k_tc_rowgemm(const __grid_constant__ Prob pb, int *status) {
  /* 8 warps: 4 TMEM lane quarters x NS column halves; a thread moves CW columns of a slice */
  constexpr int NS = 2, CW = kSlice / NS, NF = CW / 4;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ uint64_t mbar, bbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  /* load map: for slice s, column group h and float4 i, the A chunk (low byte, 0xFF = zero)
   * and the float offset within that chunk's row (high bits) */
  __shared__ int lmap[4][NS][NF];
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
    mbar_init(&bbar, 1);
    fence_mbar_init();
    abort_flag = 0;
  }
  if (tid < 4 * NS * NF) {
    const int sl = tid / (NS * NF), h = (tid / NF) % NS, i = tid % NF;
    const int k0 = sl * ks, k = k0 + h * CW + 4 * i;
    int e = 0xFF;
    if (sl < nslices && h * CW + 4 * i < ks && k < kpad)
      for (int c = 0; c < pb.nchunks; ++c)
        if (k >= pb.coff[c] && k < pb.coff[c] + pb.clen[c]) e = c | ((k - pb.coff[c]) << 8);
    lmap[sl][h][i] = e;
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;
  /* accumulator columns [0, npad): A x B_hi, [npad, 2 npad): A x B_lo (B_lo follows B_hi in
   * shared memory as the next row groups, so one descriptor of N = 2 npad covers both) */
  const uint32_t d_cols = (uint32_t)(((2 * npad + 31) / 32) * 32);
  const uint32_t t_ahi = tmem + d_cols, t_alo = tmem + d_cols + (uint32_t)ks;
  const uint32_t idesc = make_idesc_tf32(2 * npad);
  const uint32_t b_sbo = (uint32_t)kpad * 32, lbo = 128;
  const uint32_t bh = smem_addr(Bhi), bl = smem_addr(Blo);
  const int tiles_per_batch = (int)((pb.rows + kRows - 1) / kRows);
  const int ntiles = tiles_per_batch * pb.batches;
  const int quarter = warp & 3, my_half = warp >> 2;
  const int my_m = quarter * 32 + lane;
  const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;

  float4 v[NF];
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
    for (int i = 0; i < NF; ++i) {
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
  /* one operator per batch: a CTA takes a contiguous run of tiles, so that it stages a new B
   * once or twice rather than at almost every tile; one batch: tiles strided by the grid */
  const bool runs = pb.batches > 1;
  const int tile_end = runs ? (int)(((long)ntiles * (blockIdx.x + 1)) / gridDim.x) : ntiles;
  const int tile_step = runs ? 1 : (int)gridDim.x;
  /* B of a batch: its shared-memory image, one bulk copy issued by thread 0 (the MMA issuer,
   * who waits for it before the next MMAs); the MMAs reading the previous one have completed */
  uint32_t bphase = 0;
  bool b_pending = false;
  const uint32_t b_bytes = (uint32_t)(smem_bytes(kpad, npad));
  auto stage_b = [&](int batch) {
    if (tid == 0) {
      mbar_expect_tx(&bbar, b_bytes);
      bulk_g2s(smem_addr(smem_raw), pb.bimg + (long)batch * pb.bimg_stride, b_bytes, &bbar);
      b_pending = true;
    }
    cur_batch = batch;
  };
  int tile = runs ? (int)(((long)ntiles * blockIdx.x) / gridDim.x) : (int)blockIdx.x, slice = 0;
  /* the operators are plan constants: the first one is staged before waiting for the kernel
   * this one depends on (its rows are this kernel's A); nothing global is read or written
   * before the wait */
  pdl_trigger();
  if (tile < tile_end) stage_b(tile / tiles_per_batch);
  pdl_wait();
  if (tile < tile_end) load_step(tile, 0);
  while (tile < tile_end) {
    const int batch = tile / tiles_per_batch;
    const long r0 = (long)(tile - batch * tiles_per_batch) * kRows;
    const int k0 = slice * ks, k1 = k0 + ks;
    if (batch != cur_batch) stage_b(batch); /* the previous step's MMAs have completed */
    /* split into TF32 hi / lo and write both into this thread's TMEM lane, 8 columns at a time */
    if (my_half * CW < ks) {
      const uint32_t col = (uint32_t)(my_half * CW);
#pragma unroll
      for (int q = 0; q < CW / 8; ++q) {
        if (my_half * CW + 8 * q >= ks) break;
        float h[8], l[8];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const float a[4] = {v[2 * q + i].x, v[2 * q + i].y, v[2 * q + i].z, v[2 * q + i].w};
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            h[4 * i + j] = tf32_rna(a[j]);
            l[4 * i + j] = tf32_rna(a[j] - h[4 * i + j]);
          }
        }
        tmem_st8(t_ahi + lane_addr + col + 8 * q, h);
        tmem_st8(t_alo + lane_addr + col + 8 * q, l);
      }
    }
    tmem_st_wait();
    fence_before_sync();
    __syncthreads();
    if (warp == 0) { /* lane 0 issues; the rest of warp 0 waits at __syncwarp */
      if (lane == 0) {
        fence_after_sync();
        bool b_ok = true;
        if (b_pending) { /* the operator image has landed */
          b_ok = mbar_wait_bounded(&bbar, bphase);
          bphase ^= 1, b_pending = !b_ok;
          if (!b_ok) atomicExch(status, kErrWaitTimeout), abort_flag = 1;
        }
        /* the last slice may extend past kpad: only its real K steps are issued */
        const int ksteps = b_ok ? ((k1 < kpad ? k1 : kpad) - k0) >> 3 : 0, kb = k0 >> 3;
#pragma unroll 1
        for (int s = 0; s < 2; ++s) { /* A_hi x [B_hi; B_lo], A_lo x [B_hi; B_lo] */
          uint32_t ta = (s == 1) ? t_alo : t_ahi;
          /* a K step of 8 TF32 is 256 bytes of B = 16 units of the descriptor's address */
          uint64_t db = make_desc(bh + 256u * kb, lbo, b_sbo);
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
    const int ntile = last_slice ? tile + tile_step : tile;
    const int nslice = last_slice ? 0 : slice + 1;
    if (ntile < tile_end) load_step(ntile, nslice);
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
      /* this warp's 8-column chunks of padded N: one half each, or dealt alternately to the two
       * halves where the problem's stored columns are not split evenly by halves */
      constexpr bool deal = Prob::kEpiAlternate;
      const int cstep = deal ? 8 * NS : 8;
      const int cbeg = deal ? 8 * my_half : my_half * (npad >> 1);
      const int cend = deal ? npad : cbeg + (npad >> 1);
      for (int c0 = cbeg; c0 < cend; c0 += cstep) {
        uint32_t th[8], tl[8];
        tmem_ld8_issue(tmem + lane_addr + (uint32_t)c0, th);
        tmem_ld8_issue(tmem + lane_addr + (uint32_t)(npad + c0), tl);
        tmem_ld_wait();
        reg_fence8(th);
        reg_fence8(tl);
        float t[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) t[i] = __uint_as_float(th[i]) + __uint_as_float(tl[i]);
        if (dst) pb.put8(dst, r, batch, c0, t);
      }
      fence_before_sync();
      __syncthreads();
    }
    tile = ntile, slice = nslice;
  }
  /* after an expired wait, give the MMAs in flight (bounded) time to finish before TMEM goes */
  if (tid == 0 && abort_flag) mbar_wait_bounded(&mbar, phase ^ 1);
  if (tid == 0 && b_pending) mbar_wait_bounded(&bbar, bphase); /* a copy in flight lands */
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}


/* ================================================================ neighbour-sum row form */

constexpr int kNbOut = kRows - 2; /* output rows of a tile: lanes 1..126 (0 and 127 are the
                                   * neighbours of the tile's first and last output rows) */

/* Tensor-memory columns of the neighbour-sum form: the accumulator (npad, rounded up to 32, all
 * four products accumulated in place) plus A hi and A lo of one K slice, as a power of two. */
__host__ __device__ constexpr int nb_tmem_cols(int kpad, int npad) {
  int need = ((npad + 31) / 32) * 32 + 2 * (kpad < kSlice ? kpad : kSlice);
  return need <= 32 ? 32 : need <= 64 ? 64 : need <= 128 ? 128 : need <= 256 ? 256 : 512;
}

/* A row contraction whose output row i is its own row's block of D plus blocks of the rows
 * before and after it: out[i] = D[i][0, w) + D[i-1][w, 2w) + D[i+1][2w, 3w), and, where the
 * problem has them, h[i] = D[i][3w] + D[i-1][3w+1] + D[i+1][3w+2] (w = pb.b).  A convolution-like
 * stage whose row i needs the data of rows i-1..i+1 (a window) then loads each row's data once
 * instead of three times.  Rows are strips of pb.s (a power of two) periodic units; a tile holds
 * 128 consecutive units of one strip (wrapping modulo s) and outputs the middle 126.  The MMA part
 * is k_tc_rowgemm's (A split into TF32 hi/lo in registers, written into the row's TMEM lane; B
 * pre-split in shared memory), with the four products accumulated in place (N = npad) so that the
 * accumulator and one K slice of A fit two CTAs per SM.  Prob supplies, beyond k_tc_rowgemm's:
 *   long s; int b;                         units per strip, block width w (a multiple of 8, <= 32)
 *   long strips;                           strips per batch
 *   __device__ bool has_h(int batch) const;                 the three h columns are in use
 *   __device__ void fix_apply(int batch, const float (&x)[9], float *t) const;
 *                                          adds to out[r][c0..c0+8) what the operator leaves out,
 *                                          from the row's samples x[c0-1 .. c0+7] (A chunk 1,
 *                                          which the kernel keeps in shared memory in FP32)
 *   __device__ void put8_nb(long r, int batch, int c0, const float *t) const;
 *                                          stores out[r][c0..c0+8)
 *   __device__ void put_h(long r, int batch, float v) const;  stores h[r]
 * Row r of strip st is unit r - st * s; src(c, r, batch) addresses row r's chunk c. */
template <class Prob>
__global__ void __launch_bounds__(256, 2) k_tc_nbr(const __grid_constant__ Prob pb, int *status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ uint64_t mbar, bbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  __shared__ int lmap[4][2][8];
  /* warp-edge values: [half][quarter][chunk 0, 1, h][0: lane 31's next block, 1: lane 0's
   * previous block][8] */
  __shared__ float xch[2][4][3][2][8];
  /* the tile's samples (A chunk 1, b <= 32 of them a row) in FP32, for the terms the operator
   * leaves to the epilogue; rows padded to 36 floats against bank conflicts */
  __shared__ __align__(16) float xstage[kRows][36];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kpad = pb.kpad, npad = pb.npad;
  const int ks = kpad < kSlice ? kpad : kSlice;
  const int nslices = (kpad + ks - 1) / ks;
  float *Bhi = reinterpret_cast<float *>(smem_raw);
  float *Blo = Bhi + npad * kpad;
  const uint32_t ncols = (uint32_t)nb_tmem_cols(kpad, npad);
  if (warp == 0) tmem_alloc(&tmem_slot, ncols);
  if (tid == 0) {
    mbar_init(&mbar, 1);
    mbar_init(&bbar, 1);
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
  const long s = pb.s;
  const int tps = (int)((s + kNbOut - 1) / kNbOut); /* tiles per strip */
  const int tiles_per_batch = tps * (int)pb.strips;
  const int ntiles = tiles_per_batch * pb.batches;
  const int quarter = warp & 3, my_half = warp >> 2;
  const int my_m = quarter * 32 + lane;
  const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
  const int w = pb.b, nw8 = w >> 3; /* output chunks of 8 columns */

  /* row of this thread's lane in a tile: unit (t * 126 - 1 + lane) mod s of the tile's strip */
  auto tile_row = [&](int tile, int &batch) -> long {
    batch = tile / tiles_per_batch;
    const int tib = tile - batch * tiles_per_batch;
    const int strip = tib / tps, t = tib - strip * tps;
    return (long)strip * s + (((long)t * kNbOut - 1 + my_m) & (s - 1));
  };

  float4 v[8];
  const float *rowp[4];
  auto load_step = [&](int tile, int slice) {
    if (slice == 0) {
      int batch;
      const long r = tile_row(tile, batch);
#pragma unroll
      for (int c = 0; c < 4; ++c) rowp[c] = c < pb.nchunks ? pb.src(c, r, batch) : nullptr;
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
  const bool runs = pb.batches > 1;
  const int tile_end = runs ? (int)(((long)ntiles * (blockIdx.x + 1)) / gridDim.x) : ntiles;
  const int tile_step = runs ? 1 : (int)gridDim.x;
  /* B of a batch: its shared-memory image, one bulk copy issued by thread 0 (the MMA issuer,
   * who waits for it before the next MMAs); the MMAs reading the previous one have completed */
  uint32_t bphase = 0;
  bool b_pending = false;
  const uint32_t b_bytes = (uint32_t)(smem_bytes(kpad, npad));
  auto stage_b = [&](int batch) {
    if (tid == 0) {
      mbar_expect_tx(&bbar, b_bytes);
      bulk_g2s(smem_addr(smem_raw), pb.bimg + (long)batch * pb.bimg_stride, b_bytes, &bbar);
      b_pending = true;
    }
    cur_batch = batch;
  };
  int tile = runs ? (int)(((long)ntiles * blockIdx.x) / gridDim.x) : (int)blockIdx.x, slice = 0;
  pdl_trigger();
  if (tile < tile_end) stage_b(tile / tiles_per_batch);
  pdl_wait();
  if (tile < tile_end) load_step(tile, 0);
  while (tile < tile_end) {
    int batch;
    const long r = tile_row(tile, batch);
    const int k0 = slice * ks, k1 = k0 + ks;
    if (batch != cur_batch) stage_b(batch);
    if (my_half * 32 < ks) { /* split 8 columns at a time into TF32 hi / lo, both into TMEM */
      const uint32_t col = (uint32_t)(my_half * 32);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (my_half * 32 + 8 * q >= ks) break;
        float h[8], l[8];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const float a[4] = {v[2 * q + i].x, v[2 * q + i].y, v[2 * q + i].z, v[2 * q + i].w};
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            h[4 * i + j] = tf32_rna(a[j]);
            l[4 * i + j] = tf32_rna(a[j] - h[4 * i + j]);
          }
        }
        tmem_st8(t_ahi + lane_addr + col + 8 * q, h);
        tmem_st8(t_alo + lane_addr + col + 8 * q, l);
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) { /* this thread's samples of the row, kept in FP32 */
        const int e = lmap[slice][my_half][i];
        if ((e & 0xFF) == 1) *reinterpret_cast<float4 *>(&xstage[my_m][e >> 8]) = v[i];
      }
    }
    tmem_st_wait();
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
      if (lane == 0) {
        fence_after_sync();
        bool b_ok = true;
        if (b_pending) { /* the operator image has landed */
          b_ok = mbar_wait_bounded(&bbar, bphase);
          bphase ^= 1, b_pending = !b_ok;
          if (!b_ok) atomicExch(status, kErrWaitTimeout), abort_flag = 1;
        }
        const int ksteps = b_ok ? ((k1 < kpad ? k1 : kpad) - k0) >> 3 : 0, kb = k0 >> 3;
#pragma unroll 1
        for (int p = 0; p < 4; ++p) { /* A_hi B_hi, A_hi B_lo, A_lo B_hi, A_lo B_lo, in place */
          uint32_t ta = (p & 2) ? t_alo : t_ahi;
          uint64_t db = make_desc(((p & 1) ? bl : bh) + 256u * kb, lbo, b_sbo);
#pragma unroll 1
          for (int kk = 0; kk < ksteps; ++kk, ta += 8, db += 16)
            mma_tf32_ts(tmem, ta, db, idesc, (k0 | p | kk) != 0);
        }
        mma_commit(&mbar);
      }
      __syncwarp();
    }
    const bool last_slice = slice == nslices - 1;
    const int ntile = last_slice ? tile + tile_step : tile;
    const int nslice = last_slice ? 0 : slice + 1;
    if (ntile < tile_end) load_step(ntile, nslice);
    if (tid == 0 && !mbar_wait_bounded(&mbar, phase)) {
      atomicExch(status, kErrWaitTimeout);
      abort_flag = 1;
    }
    phase ^= 1;
    __syncthreads();
    fence_after_sync();
    if (abort_flag) break;
    if (last_slice) {
      /* epilogue: half h takes the 8-column chunks h, h + 2 of the w outputs, half 1 also the h
       * columns; lane i's neighbours are lanes i -+ 1 (shuffles), across warps shared memory */
      const int tib = tile - batch * tiles_per_batch;
      const long unit = (long)(tib - (tib / tps) * tps) * kNbOut - 1 + my_m;
      const bool out_row = my_m >= 1 && my_m <= kNbOut && unit < s;
      const bool hcols = my_half == 1 && pb.has_h(batch);
      /* one chunk at a time (its own exchange slot): own, next and previous blocks from TMEM,
       * the warp-edge values to shared memory, this half's barrier, then the sums */
      auto half_bar = [&]() {
        if (my_half) asm volatile("bar.sync 2, 128;" ::: "memory");
        else asm volatile("bar.sync 1, 128;" ::: "memory");
      };
      /* the samples the FP32 terms need, x[j-1 .. j+7] of each chunk (the one before the box's
       * first is the previous row's last) */
      float fx[2][9];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = my_half + 2 * j;
        if (out_row && c < nw8) {
          fx[j][0] = c == 0 ? xstage[my_m - 1][w - 1] : xstage[my_m][8 * c - 1];
          const float4 a = *reinterpret_cast<const float4 *>(&xstage[my_m][8 * c]);
          const float4 e = *reinterpret_cast<const float4 *>(&xstage[my_m][8 * c + 4]);
          fx[j][1] = a.x, fx[j][2] = a.y, fx[j][3] = a.z, fx[j][4] = a.w;
          fx[j][5] = e.x, fx[j][6] = e.y, fx[j][7] = e.z, fx[j][8] = e.w;
        }
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = my_half + 2 * j;
        if (c >= nw8) break; /* warp-uniform */
        uint32_t rc[8], rn[8], rp[8];
        tmem_ld8_issue(tmem + lane_addr + (uint32_t)(8 * c), rc);
        tmem_ld8_issue(tmem + lane_addr + (uint32_t)(w + 8 * c), rn);
        tmem_ld8_issue(tmem + lane_addr + (uint32_t)(2 * w + 8 * c), rp);
        tmem_ld_wait();
        reg_fence8(rc);
        reg_fence8(rn);
        reg_fence8(rp);
        float cen[8], nxt[8], prv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
          cen[i] = __uint_as_float(rc[i]), nxt[i] = __uint_as_float(rn[i]), prv[i] = __uint_as_float(rp[i]);
        if (lane == 31)
#pragma unroll
          for (int i = 0; i < 8; ++i) xch[my_half][quarter][j][0][i] = nxt[i];
        if (lane == 0)
#pragma unroll
          for (int i = 0; i < 8; ++i) xch[my_half][quarter][j][1][i] = prv[i];
        half_bar();
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          float fl = __shfl_up_sync(0xffffffffu, nxt[i], 1);
          float fr = __shfl_down_sync(0xffffffffu, prv[i], 1);
          if (lane == 0) fl = quarter > 0 ? xch[my_half][quarter - 1][j][0][i] : 0.f;
          if (lane == 31) fr = quarter < 3 ? xch[my_half][quarter + 1][j][1][i] : 0.f;
          cen[i] += fl + fr;
        }
        if (out_row) {
          pb.fix_apply(batch, fx[j], cen); /* the terms the operator leaves to FP32 */
          pb.put8_nb(r, batch, 8 * c, cen);
        }
      }
      if (hcols) {
        float hv[8];
        tmem_ld8(tmem + lane_addr + (uint32_t)(3 * w), hv);
        if (lane == 31) xch[1][quarter][2][0][0] = hv[1];
        if (lane == 0) xch[1][quarter][2][1][0] = hv[2];
        half_bar();
        float fl = __shfl_up_sync(0xffffffffu, hv[1], 1);
        float fr = __shfl_down_sync(0xffffffffu, hv[2], 1);
        if (lane == 0) fl = quarter > 0 ? xch[1][quarter - 1][2][0][0] : 0.f;
        if (lane == 31) fr = quarter < 3 ? xch[1][quarter + 1][2][1][0] : 0.f;
        if (out_row) pb.put_h(r, batch, hv[0] + (fl + fr));
      }
      fence_before_sync();
      __syncthreads();
    }
    tile = ntile, slice = nslice;
  }
  if (tid == 0 && abort_flag) mbar_wait_bounded(&mbar, phase ^ 1);
  if (tid == 0 && b_pending) mbar_wait_bounded(&bbar, bphase); /* a copy in flight lands */
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

/* ===================================================================== 16-lane row form */

/* Column permutation within each group of 16 (an involution-free bijection): TMEM / shared
 * column 16g + 8h + 2j + e holds source column 16g + 4j + 2h + e (h, e in {0, 1}, j < 4). */
__host__ __device__ __forceinline__ int perm16(int c) {
  return (c & ~15) + 4 * ((c >> 1) & 3) + 2 * ((c >> 3) & 1) + (c & 1);
}
__host__ __device__ constexpr int round16(int v) { return (v + 15) & ~15; }

/* Shared memory of the 16-lane row form: B hi and lo with K padded to 16. */
__host__ __device__ constexpr size_t smem16_bytes(int kpad, int npad) {
  return (size_t)(2 * npad * round16(kpad)) * sizeof(float);
}

/* The row contraction of k_tc_rowgemm (same TMEM budget, operator staging and MMAs, two CTAs
 * per SM, persistent over tiles) with another path for A into TMEM and for D out of it.
 * Warp w owns the 16 TMEM lanes (tile rows) 32 (w % 4) + 16 (w / 4) .. +15 across all K columns
 * of a slice, through tcgen05.st / ld of shape 16x256b: thread t holds rows t/4 and t/4 + 8 and
 * columns 2 (t % 4), 2 (t % 4) + 1 of each 8-column chunk.  K (A's columns and B's K columns) and
 * N (B's rows, so D's columns) are permuted within each group of 16 by perm16, alike for A and
 * B, which leaves the contraction unchanged up to the order of its sums; with it the column
 * pairs a thread holds in two chunks are four consecutive source columns.  So a thread loads
 * one float4 per row and 16-column group of A and stores one float4 per row and group of the
 * output: 8 rows x 64 contiguous bytes per warp instruction, where one row per lane (the 32x32b
 * shape) makes every instruction touch 32 rows x 16 bytes.  Prob supplies put4(dst, r, batch,
 * c, v): output columns c..c+3 of row r. */
template <class Prob>
__global__ void __launch_bounds__(256, 2) k_tc_rowgemm16(const __grid_constant__ Prob pb, int *status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ uint64_t mbar, bbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  /* load map: for slice s, 16-column group g and quad j (source columns 16g + 4j .. +3 of the
   * slice), the A chunk (low byte, 0xFF = zero) and the float offset within that chunk's row */
  __shared__ int lmap[4][4][4];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kpad = pb.kpad, npad = pb.npad;
  const int kp = round16(kpad);              /* K extent of staged B and of A in TMEM */
  const int ks = kp < kSlice ? kp : kSlice;  /* a multiple of 16 */
  const int nslices = (kp + ks - 1) / ks;    /* <= 4: kpad <= 256 */
  const int ngroups = ks >> 4;
  float *Bhi = reinterpret_cast<float *>(smem_raw);
  float *Blo = Bhi + npad * kp;
  const uint32_t ncols = (uint32_t)tmem_cols(kp, npad);
  if (warp == 0) tmem_alloc(&tmem_slot, ncols);
  if (tid == 0) {
    mbar_init(&mbar, 1);
    mbar_init(&bbar, 1);
    fence_mbar_init();
    abort_flag = 0;
  }
  if (tid < 4 * 4 * 4) {
    const int sl = tid >> 4, g = (tid >> 2) & 3, j = tid & 3;
    const int k = sl * ks + 16 * g + 4 * j;
    int e = 0xFF;
    if (sl < nslices && 16 * g < ks && k < kpad)
      for (int c = 0; c < pb.nchunks; ++c)
        if (k >= pb.coff[c] && k < pb.coff[c] + pb.clen[c]) e = c | ((k - pb.coff[c]) << 8);
    lmap[sl][g][j] = e;
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;
  /* accumulator columns [0, npad): A x B_hi, [npad, 2 npad): A x B_lo (B_lo follows B_hi in
   * shared memory as the next row groups, so one descriptor of N = 2 npad covers both) */
  const uint32_t d_cols = (uint32_t)(((2 * npad + 31) / 32) * 32);
  const uint32_t t_ahi = tmem + d_cols, t_alo = tmem + d_cols + (uint32_t)ks;
  const uint32_t idesc = make_idesc_tf32(2 * npad);
  const uint32_t b_sbo = (uint32_t)kp * 32, lbo = 128;
  const uint32_t bh = smem_addr(Bhi);
  const int tiles_per_batch = (int)((pb.rows + kRows - 1) / kRows);
  const int ntiles = tiles_per_batch * pb.batches;
  const int quarter = warp & 3, half = warp >> 2, j4 = lane & 3;
  const int row0 = quarter * 32 + half * 16 + (lane >> 2); /* tile rows row0 and row0 + 8 */
  const uint32_t lane_addr = (uint32_t)(quarter * 32 + half * 16) << 16;

  float4 v[2][4]; /* [row][16-column group] */
  const float *rowp[2][4];
  auto load_step = [&](int tile, int slice) {
    if (slice == 0) {
      const int batch = tile / tiles_per_batch;
      const long rb = (long)(tile - batch * tiles_per_batch) * kRows + row0;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const long r = rb + 8 * i;
        const bool live = r < pb.rows;
#pragma unroll
        for (int c = 0; c < 4; ++c) rowp[i][c] = (live && c < pb.nchunks) ? pb.src(c, r, batch) : nullptr;
      }
    }
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const int e = lmap[slice][g][j4];
      const int c = e & 0xFF;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        v[i][g] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c != 0xFF) {
          const float *rp = c == 0 ? rowp[i][0] : (c == 1 ? rowp[i][1] : (c == 2 ? rowp[i][2] : rowp[i][3]));
          if (rp) v[i][g] = __ldg(reinterpret_cast<const float4 *>(rp + (e >> 8)));
        }
      }
    }
  };

  int cur_batch = -1;
  uint32_t phase = 0;
  const bool runs = pb.batches > 1;
  const int tile_end = runs ? (int)(((long)ntiles * (blockIdx.x + 1)) / gridDim.x) : ntiles;
  const int tile_step = runs ? 1 : (int)gridDim.x;
  /* B of a batch, pre-split, in the core-matrix layout with K extent kp; shared element
   * (n, k) holds operator element (perm16(n), perm16(k)), zero for k >= kpad */
  /* B of a batch: its shared-memory image, one bulk copy issued by thread 0 (the MMA issuer,
   * who waits for it before the next MMAs); the MMAs reading the previous one have completed */
  uint32_t bphase = 0;
  bool b_pending = false;
  const uint32_t b_bytes = (uint32_t)(smem16_bytes(kpad, npad));
  auto stage_b = [&](int batch) {
    if (tid == 0) {
      mbar_expect_tx(&bbar, b_bytes);
      bulk_g2s(smem_addr(smem_raw), pb.bimg16 + (long)batch * pb.bimg16_stride, b_bytes, &bbar);
      b_pending = true;
    }
    cur_batch = batch;
  };
  int tile = runs ? (int)(((long)ntiles * blockIdx.x) / gridDim.x) : (int)blockIdx.x, slice = 0;
  /* programmatic dependent launch: the first operator (a plan constant) is staged before the
   * wait; nothing global is read or written before it */
  pdl_trigger();
  if (tile < tile_end) stage_b(tile / tiles_per_batch);
  pdl_wait();
  if (tile < tile_end) load_step(tile, 0);
  while (tile < tile_end) {
    const int batch = tile / tiles_per_batch;
    const long r0 = (long)(tile - batch * tiles_per_batch) * kRows;
    const int k0 = slice * ks, k1 = k0 + ks;
    if (batch != cur_batch) stage_b(batch); /* the previous step's MMAs have completed */
    /* split into TF32 hi / lo and write both into this warp's 16 TMEM lanes */
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      if (g >= ngroups) break;
      const float a[8] = {v[0][g].x, v[0][g].y, v[1][g].x, v[1][g].y, v[0][g].z, v[0][g].w, v[1][g].z, v[1][g].w};
      float h[8], l[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        h[i] = tf32_rna(a[i]);
        l[i] = tf32_rna(a[i] - h[i]);
      }
      tmem_st16x2(t_ahi + lane_addr + 16u * g, h);
      tmem_st16x2(t_alo + lane_addr + 16u * g, l);
    }
    tmem_st_wait();
    fence_before_sync();
    __syncthreads();
    if (warp == 0) { /* lane 0 issues; the rest of warp 0 waits at __syncwarp */
      if (lane == 0) {
        fence_after_sync();
        bool b_ok = true;
        if (b_pending) { /* the operator image has landed */
          b_ok = mbar_wait_bounded(&bbar, bphase);
          bphase ^= 1, b_pending = !b_ok;
          if (!b_ok) atomicExch(status, kErrWaitTimeout), abort_flag = 1;
        }
        const int ksteps = b_ok ? ((k1 < kp ? k1 : kp) - k0) >> 3 : 0, kb = k0 >> 3;
#pragma unroll 1
        for (int s = 0; s < 2; ++s) { /* A_hi x [B_hi; B_lo], A_lo x [B_hi; B_lo] */
          uint32_t ta = (s == 1) ? t_alo : t_ahi;
          uint64_t db = make_desc(bh + 256u * kb, lbo, b_sbo);
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
    const int ntile = last_slice ? tile + tile_step : tile;
    const int nslice = last_slice ? 0 : slice + 1;
    if (ntile < tile_end) load_step(ntile, nslice);
    if (tid == 0 && !mbar_wait_bounded(&mbar, phase)) {
      atomicExch(status, kErrWaitTimeout);
      abort_flag = 1;
    }
    phase ^= 1;
    __syncthreads();
    fence_after_sync();
    if (abort_flag) break;
    if (last_slice) {
      /* epilogue: D column 16g + 8h + 2j + e is output perm16(.) = 16g + 4j + 2h + e, so this
       * thread's columns of a group are the four outputs 16g + 4j .. +3 of its two rows */
      float *dst[2];
      long rr[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        rr[i] = r0 + row0 + 8 * i;
        dst[i] = rr[i] < pb.rows ? pb.dst(rr[i], batch) : nullptr;
      }
      for (int g = 0; g < (npad >> 4); ++g) {
        float t[8];
        {
          uint32_t rh[8], rl[8];
          tmem_ld16x2_issue(tmem + lane_addr + 16u * g, rh);
          tmem_ld16x2_issue(tmem + lane_addr + (uint32_t)npad + 16u * g, rl);
          tmem_ld_wait();
          reg_fence8(rh);
          reg_fence8(rl);
#pragma unroll
          for (int i = 0; i < 8; ++i) t[i] = __uint_as_float(rh[i]) + __uint_as_float(rl[i]);
        }
        const int c = 16 * g + 4 * j4;
        if (dst[0]) pb.put4(dst[0], rr[0], batch, c, make_float4(t[0], t[1], t[4], t[5]));
        if (dst[1]) pb.put4(dst[1], rr[1], batch, c, make_float4(t[2], t[3], t[6], t[7]));
      }
      fence_before_sync();
      __syncthreads();
    }
    tile = ntile, slice = nslice;
  }
  /* after an expired wait, give the MMAs in flight (bounded) time to finish before TMEM goes */
  if (tid == 0 && abort_flag) mbar_wait_bounded(&mbar, phase ^ 1);
  if (tid == 0 && b_pending) mbar_wait_bounded(&bbar, bphase); /* a copy in flight lands */
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}


constexpr unsigned long long kWaitNs = 2000000000ull; /* 2 s per wait */


__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" : : "r"(smem_addr(bar)) : "memory");
}

/* Waits for phase `parity` of `bar`; false when the CTA aborted or 2 s passed (then the abort
 * flag and the status word are set).  The clock is read only after 4096 unsuccessful polls. */
__device__ __forceinline__ bool t_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag,
                                       int *status, unsigned long long limit_ns = kWaitNs) {
  unsigned long long t0 = 0;
  for (unsigned it = 0;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63) == 63 && *abort_flag) return false;
    if ((it & 4095) == 4095) {
      const unsigned long long now = global_ns();
      if (t0 == 0) {
        t0 = now;
      } else if (now - t0 > limit_ns) {
        atomicExch(status, kErrWaitTimeout);
        *abort_flag = 1;
        return false;
      }
    }
  }
}

/* t_wait that sleeps nap_ns between polls once the first few have failed, so that a warp
 * waiting for long (an epilogue warp for its next tile) leaves its sub-partition's issue slots to
 * the warps that have work; nap_ns = 0 polls without sleeping. */
__device__ __forceinline__ bool t_wait_nap(uint64_t *bar, uint32_t parity, volatile int *abort_flag,
                                           int *status, unsigned nap_ns) {
  if (nap_ns == 0) return t_wait(bar, parity, abort_flag, status);
  unsigned long long t0 = 0;
  for (unsigned it = 0;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it < 4) continue;
    __nanosleep(nap_ns);
    if ((it & 15) == 15 && *abort_flag) return false;
    if ((it & 63) == 63) {
      const unsigned long long now = global_ns();
      if (t0 == 0) {
        t0 = now;
      } else if (now - t0 > kWaitNs) {
        atomicExch(status, kErrWaitTimeout);
        *abort_flag = 1;
        return false;
      }
    }
  }
}

/* Waits for phase `parity` of `bar` for at most about 2 s, whatever the abort flag says. */
__device__ __forceinline__ bool t_wait_time(uint64_t *bar, uint32_t parity) {
  unsigned long long t0 = 0;
  for (unsigned it = 0;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 4095) == 4095) {
      const unsigned long long now = global_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > kWaitNs) return false;
    }
  }
}



/* ======================================================================== warp-specialised form */

/* The row contraction D[r][0..nout) = sum_k A(r, k) B[k][.] with every step of it overlapped:
 * loads of A, its split into TF32 hi / lo, the MMAs and the epilogue run in separate warps that
 * hand work to one another through mbarriers, so that no step waits for the one before it to
 * finish on the same tile.  One CTA per SM (all of its tensor memory), persistent over 128-row
 * tiles, K taken in slots of 32 columns:
 *
 *   warps 0-7   producers, each on its own: warp w (lane quarter q = w % 4, column half
 *               h = w / 4) owns rows 32 q .. 32 q + 31 and columns 16 h .. 16 h + 15 of every
 *               slot.  Global -> shared: it copies that block with 16-byte cp.async (8 rows x 64
 *               bytes per instruction) into a ring of kWStages shared-memory stages, kWStages - 1
 *               slots in flight.  Shared -> TMEM: lane i reads its row 32 q + i, splits it into
 *               hi / lo and writes both into one of kWSlots A slots in tensor memory
 *               (tcgen05.st), then the warp arrives on the slot's `full` barrier.  A warp reads
 *               only what it copied, so warps wait for nothing but their own copies.  Units are
 *               stored XOR-swizzled in shared memory (16-byte unit j of row i at position
 *               j ^ (i & 7)): copies and row reads take four wavefronts per warp instruction.
 *   warp 12     one thread issues, per K step of 8, A_hi x [B_hi; B_lo] (N = 2 npad) and
 *               A_lo x B_hi (N = npad) into one of two TMEM accumulators: split TF32 with three
 *               products (the A_lo B_lo term, 2^-22 relative, is left out), FP32 accumulation;
 *               it commits each slot to the slot's `empty` barrier and each tile to the
 *               accumulator's `full` barrier.  It also stages B: the host lays each batch's
 *               operator out in the MMA's K-major core-matrix layout (hi rows, then lo rows), so
 *               one bulk copy brings it into shared memory.
 *   warps 8-11  epilogue: warp 8 + q reads lane quarter q of the accumulator, adds its two
 *               column halves and stores each row's 8-column chunks through Prob::put8, then
 *               frees the accumulator for the tile after next.
 *
 * Prob supplies rows, batches, nchunks / clen / coff (A chunks, multiples of 4 floats), kpad
 * (multiple of 8), npad (multiple of 16, at most 64), nout, wsb (the B operator of batch z at
 * wsb + z * wsb_stride floats, 2 npad rows x round32(kpad) columns in core-matrix layout),
 * src(c, r, z) (16-byte-aligned row of chunk c), dst(r, z) and put8(dst, r, z, c0, t).
 * Every wait is bounded (2 s); on expiry the CTA records kErrWaitTimeout, every role leaves its
 * loop, copies in flight land and the MMAs in flight complete before TMEM is freed. */
constexpr int kWKs = 64;       /* K columns per A slot */
constexpr int kWSlots = 2;     /* A slots in tensor memory: hi + lo, 128 columns each */
constexpr int kWStages = 4;    /* shared-memory ring of A: 128 rows x 64 floats (32 KB) per stage */
constexpr int kWProd = 8;      /* producer warps */
constexpr int kWEpi = 4;       /* epilogue warps: one per TMEM lane quarter */
constexpr int kWThreads = (kWProd + kWEpi + 1) * 32;
constexpr int kWMaxSlots = 4;  /* K <= 256 */
constexpr int kWUnits = kWKs / 4;       /* 16-byte units per row of a slot */
constexpr int kWRowBytes = kWKs * 4;    /* a slot row in the ring */
constexpr int kWStageBytes = kRows * kWRowBytes;

__host__ __device__ constexpr int round32(int v) { return (v + 31) & ~31; }
/* accumulator columns of one tile: B_hi and B_lo products side by side */
__host__ __device__ constexpr int ws_acc_cols(int npad) { return round32(2 * npad); }
__host__ __device__ constexpr size_t ws_b_floats(int kpad, int npad) {
  return (size_t)2 * npad * round32(kpad);
}
/* eb: bytes per operator element, 4 (TF32) or 2 (BF16) */
__host__ __device__ constexpr size_t ws_smem_bytes(int kpad, int npad, int eb = 4) {
  return ws_b_floats(kpad, npad) * eb + (size_t)kWStages * kWStageBytes;
}
/* the operator fits: two accumulators and the A slots within 512 TMEM columns, K <= 256 */
__host__ __device__ constexpr bool ws_fits(int kpad, int npad) {
  return npad % 16 == 0 && npad <= 64 && kpad % 8 == 0 && kpad <= kWKs * kWMaxSlots &&
         2 * ws_acc_cols(npad) + kWSlots * 2 * kWKs <= 512 && ws_smem_bytes(kpad, npad) <= 220 * 1024;
}
/* element index of operator element (n, k), n < 2 npad (hi rows, then lo rows), in the layout
 * the kernel copies: 8-row groups of core matrices of 8 rows x 16 bytes along K (4 TF32 or 8
 * BF16 values per row of a core matrix) */
__host__ __device__ inline long ws_b_index(int n, int k, int kpad) {
  return (long)(n >> 3) * (round32(kpad) * 8) + (k >> 2) * 32 + (n & 7) * 4 + (k & 3);
}
__host__ __device__ inline long ws_b_index_bf16(int n, int k, int kpad) {
  return (long)(n >> 3) * (round32(kpad) * 8) + (k >> 3) * 64 + (n & 7) * 8 + (k & 7);
}

/* Instruction descriptor, kind::f16 with BF16 A and B: D = F32, both K-major, M = 128. */
__host__ __device__ constexpr uint32_t make_idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
/* BF16 MMA, A from tensor memory (two values per 32-bit column, K = 16 per instruction). */
__device__ __forceinline__ void mma_bf16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(d_tmem), "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0),
        "r"(0)
      : "memory");
}
/* two floats to BF16 (round to nearest even), packed: `lo` in bits 0-15, `hi` in bits 16-31 */
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}

__device__ __forceinline__ void cp_async16_cg(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" : : "r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" : : "n"(N) : "memory");
}
/* barrier `id` over `nthreads` threads that ORs a flag across them (the same answer for all) */
__device__ __forceinline__ bool named_bar_or(int id, int nthreads, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}

template <class Prob, bool kBF = false>
/* 13 warps: at most 4 on an SM sub-partition, so up to 128 registers a thread */
__global__ void __maxnreg__(128) k_tc_ws(const __grid_constant__ Prob pb, int *status) {
  /* kBF: BF16x3 instead of split TF32: A and B split into BF16 hi + lo (the lo part the BF16
   * rounding of the residual), products A_hi B_hi + A_hi B_lo + A_lo B_hi, kind::f16 MMAs of
   * K = 16; about 2^-17 relative per product, for orders whose truncation is far above that */
  constexpr int kEB = kBF ? 2 : 4;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ uint64_t tfull[kWSlots], tempty[kWSlots], afull[2], aempty[2], bbar, fin;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  /* per slot j and 16-byte unit u of its 32 columns: A chunk (low byte, 0xFF = zero), float
   * offset in that chunk's row (high bits) */
  __shared__ int lmap[kWMaxSlots][kWUnits];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kpad = pb.kpad, npad = pb.npad;
  const int nsl = (kpad + kWKs - 1) / kWKs;
  float *Bs = reinterpret_cast<float *>(smem_raw);
  unsigned char *ring = smem_raw + ws_b_floats(kpad, npad) * kEB;
  const int mma_warp = kWProd + kWEpi;
  if (warp == mma_warp) tmem_alloc(&tmem_slot, 512);
  if (tid == 0) {
    for (int i = 0; i < kWSlots; ++i) mbar_init(&tfull[i], kWProd), mbar_init(&tempty[i], 1);
    for (int i = 0; i < 2; ++i) mbar_init(&afull[i], 1), mbar_init(&aempty[i], kWEpi);
    mbar_init(&bbar, 1);
    mbar_init(&fin, 1);
    fence_mbar_init();
    abort_flag = 0;
  }
  if (tid < kWMaxSlots * kWUnits) {
    const int j = tid / kWUnits, u = tid % kWUnits, k = j * kWKs + 4 * u;
    int e = 0xFF;
    if (j < nsl && k < kpad)
      for (int c = 0; c < pb.nchunks; ++c)
        if (k >= pb.coff[c] && k < pb.coff[c] + pb.clen[c]) e = c | ((k - pb.coff[c]) << 8);
    lmap[j][u] = e;
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const int acc_cols = ws_acc_cols(npad);
  const int tiles_per_batch = (int)((pb.rows + kRows - 1) / kRows);
  const int ntiles = tiles_per_batch * pb.batches;
  /* one operator per batch: a CTA takes a contiguous run of tiles (it restages B once or twice);
   * one batch: tiles strided by the grid */
  const bool runs = pb.batches > 1;
  const int tile0 = runs ? (int)(((long)ntiles * blockIdx.x) / gridDim.x) : (int)blockIdx.x;
  const int tile_end = runs ? (int)(((long)ntiles * (blockIdx.x + 1)) / gridDim.x) : ntiles;
  const int tile_step = runs ? 1 : (int)gridDim.x;
  const int my_tiles = tile0 < tile_end ? (tile_end - tile0 + tile_step - 1) / tile_step : 0;
  const uint32_t b_bytes = (uint32_t)(ws_b_floats(kpad, npad) * kEB);

  /* the operators are plan constants: the first batch's is requested before waiting for the
   * kernel this one depends on */
  pdl_trigger();
  if (warp == mma_warp && lane == 0 && my_tiles > 0) {
    mbar_expect_tx(&bbar, b_bytes);
    bulk_g2s(smem_addr(Bs), pb.wsb + (long)(tile0 / tiles_per_batch) * pb.wsb_stride, b_bytes, &bbar);
  }
  pdl_wait();

  if (warp < kWProd) {
    /* ------------------------------------------------------------ producers */
    const int q = warp & 3, h = warp >> 2;
    const int my_row = q * 32 + lane;                 /* TMEM lane = tile row this thread splits */
    const uint32_t lane_addr = (uint32_t)(q * 32) << 16;
    /* this warp copies exactly what it splits: its 32 rows, 16-byte units 8 h .. 8 h + 7 of each
     * (32 columns); lane: unit 8 h + lane % 8 of rows 32 q + 4 m + lane / 8, so each copy
     * instruction moves 4 rows x 128 contiguous bytes, and a warp waits for no other warp */
    const int cu = 8 * h + (lane & 7), crow = q * 32 + (lane >> 3);
    const uint32_t ring0 = smem_addr(ring);
    const int G = my_tiles * nsl;
    /* copy cursor: the next slot whose copies are issued, kept incrementally (no divisions by
     * runtime values per slot: those run on the conversion pipe) */
    int c_g = 0, c_j = 0, c_t = tile0, c_batch = 0;
    long c_r0 = 0;
    auto c_tile = [&]() {
      c_batch = c_t / tiles_per_batch;
      c_r0 = (long)(c_t - c_batch * tiles_per_batch) * kRows;
    };
    if (G > 0) c_tile();
    auto issue = [&]() {
      if (c_g < G) {
        const int e = lmap[c_j][cu], c = e & 0xFF;
        if (c != 0xFF) {
          const uint32_t st = ring0 + (uint32_t)((c_g & (kWStages - 1)) * kWStageBytes);
#pragma unroll
          for (int m = 0; m < 8; ++m) {
            const int row = crow + 4 * m;
            const long r = c_r0 + row;
            if (r < pb.rows)
              cp_async16_cg(st + (uint32_t)(row * kWRowBytes + ((cu ^ (row & 7)) << 4)),
                            pb.src(c, r, c_batch) + (e >> 8));
          }
        }
        ++c_g;
        if (++c_j == nsl) {
          c_j = 0, c_t += tile_step;
          if (c_g < G) c_tile();
        }
      }
      cp_async_commit(); /* one group per slot, empty or not: wait_group counts stay exact */
    };
    /* this lane's row of slot g (slot f_j of its tile) from the ring, after its copies landed */
    float4 a[8];
    int f_j = 0;
    auto fetch = [&](int g) {
      cp_async_wait<kWStages - 2>(); /* this thread's copies of slot g have landed */
      __syncwarp(); /* ... and the warp's; its lanes have read slot g - 1, whose stage is refilled */
      issue();      /* slot g + kWStages - 1 */
      const uint32_t st = ring0 + (uint32_t)((g & (kWStages - 1)) * kWStageBytes) + (uint32_t)(my_row * kWRowBytes);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int u = 8 * h + i;
        a[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        if ((lmap[f_j][u] & 0xFF) != 0xFF)
          asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                       : "=f"(a[i].x), "=f"(a[i].y), "=f"(a[i].z), "=f"(a[i].w)
                       : "r"(st + (uint32_t)((u ^ (my_row & 7)) << 4)));
      }
      if (++f_j == nsl) f_j = 0;
    };
    /* split into hi / lo: 32 TF32 pairs, or 16 packed BF16 pairs of words */
    float hv[32], lv[32];
    auto split = [&]() {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float av[4] = {a[i].x, a[i].y, a[i].z, a[i].w};
        if constexpr (kBF) {
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const uint32_t hw = pack_bf16x2(av[2 * k], av[2 * k + 1]);
            const float h0 = __uint_as_float(hw << 16), h1 = __uint_as_float(hw & 0xFFFF0000u);
            hv[2 * i + k] = __uint_as_float(hw);
            lv[2 * i + k] = __uint_as_float(pack_bf16x2(av[2 * k] - h0, av[2 * k + 1] - h1));
          }
        } else {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            hv[4 * i + k] = tf32_rna(av[k]);
            lv[4 * i + k] = tf32_rna(av[k] - hv[4 * i + k]);
          }
        }
      }
    };
#pragma unroll 1
    for (int g = 0; g < kWStages - 1; ++g) issue();
    if (G > 0) {
      fetch(0);
      split();
    }
    /* per slot: wait for its TMEM slot, store hi / lo, then (while the stores complete) fetch the
     * next slot's row, then wait for the stores, signal, and split the next slot */
    static_assert(kWSlots == 2 && (kWStages & (kWStages - 1)) == 0, "slot and stage indices are masks");
    for (int g = 0; g < G; ++g) {
      const int s = g & 1;
      bool ok = true;
      if (lane == 0) ok = t_wait_nap(&tempty[s], (uint32_t)(((g >> 1) & 1) ^ 1), &abort_flag, status, pb.nap / 4);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      fence_after_sync();
      const uint32_t base = tmem + lane_addr + (uint32_t)(2 * acc_cols + s * 2 * kWKs);
      if constexpr (kBF) { /* 32 values = 16 columns per half; lo 32 columns after hi */
        tmem_st8(base + 16 * h, hv);
        tmem_st8(base + 16 * h + 8, hv + 8);
        tmem_st8(base + kWKs / 2 + 16 * h, lv);
        tmem_st8(base + kWKs / 2 + 16 * h + 8, lv + 8);
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          tmem_st8(base + 32 * h + 8 * i, hv + 8 * i);
          tmem_st8(base + kWKs + 32 * h + 8 * i, lv + 8 * i);
        }
      }
      const bool more = g + 1 < G && !__any_sync(0xffffffffu, abort_flag != 0);
      if (more) fetch(g + 1);
      tmem_st_wait();
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tfull[s]);
      if (!more) break;
      split();
    }
    cp_async_wait<0>(); /* nothing may still write shared memory when the CTA ends */
  } else if (warp < kWProd + kWEpi) {
    /* ------------------------------------------------------------ epilogue */
    const int q = warp & 3, eh = (warp - kWProd) >> 2, estep = 8 * (kWEpi / 4);
    const uint32_t lane_addr = (uint32_t)(q * 32) << 16;
    for (int lt = 0; lt < my_tiles; ++lt) {
      const int t = tile0 + lt * tile_step, a = lt & 1;
      bool ok = true;
      if (lane == 0) ok = t_wait_nap(&afull[a], (uint32_t)((lt >> 1) & 1), &abort_flag, status, pb.nap);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      fence_after_sync();
      const int batch = t / tiles_per_batch;
      const long r = (long)(t - batch * tiles_per_batch) * kRows + q * 32 + lane;
      float *dst = r < pb.rows ? pb.dst(r, batch) : nullptr;
      const uint32_t acc = tmem + lane_addr + (uint32_t)(a * acc_cols);
      for (int c0 = 8 * eh; c0 < npad; c0 += estep) {
        float v[8], w[8];
        tmem_ld8(acc + (uint32_t)c0, v);
        tmem_ld8(acc + (uint32_t)(npad + c0), w);
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] += w[i];
        if (dst) pb.put8(dst, r, batch, c0, v);
      }
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&aempty[a]);
    }
  } else {
   if (lane == 0) {
    /* ---------------------------------------------------------- MMA issue, B staging */
    const uint32_t idesc2 = kBF ? make_idesc_bf16(2 * npad) : make_idesc_tf32(2 * npad);
    const uint32_t idesc1 = kBF ? make_idesc_bf16(npad) : make_idesc_tf32(npad);
    const uint32_t bsm = smem_addr(Bs), b_sbo = (uint32_t)round32(kpad) * 8 * kEB;
    int cur_batch = my_tiles > 0 ? tile0 / tiles_per_batch : -1;
    uint32_t bphase = 0;
    bool ok = my_tiles == 0 || t_wait(&bbar, bphase, &abort_flag, status);
    bphase ^= 1;
    int g = 0;
    for (int lt = 0; lt < my_tiles && ok; ++lt) {
      const int t = tile0 + lt * tile_step, a = lt & 1;
      const int batch = t / tiles_per_batch;
      if (batch != cur_batch && pb.wsb_stride != 0) { /* the MMAs reading the old operator
                                                        * complete, then the new one is staged */
        mma_commit(&bbar);
        ok = t_wait(&bbar, bphase, &abort_flag, status);
        bphase ^= 1;
        if (!ok) break;
        mbar_expect_tx(&bbar, b_bytes);
        bulk_g2s(bsm, pb.wsb + (long)batch * pb.wsb_stride, b_bytes, &bbar);
        ok = t_wait(&bbar, bphase, &abort_flag, status);
        bphase ^= 1;
        if (!ok) break;
        cur_batch = batch;
      }
      ok = t_wait_nap(&aempty[a], (uint32_t)(((lt >> 1) & 1) ^ 1), &abort_flag, status, pb.nap / 8);
      if (!ok) break;
      fence_after_sync();
      const uint32_t d = tmem + (uint32_t)(a * acc_cols);
      for (int j = 0; j < nsl; ++j, ++g) {
        const int s = g & 1;
        ok = t_wait_nap(&tfull[s], (uint32_t)((g >> 1) & 1), &abort_flag, status, pb.nap / 8);
        if (!ok) break;
        fence_after_sync();
        const int k0 = j * kWKs;
        const uint32_t ahi = tmem + (uint32_t)(2 * acc_cols + s * 2 * kWKs);
        if constexpr (kBF) {
          /* K step of 16 BF16 = two core matrices along K = 256 bytes; 8 TMEM columns of A (lo
           * 32 columns after hi) */
          const int ksteps = (((kpad - k0) < kWKs ? (kpad - k0) : kWKs) + 15) >> 4;
          for (int kk = 0; kk < ksteps; ++kk) {
            const uint64_t db = make_desc(bsm + 256u * (uint32_t)((k0 >> 4) + kk), 128, b_sbo);
            mma_bf16_ts(d, ahi + 8u * kk, db, idesc2, (j | kk) != 0);
            mma_bf16_ts(d, ahi + kWKs / 2 + 8u * kk, db, idesc1, 1);
          }
        } else {
          const int ksteps = ((kpad - k0) < kWKs ? (kpad - k0) : kWKs) >> 3;
          for (int kk = 0; kk < ksteps; ++kk) {
            /* K step of 8 TF32 = two core matrices along K = 256 bytes of each 8-row group */
            const uint64_t db = make_desc(bsm + 256u * (uint32_t)((k0 >> 3) + kk), 128, b_sbo);
            mma_tf32_ts(d, ahi + 8u * kk, db, idesc2, (j | kk) != 0);
            mma_tf32_ts(d, ahi + kWKs + 8u * kk, db, idesc1, 1);
          }
        }
        mma_commit(&tempty[s]);
      }
      if (!ok) break;
      mma_commit(&afull[a]);
    }
    /* every MMA and copy issued has completed before shared and tensor memory go */
    mma_commit(&fin);
    if (!t_wait_time(&fin, 0)) atomicExch(status, kErrWaitTimeout);
    if (!ok && my_tiles > 0) t_wait_time(&bbar, bphase ^ 1);
   }
    __syncwarp(); /* the MMA warp meets the CTA barrier converged */
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == mma_warp) tmem_dealloc(tmem, 512);
}


}  // namespace tc
