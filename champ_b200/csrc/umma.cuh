// umma.cuh — LCAO contraction on the 5th-generation tensor cores (mixed
// precision path): orb[r][o] = sum_m phi[r][m] coef(m,o) with the FP64
// operands split into two TF32-representable FP32 parts,
//   x = x_hi + x_lo,   x_hi = rna_tf32(x),   x_lo = fp32(x - x_hi),
// and three products per k-block accumulated in FP32 in tensor memory:
//   hi*hi + hi*lo + lo*hi   (relative error ~2^-21 per product, the dropped
//   lo*lo term ~2^-22).
//
// One CTA per 128-row tile, all output columns (N padded to a multiple of
// 16, <= 256) in one UMMA accumulator:
//   warp 0 lane 0   TMA producer: per k-block of 32 elements, the A_hi/A_lo
//                   tiles (128 rows x 128 B) and the B_hi/B_lo tiles (NP rows
//                   x 128 B), 128-byte swizzle, into a ring of stages
//   warp 1 lane 0   MMA issuer: 4 k-steps x 3 tcgen05.mma.kind::tf32 per
//                   stage, tcgen05.commit releases the stage
//   4 warps         epilogue: tcgen05.ld of the warp's 32 TMEM lanes, FP64
//                   stores of the valid rows and columns
// Every mbarrier wait is bounded (about 2 s of globaltimer); a timeout sets
// *err, skips the epilogue and still frees the tensor memory.
#pragma once
#include <cuda.h>
#include "common.cuh"

namespace cw {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t gtimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Wait for the phase with the given parity to complete; false after ~2 s.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const uint64_t t0 = gtimer_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (gtimer_ns() - t0 > 2000000000ull) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major operand tile in shared memory, rows of 128 B with the 128-byte
// swizzle: 8-row groups 1024 B apart (stride byte offset), leading byte
// offset unused, descriptor version 1, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t sdesc_k_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)(1024u >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// kind::tf32 instruction descriptor: FP32 accumulator, TF32 A and B, both
// K-major, M = 128, N = np.
__device__ __forceinline__ uint32_t idesc_tf32(int np) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory bytes of one launch (stages of A_hi, A_lo, B_hi, B_lo plus
// alignment slack and barriers).
__host__ __device__ inline size_t umma_stage_bytes(int np) { return 2u * 128u * 128u + 2u * (size_t)np * 128u; }
// two CTAs per SM (each up to ~110 KB of stages), at least 2 stages: the
// tiles of a launch then fit one wave instead of 1.7 at one CTA per SM
__host__ inline int umma_stages(int np) {
  const size_t sb = umma_stage_bytes(np);
  int s = (int)((110u * 1024u) / sb);
  return s > 4 ? 4 : (s < 2 ? 2 : s);
}
__host__ inline size_t umma_smem_bytes(int np) {
  return 1024 + (size_t)umma_stages(np) * umma_stage_bytes(np) + 256;
}

// One 128-row tile at row m0.  The tensor maps are kernel parameters (one
// system per launch) or 64-byte-aligned objects in global memory written
// before the launch (several systems per launch).
__device__ __forceinline__ void lcao_tf32x3_tile(const CUtensorMap *ta_hi, const CUtensorMap *ta_lo,
                                                 const CUtensorMap *tb_hi, const CUtensorMap *tb_lo, int M, int K,
                                                 int np, int nc, int stages, double *__restrict__ C, int ldc,
                                                 int *err, const int m0) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *sb = smem_raw + (base - raw);
  const uint32_t a_bytes = 128u * 128u, b_bytes = (uint32_t)np * 128u;
  const uint32_t stage_bytes = 2u * a_bytes + 2u * b_bytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(sb + (size_t)stages * stage_bytes);
  uint64_t *empty = full + stages;
  uint64_t *done = empty + stages;
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(done + 1);
  volatile int *s_abort = reinterpret_cast<volatile int *>(s_tmem + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (K + 31) / 32;
  const uint32_t ncols = np <= 32 ? 32u : np <= 64 ? 64u : np <= 128 ? 128u : 256u;

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  if (warp == 0 && lane == 0) {
    // producer
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % stages, u = kb / stages;
      if (u > 0 && !mbar_wait(&empty[s], (uint32_t)((u - 1) & 1))) {
        *s_abort = 1;
        atomicOr(err, 1);
        break;
      }
      if (*s_abort) break;
      uint8_t *st = sb + (size_t)s * stage_bytes;
      mbar_expect_tx(&full[s], stage_bytes);
      tma_load_2d(st, ta_hi, &full[s], kb * 32, m0);
      tma_load_2d(st + a_bytes, ta_lo, &full[s], kb * 32, m0);
      tma_load_2d(st + 2 * a_bytes, tb_hi, &full[s], kb * 32, 0);
      tma_load_2d(st + 2 * a_bytes + b_bytes, tb_lo, &full[s], kb * 32, 0);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t idesc = idesc_tf32(np);
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % stages, u = kb / stages;
      if (!mbar_wait(&full[s], (uint32_t)(u & 1))) {
        *s_abort = 1;
        atomicOr(err, 2);
        break;
      }
      tc_fence_after();
      const uint32_t st = base + (uint32_t)s * stage_bytes;
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const uint64_t ahi = sdesc_k_sw128(st + kk * 32), alo = sdesc_k_sw128(st + a_bytes + kk * 32);
        const uint64_t bhi = sdesc_k_sw128(st + 2 * a_bytes + kk * 32);
        const uint64_t blo = sdesc_k_sw128(st + 2 * a_bytes + b_bytes + kk * 32);
        umma_tf32(tmem, ahi, bhi, idesc, (kb | kk) != 0 ? 1u : 0u);
        umma_tf32(tmem, ahi, blo, idesc, 1u);
        umma_tf32(tmem, alo, bhi, idesc, 1u);
      }
      umma_commit(&empty[s]);
    }
    // arrives once every MMA issued above has completed (at once if none)
    umma_commit(done);
  }
  __syncwarp();
  // epilogue: the accumulator is complete when `done` arrives
  const bool finished = mbar_wait(done, 0u);
  if (!finished) atomicOr(err, 4);
  // one decision for the whole CTA: tcgen05.ld is warp-collective
  const int go = __syncthreads_and(finished && !*s_abort);
  tc_fence_after();
  if (go) {
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < np; c0 += 16) {
      uint32_t v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (row < M) {
        double *out = C + (size_t)row * ldc;
#pragma unroll
        for (int j = 0; j < 16; j++)
          if (c0 + j < nc) out[c0 + j] = (double)__uint_as_float(v[j]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}
__global__ void __launch_bounds__(128, 2)
    k_lcao_tf32x3(const __grid_constant__ CUtensorMap ta_hi, const __grid_constant__ CUtensorMap ta_lo,
                  const __grid_constant__ CUtensorMap tb_hi, const __grid_constant__ CUtensorMap tb_lo, int M, int K,
                  int np, int nc, int stages, double *__restrict__ C, int ldc, int *err) {
  lcao_tf32x3_tile(&ta_hi, &ta_lo, &tb_hi, &tb_lo, M, K, np, nc, stages, C, ldc, err, blockIdx.x * 128);
}

}  // namespace cw
