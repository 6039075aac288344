// gemm.cuh — FP64 LCAO contraction C[M][N] = A[M][K] * B[K][N] (row-major).
//
// A holds basis-function rows (value/gradient/Laplacian of one electron of
// one walker per row), B the LCAO coefficients (basis x orbital), C the
// orbitals.  128x64 output tile per CTA, 128 threads, 8x8 register tile (16
// shared-memory doubles per 64 FMAs: the FP64 FMA rate of an SM needs at
// most one shared double per 4 FMAs), 8-deep K slices staged in shared
// memory (rows padded by 2 doubles: conflict-free transposed stores, 16-byte
// aligned vector loads) with a register prefetch of the next slice.  This
// SIMT kernel serves the shapes the FP64 tensor-core kernel below does not
// (odd K or N, N <= 16).
#pragma once
#include "common.cuh"

namespace cw {

// One BM x BN output tile at (m0, n0); As/Bs: the two-stage shared slices.
// Every output element sums its K terms in order, one FMA each, whatever the
// tile shape.
template <int BM, int BN, int BK, int TM, int TN>
__device__ __forceinline__ void dgemm_simt_tile(int M, int N, int K, const double *__restrict__ A,
                                                const double *__restrict__ B, double *__restrict__ C, int m0, int n0,
                                                double (*As)[BK][BM + 2], double (*Bs)[BK][BN]) {
  constexpr int NT = (BM / TM) * (BN / TN);
  const int tid = threadIdx.x;
  const int tx = tid % (BN / TN), ty = tid / (BN / TN);
  double acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) acc[i][j] = 0.0;

  constexpr int A_PER = BM * BK / NT;  // elements of the A slice per thread
  constexpr int B_PER = BK * BN / NT;
  double ra[A_PER], rb[B_PER];
  auto loadA = [&](int k0) {
#pragma unroll
    for (int r = 0; r < A_PER; r++) {
      const int idx = tid + r * NT;
      const int mm = idx / BK, kk = idx % BK;
      const int gm = m0 + mm, gk = k0 + kk;
      ra[r] = (gm < M && gk < K) ? __ldg(A + (size_t)gm * K + gk) : 0.0;
    }
  };
  auto loadB = [&](int k0) {
#pragma unroll
    for (int r = 0; r < B_PER; r++) {
      const int idx = tid + r * NT;
      const int kk = idx / BN, nn = idx % BN;
      const int gk = k0 + kk, gn = n0 + nn;
      rb[r] = (gk < K && gn < N) ? __ldg(B + (size_t)gk * N + gn) : 0.0;
    }
  };
  auto storeS = [&](int buf) {
#pragma unroll
    for (int r = 0; r < A_PER; r++) {
      const int idx = tid + r * NT;
      As[buf][idx % BK][idx / BK] = ra[r];
    }
#pragma unroll
    for (int r = 0; r < B_PER; r++) {
      const int idx = tid + r * NT;
      Bs[buf][idx / BN][idx % BN] = rb[r];
    }
  };
  loadA(0);
  loadB(0);
  storeS(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < K; k0 += BK) {
    const bool more = k0 + BK < K;
    if (more) {
      loadA(k0 + BK);
      loadB(k0 + BK);
    }
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      double a[TM], b[TN];
      if constexpr (TM % 2 == 0 && TN % 2 == 0) {
        const double2 *pa = reinterpret_cast<const double2 *>(&As[buf][kk][ty * TM]);
        const double2 *pb = reinterpret_cast<const double2 *>(&Bs[buf][kk][tx * TN]);
#pragma unroll
        for (int i = 0; i < TM / 2; i++) {
          const double2 v = pa[i];
          a[2 * i] = v.x;
          a[2 * i + 1] = v.y;
        }
#pragma unroll
        for (int j = 0; j < TN / 2; j++) {
          const double2 v = pb[j];
          b[2 * j] = v.x;
          b[2 * j + 1] = v.y;
        }
      } else {
#pragma unroll
        for (int i = 0; i < TM; i++) a[i] = As[buf][kk][ty * TM + i];
#pragma unroll
        for (int j = 0; j < TN; j++) b[j] = Bs[buf][kk][tx * TN + j];
      }
#pragma unroll
      for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (more) {
      storeS(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
#pragma unroll
  for (int i = 0; i < TM; i++) {
    const int gm = m0 + ty * TM + i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < TN; j++) {
      const int gn = n0 + tx * TN + j;
      if (gn < N) C[(size_t)gm * N + gn] = acc[i][j];
    }
  }
}
template <int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
k_dgemm(int M, int N, int K, const double *__restrict__ A, const double *__restrict__ B, double *__restrict__ C) {
  __shared__ __align__(16) double As[2][BK][BM + 2];
  __shared__ __align__(16) double Bs[2][BK][BN];
  dgemm_simt_tile<BM, BN, BK, TM, TN>(M, N, K, A, B, C, blockIdx.x * BM, blockIdx.y * BN, As, Bs);
}

// ---------------------------------------------------------------------------
// FP64 tensor-core variant (mma.sync m16n8k4 .f64; tcgen05 has no FP64 kind):
// 128 x BN output tile per CTA, 4 warps of 32 x BN (2 x BN/8 m16n8
// accumulators in registers), 16-deep K slices in a 3-stage cp.async ring.
// Shared rows are padded (A: 20 doubles, B: BN + 4) so that the fragment
// loads of a half-warp hit 16 distinct 8-byte bank pairs.  Needs K and N even
// (16-byte row chunks); out-of-range chunks are zero-filled by the copy.  BN
// (32, 48, 64 or 80 orbitals) is picked per context by timing (cw_autotune);
// every output element sums its K slices in the same order whatever the tile.
// ---------------------------------------------------------------------------
constexpr int kMmaBM = 128, kMmaBK = 16, kMmaSA = kMmaBK + 4, kMmaStages = 3;
constexpr size_t mma_smem(int bn) {
  return sizeof(double) * (size_t)kMmaStages * (kMmaBM * kMmaSA + kMmaBK * (bn + 4));
}

__device__ __forceinline__ void cp_async16(double *dst, const double *src, int bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory");
}
__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], const double (&a)[2], double b) {
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a[0]), "d"(a[1]), "d"(b));
}

// One 128 x BN output tile at (m0, n0); gsm: mma_smem(BN) bytes of shared memory
template <int BN>
__device__ __forceinline__ void dgemm_mma_tile(int M, int N, int K, const double *__restrict__ A,
                                               const double *__restrict__ B, double *__restrict__ C, int m0, int n0,
                                               double *gsm) {
  constexpr int BM = kMmaBM, BK = kMmaBK, SA = kMmaSA, SB = BN + 4, ST = kMmaStages, NI = BN / 8;
  double *As = gsm;                          // [ST][BM][SA]
  double *Bs = gsm + (size_t)ST * BM * SA;   // [ST][BK][SB]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int nk = (K + BK - 1) / BK;
  auto load_stage = [&](int kt, int s) {
    const int k0 = kt * BK;
#pragma unroll
    for (int c = tid; c < BM * (BK / 2); c += 128) {
      const int r = c / (BK / 2), kc = (c % (BK / 2)) * 2;
      const int gm = m0 + r, gk = k0 + kc;
      const bool ok = gm < M && gk < K;
      cp_async16(As + ((size_t)s * BM + r) * SA + kc, ok ? A + (size_t)gm * K + gk : A, ok ? 16 : 0);
    }
#pragma unroll
    for (int c = tid; c < BK * (BN / 2); c += 128) {
      const int r = c / (BN / 2), nc = (c % (BN / 2)) * 2;
      const int gk = k0 + r, gn = n0 + nc;
      const bool ok = gk < K && gn < N;
      cp_async16(Bs + ((size_t)s * BK + r) * SB + nc, ok ? B + (size_t)gk * N + gn : B, ok ? 16 : 0);
    }
  };
  double acc[2][NI][4];
#pragma unroll
  for (int mi = 0; mi < 2; mi++)
#pragma unroll
    for (int ni = 0; ni < NI; ni++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[mi][ni][q] = 0.0;
#pragma unroll
  for (int s = 0; s < ST - 1; s++) {
    if (s < nk) load_stage(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; kt++) {
    cp_async_wait<ST - 2>();
    __syncthreads();  // slice kt landed for every thread; slice kt-1's stage is free
    if (kt + ST - 1 < nk) load_stage(kt + ST - 1, (kt + ST - 1) % ST);
    cp_async_commit();
    const double *as = As + ((size_t)(kt % ST) * BM + warp * 32) * SA;
    const double *bs = Bs + (size_t)(kt % ST) * BK * SB;
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      double a[2][2], b[NI];
#pragma unroll
      for (int mi = 0; mi < 2; mi++) {
        a[mi][0] = as[(mi * 16 + g) * SA + k4 + t];
        a[mi][1] = as[(mi * 16 + g + 8) * SA + k4 + t];
      }
#pragma unroll
      for (int ni = 0; ni < NI; ni++) b[ni] = bs[(k4 + t) * SB + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < NI; ni++) dmma_16x8x4(acc[mi][ni], a[mi], b[ni]);
    }
  }
  cp_async_wait<0>();
  // accumulator (mi, ni): rows m0 + warp*32 + mi*16 + g (+8), columns n0 + ni*8 + 2t (+1)
#pragma unroll
  for (int mi = 0; mi < 2; mi++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int gm = m0 + warp * 32 + mi * 16 + g + 8 * h;
      if (gm >= M) continue;
#pragma unroll
      for (int ni = 0; ni < NI; ni++) {
        const int gn = n0 + ni * 8 + 2 * t;
        if (gn < N) *reinterpret_cast<double2 *>(C + (size_t)gm * N + gn) = make_double2(acc[mi][ni][2 * h], acc[mi][ni][2 * h + 1]);
      }
    }
  }
}
template <int BN>
__global__ void __launch_bounds__(128, 2)
k_dgemm_mma(int M, int N, int K, const double *__restrict__ A, const double *__restrict__ B, double *__restrict__ C) {
  extern __shared__ __align__(16) double gsm[];
  dgemm_mma_tile<BN>(M, N, K, A, B, C, blockIdx.x * kMmaBM, blockIdx.y * BN, gsm);
}

// N tiles of the tensor-core GEMM the autotuner chooses from
constexpr int kMmaTiles[4] = {32, 48, 64, 80};

template <int BN>
inline void launch_dgemm_mma(cudaStream_t s, int M, int N, int K, const double *A, const double *B, double *C) {
  dim3 grid((M + kMmaBM - 1) / kMmaBM, (N + BN - 1) / BN);
  k_dgemm_mma<BN><<<grid, 128, mma_smem(BN), s>>>(M, N, K, A, B, C);
}

// bn: N tile of the tensor-core kernel (one of kMmaTiles)
inline void dgemm(cudaStream_t s, int M, int N, int K, const double *A, const double *B, double *C, int bn = 64) {
  const bool al16 = ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(C)) & 15) == 0;
  if (N > 16 && (K % 2) == 0 && (N % 2) == 0 && al16) {
    switch (bn) {
      case 32: launch_dgemm_mma<32>(s, M, N, K, A, B, C); break;
      case 48: launch_dgemm_mma<48>(s, M, N, K, A, B, C); break;
      case 80: launch_dgemm_mma<80>(s, M, N, K, A, B, C); break;
      default: launch_dgemm_mma<64>(s, M, N, K, A, B, C); break;
    }
  } else if (N <= 16) {
    constexpr int BM = 64, BN = 16, BK = 16, TM = 4, TN = 1;
    dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN);
    k_dgemm<BM, BN, BK, TM, TN><<<grid, (BM / TM) * (BN / TN), 0, s>>>(M, N, K, A, B, C);
  } else {
    constexpr int BM = 128, BN = 64, BK = 8, TM = 8, TN = 8;
    dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN);
    k_dgemm<BM, BN, BK, TM, TN><<<grid, (BM / TM) * (BN / TN), 0, s>>>(M, N, K, A, B, C);
  }
}

}  // namespace cw
