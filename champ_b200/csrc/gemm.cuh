// gemm.cuh — FP64 LCAO contraction C[M][N] = A[M][K] * B[K][N] (row-major).
//
// A holds basis-function rows (value/gradient/Laplacian of one electron of
// one walker per row), B the LCAO coefficients (basis x orbital), C the
// orbitals.  128x64 output tile per CTA, 128 threads, 8x8 register tile (16
// shared-memory doubles per 64 FMAs: the FP64 FMA rate of an SM needs at
// most one shared double per 4 FMAs), 8-deep K slices staged in shared
// memory (rows padded by 2 doubles: conflict-free transposed stores, 16-byte
// aligned vector loads) with a register prefetch of the next slice.  FP64
// SIMT: the B200 has no FP64 tensor-core path wider than its FMA units.
#pragma once
#include "common.cuh"

namespace cw {

template <int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
k_dgemm(int M, int N, int K, const double *__restrict__ A, const double *__restrict__ B, double *__restrict__ C) {
  constexpr int NT = (BM / TM) * (BN / TN);
  __shared__ __align__(16) double As[2][BK][BM + 2];
  __shared__ __align__(16) double Bs[2][BK][BN];
  const int tid = threadIdx.x;
  const int tx = tid % (BN / TN), ty = tid / (BN / TN);
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
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

inline void dgemm(cudaStream_t s, int M, int N, int K, const double *A, const double *B, double *C) {
  if (N <= 16) {
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
