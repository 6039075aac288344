// ragged.cuh — one launch per move stage for the walkers of many systems.
//
// A ragged batch holds systems of different electron, centre, basis and
// orbital counts (config 3's 64 molecules of 8-200 electrons).  Electron k of
// every system with more than k electrons moves in the same six launches
// (proposal, move Jastrow, basis, LCAO, decision, commit); the systems are
// sorted by electron count, so the systems still moving at step k are a
// prefix of the slot array, and every launch's grid is that prefix's share
// of a precomputed block map.  Each block reads its (system, block-in-system)
// pair from the map, its system's constant block from global memory and runs
// the same body as the one-system kernels (move.cuh), so every system takes
// the walk it takes alone: the same streams and decisions, bitwise in mixed
// precision, to rounding in FP64 (the FP64 bodies read the constant block
// from global memory here and from the parameter space alone, and the
// compiler contracts a different set of multiply-adds).  The LCAO launch is a
// grouped GEMM over (system, row tile, column tile) work items; the commit is
// a persistent launch over the concatenated accepted-walker lists.
#pragma once
#include "move.cuh"
#include "hpsi.cuh"
#include "gemm.cuh"
#include "umma.cuh"

namespace cw {

constexpr int kRagMaxSlots = 256;

// One system of a ragged batch.
struct RagSlot {
  WState st;
  MoveBuf mb;
  GSys g;
  int *acc_list, *acc_count; // accepted walkers of the current move
  int W, K, Oa;              // move LCAO: phi [4W][K] x coefT [K][Oa] -> orbn
  const CUtensorMap *tm;     // mixed precision: A_hi, A_lo, B_hi, B_lo of the move LCAO
  int np, stages;            // mixed precision: padded orbital count, pipeline stages
  int *err;                  // mixed precision: the system's tensor-core error flags
};

// Work item of the grouped LCAO: slot, kind (0: FP64 tensor-core tile,
// 1: SIMT tile, 2: TF32x3 tcgen05 tile), first row, first column.
struct RagTile {
  int slot, kind, m0, n0;
};

// SIMT tile of the grouped FP64 LCAO (128 threads)
constexpr int kRagSimtBM = 64, kRagSimtBN = 16, kRagSimtBK = 16;

__global__ void __launch_bounds__(128) k_rotqua_rag(const CSys *__restrict__ csa, const RagSlot *__restrict__ sl, const int2 *__restrict__ map) {
  const int2 e = map[blockIdx.x];
  const RagSlot &s = sl[e.x];
  const WState st = s.st;
  rotqua_body(csa[e.x], st, e.y);
}

__global__ void __launch_bounds__(128) k_propose_rag(const CSys *__restrict__ csa, const RagSlot *__restrict__ sl, const int2 *__restrict__ map,
                                                     int iel) {
  const int2 e = map[blockIdx.x];
  const RagSlot &s = sl[e.x];
  const WState st = s.st;
  const MoveBuf mb = s.mb;
  propose_body(csa[e.x], st, mb, iel, s.acc_count, e.y);
}

template <int NORD>
__global__ void __launch_bounds__(128, 5) k_jastrow_move_rag(const CSys *__restrict__ csa, const RagSlot *__restrict__ sl,
                                                             const int2 *__restrict__ map, int iel) {
  const int2 e = map[blockIdx.x];
  const RagSlot &s = sl[e.x];
  const WState st = s.st;
  const MoveBuf mb = s.mb;
  jastrow_move_body<NORD>(csa[e.x], st, mb, iel, e.y);
}

template <int NORD, int P>
__global__ void __launch_bounds__(128, P == 1 ? 8 : (P == 2 ? 4 : 3))
    k_jastrow_move_f32_rag(const CSys *__restrict__ csa, const RagSlot *__restrict__ sl, const int2 *__restrict__ map, int iel) {
  const int2 e = map[blockIdx.x];
  const RagSlot &s = sl[e.x];
  const WState st = s.st;
  const MoveBuf mb = s.mb;
  jastrow_move_f32_body<NORD, P>(csa[e.x], st, mb, iel, e.y);
}

__global__ void k_basis_move_rag(const CSys *__restrict__ csa, const RagSlot *__restrict__ sl, const int2 *__restrict__ map) {
  const int2 e = map[blockIdx.x];
  const RagSlot &s = sl[e.x];
  const WState st = s.st;
  const MoveBuf mb = s.mb;
  const GSys g = s.g;
  basis_move_body(csa[e.x], st, mb, g, e.y);
}

__global__ void __launch_bounds__(128) k_decide_rag(const CSys *__restrict__ csa, const RagSlot *__restrict__ sl, const int2 *__restrict__ map,
                                                    int iel) {
  const int2 e = map[blockIdx.x];
  const RagSlot &s = sl[e.x];
  const WState st = s.st;
  const MoveBuf mb = s.mb;
  const GSys g = s.g;
  decide_body(csa[e.x], st, mb, g, iel, s.acc_list, s.acc_count, e.y);
}

// FP64 LCAO of the moved electron for every system: a 128 x BN tensor-core
// tile where the system's shape allows it (as dgemm picks for the system
// alone), a 64 x 16 SIMT tile otherwise.  Dynamic shared memory: mma_smem(BN).
template <int BN>
__global__ void __launch_bounds__(128, 2) k_lcao_rag(const RagSlot *__restrict__ sl,
                                                     const RagTile *__restrict__ tiles) {
  extern __shared__ __align__(16) double gsm[];
  const RagTile t = tiles[blockIdx.x];
  const RagSlot &s = sl[t.slot];
  const int M = 4 * s.W, N = s.Oa, K = s.K;
  const double *A = s.mb.phi, *B = s.g.coefT;
  double *C = s.mb.orbn;
  if (t.kind == 0) {
    dgemm_mma_tile<BN>(M, N, K, A, B, C, t.m0, t.n0, gsm);
  } else {
    constexpr int BM = kRagSimtBM, BNS = kRagSimtBN, BK = kRagSimtBK;
    auto As = reinterpret_cast<double(*)[BK][BM + 2]>(gsm);
    auto Bs = reinterpret_cast<double(*)[BK][BNS]>(gsm + 2 * BK * (BM + 2));
    dgemm_simt_tile<BM, BNS, BK, BM * BNS / 128, 1>(M, N, K, A, B, C, t.m0, t.n0, As, Bs);
  }
}

// Mixed precision: the TF32x3 tcgen05 tile of every system's 128-row block,
// the tensor maps read from global memory.  Dynamic shared memory: the
// largest of the systems' umma_smem_bytes.
__global__ void __launch_bounds__(128, 2) k_lcao_tf32x3_rag(const RagSlot *__restrict__ sl,
                                                            const RagTile *__restrict__ tiles) {
  const RagTile t = tiles[blockIdx.x];
  const RagSlot &s = sl[t.slot];
  const CUtensorMap *tm = s.tm;
  if (threadIdx.x == 0) {
    // the maps were written to global memory by a copy: make them visible
    // to the tensor-map proxy of the producer thread (thread 0)
#pragma unroll
    for (int q = 0; q < 4; q++)
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tm + q) : "memory");
  }
  lcao_tf32x3_tile(tm + 0, tm + 1, tm + 2, tm + 3, 4 * s.W, s.K, s.np, s.Oa, s.stages, s.mb.orbn, s.Oa, s.err,
                   t.m0);
}

// detsav + jassav of the accepted walkers of the first `nslot` systems: a
// fixed grid of blocks over their concatenated lists (each block adds up the
// lists' lengths first).  Dynamic shared memory: the largest system's
// commit_tile_walker share.
__global__ void __launch_bounds__(128) k_commit_rag(const CSys *__restrict__ csa, const RagSlot *__restrict__ sl, int nslot, int iel) {
  __shared__ int s_off[kRagMaxSlots + 1];
  __shared__ int s_warp[4];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  // exclusive scan of the list lengths, 128 slots per pass
  int carry = 0;
  for (int base = 0; base < nslot; base += 128) {
    const int i = base + tid;
    const int v = i < nslot ? *sl[i].acc_count : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    int before = carry;
    for (int q = 0; q < wid; q++) before += s_warp[q];
    if (i < nslot) s_off[i] = before + x - v;
    const int total = s_warp[0] + s_warp[1] + s_warp[2] + s_warp[3];
    __syncthreads();
    carry += total;
  }
  if (tid == 0) s_off[nslot] = carry;
  __syncthreads();
  const int total = s_off[nslot];
  int k = 0;
  for (int q = blockIdx.x; q < total; q += gridDim.x) {
    while (q >= s_off[k + 1]) k++;
    const RagSlot &s = sl[k];
    WState st = s.st;
    const MoveBuf mb = s.mb;
    const GSys g = s.g;
    commit_tile_walker(csa[k], st, mb, g, s.acc_list[q - s_off[k]], iel);
    __syncthreads();  // the next walker reuses the shared memory
  }
}

}  // namespace cw
