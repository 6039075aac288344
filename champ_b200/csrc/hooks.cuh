// hooks.cuh — per-electron routines for a driver that keeps metrop6 (or its
// own move loop) on the host: the point of a move is given by the caller,
// the engine evaluates psie there, the drift at the old or the new position,
// and commits the moves the caller accepted.  Every kernel runs over all
// walkers of the population; the move tables are those of the engine's own
// sweep (MoveBuf), filled by the same Jastrow, basis and LCAO kernels.
#pragma once
#include "common.cuh"
#include "move.cuh"

namespace cw {

// The caller's point for electron iel of every walker: xnew [W][3].  The
// nearest centre (metrop6's rminn, nearestn, rvminn, kept for the next
// proposal around it) is found as the reference does (first minimum of the
// squared distance, vmc/metrop_mov1_slat.f90:327-340).
__global__ void k_hook_place(const __grid_constant__ CSys cs, WState st, MoveBuf mb, const double *__restrict__ xnew) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= st.W) return;
  MoveScratch &m = mb.ms[w];
  const double x0 = xnew[3 * w], x1 = xnew[3 * w + 1], x2 = xnew[3 * w + 2];
  double best = 99.0e9;
  int nb = 0;
  for (int j = 0; j < cs.M; j++) {
    const double d0 = x0 - cs.cent[3 * j], d1 = x1 - cs.cent[3 * j + 1], d2 = x2 - cs.cent[3 * j + 2];
    const double d = d0 * d0 + d1 * d1 + d2 * d2;
    if (d < best) {
      best = d;
      nb = j;
    }
  }
  m.xnew[0] = x0;
  m.xnew[1] = x1;
  m.xnew[2] = x2;
  m.nearestn = nb;
  m.rminn = sqrt(best);
  m.rvminn[0] = x0 - cs.cent[3 * nb];
  m.rvminn[1] = x1 - cs.cent[3 * nb + 1];
  m.rvminn[2] = x2 - cs.cent[3 * nb + 2];
  m.igeo = 0;
  m.acc = 0;
}

// psie's values at the point (vmc/hpsie.f90:3): the determinant ratio of the
// moved electron's new orbital row (determinante, vmc/determinante.f90:40-46,
// the same group dot product as k_decide), psi_D at the point and J there.
// out [W][2] = (psid, psij).  kMoveGroup lanes per walker.
__global__ void __launch_bounds__(128) k_hook_ratio(const __grid_constant__ CSys cs, WState st, MoveBuf mb, GSys g, int iel, double *out) {
  const int lane = threadIdx.x & (kMoveGroup - 1);
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) / kMoveGroup;
  if (w >= st.W) return;
  const int nmax = cs.nmax, Oa = cs.Oa;
  int iab, nel, ish;
  spin_of(cs, iel, iab, nel, ish);
  const int iloc = iel - ish;
  const double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax + (size_t)nel * iloc;
  const double *orbn = mb.orbn + (size_t)w * 4 * Oa;
  const int *slot = g.slot_orb + iab * nmax;
  double ratio = 0;
  for (int j = lane; j < nel; j += kMoveGroup) ratio += sl[j] * orbn[slot[j]];
  ratio = group_sum(ratio);
  const double detn = st.detiab[2 * w + iab] * ratio;
  const double psidn = mb.md_psidn ? mb.md_psidn[w] : detn * st.detiab[2 * w + (1 - iab)] * cs.cdet;
  if (lane != 0) return;
  MoveScratch &m = mb.ms[w];
  m.ratio = ratio;
  m.psidn = psidn;
  out[2 * w] = psidn;
  out[2 * w + 1] = mb.fsumn[w];
}

// compute_determinante_grad (vmc/determinante.f90:69) for electron iel:
// iflag_move = 1 at the current position (slmi column . dorb + the Jastrow
// gradient, + the multideterminant correction), 0 at the point of the last
// psie (the updated inverse column slmi/ratio . the new orbital gradients).
// The sums run in the order of k_propose and k_decide.  out [W][3].
__global__ void __launch_bounds__(128) k_hook_grad(const __grid_constant__ CSys cs, WState st, MoveBuf mb, GSys g, int iel, int iflag_move,
                                                   double *out) {
  const int lane = threadIdx.x & (kMoveGroup - 1);
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) / kMoveGroup;
  if (w >= st.W) return;
  const int N = cs.N, nmax = cs.nmax, Oa = cs.Oa;
  int iab, nel, ish;
  spin_of(cs, iel, iab, nel, ish);
  const int iloc = iel - ish;
  const double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax + (size_t)nel * iloc;
  double v[3];
  if (iflag_move == 1) {
    const double *d0p = st.dorbs + (((size_t)w * 3 + 0) * N + iel) * nmax;
    const double *d1p = st.dorbs + (((size_t)w * 3 + 1) * N + iel) * nmax;
    const double *d2p = st.dorbs + (((size_t)w * 3 + 2) * N + iel) * nmax;
    double g0 = 0, g1 = 0, g2 = 0;
    for (int j = lane; j < nel; j += kMoveGroup) {
      const double s = sl[j];
      g0 += s * d0p[j];
      g1 += s * d1p[j];
      g2 += s * d2p[j];
    }
    g0 = group_sum(g0);
    g1 = group_sum(g1);
    g2 = group_sum(g2);
    const double *fjo = st.fjo + (size_t)w * 3 * N;
    const double *mv = mb.md_velo ? mb.md_velo + 3 * w : nullptr;
    v[0] = (mv ? mv[0] : 0.0) + g0 + fjo[0 * N + iel];
    v[1] = (mv ? mv[1] : 0.0) + g1 + fjo[1 * N + iel];
    v[2] = (mv ? mv[2] : 0.0) + g2 + fjo[2 * N + iel];
  } else {
    const double ratio = mb.ms[w].ratio;
    const double *orbn = mb.orbn + (size_t)w * 4 * Oa;
    const int *slot = g.slot_orb + iab * nmax;
    double v0 = 0, v1 = 0, v2 = 0;
    if (ratio != 0.0) {
      for (int j = lane; j < nel; j += kMoveGroup) {
        const double sc = sl[j] / ratio;
        v0 += sc * orbn[1 * Oa + slot[j]];
        v1 += sc * orbn[2 * Oa + slot[j]];
        v2 += sc * orbn[3 * Oa + slot[j]];
      }
    }
    v0 = group_sum(v0);
    v1 = group_sum(v1);
    v2 = group_sum(v2);
    const double *mv = mb.md_veln ? mb.md_veln + 3 * w : nullptr;
    v[0] = (mv ? mv[0] : 0.0) + v0 + mb.vjn[3 * w + 0];
    v[1] = (mv ? mv[1] : 0.0) + v1 + mb.vjn[3 * w + 1];
    v[2] = (mv ? mv[2] : 0.0) + v2 + mb.vjn[3 * w + 2];
  }
  if (lane != 0) return;
  out[3 * w] = v[0];
  out[3 * w + 1] = v[1];
  out[3 * w + 2] = v[2];
}

// metrop6's accept branch for the walkers whose flag is set
// (vmc/metrop_mov1_slat.f90:592-619): the new position, psi, the nearest
// centre and the determinant take the point's values; k_commit then applies
// detsav and jassav to those walkers (the others keep their tables, which
// is distancese_restore: the engine never overwrote them).
__global__ void k_hook_accept(const __grid_constant__ CSys cs, WState st, MoveBuf mb, int iel, const int *__restrict__ accept) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= st.W) return;
  MoveScratch &m = mb.ms[w];
  const int acc = accept[w] != 0;
  m.acc = acc;
  if (!acc) return;
  const int N = cs.N;
  const int iab = iel < cs.nup ? 0 : 1;
  const double fsumn = mb.fsumn[w];
  st.psi2o[w] = log(fabs(mb.md_psi2g ? mb.md_psi2g[w] : 1.0)) + 2 * (log(fabs(m.psidn)) + fsumn);
  st.psido[w] = m.psidn;
  st.psijo[w] = fsumn;
  st.fsumo[w] = fsumn;
  st.detiab[2 * w + iab] = st.detiab[2 * w + iab] * m.ratio;
  st.rmino[(size_t)w * N + iel] = m.rminn;
  st.nearesto[(size_t)w * N + iel] = m.nearestn;
  for (int k = 0; k < 3; k++) {
    st.rvmino[((size_t)w * 3 + k) * N + iel] = m.rvminn[k];
    st.x[((size_t)w * 3 + k) * N + iel] = m.xnew[k];
  }
}

}  // namespace cw
