// hpsi.cuh — full local energy of every walker, hpsi (vmc/hpsi.f90:3).
//
//   k_jastrow_full   jastrow_factor4 (vmc/jastrow4.f90:3) + e-e Coulomb sum
//   k_basis_all      basis_fns ider=2 for a chunk of electrons
//   gemm             LCAO (vmc/orbitals_no_qmckl.f90:19)
//   k_scatter_orbs   Slater columns of each electron (determinant.f90:40-49)
//   k_slater_inv     matinv + ddx/d2dx2 (vmc/determinant.f90:50-70, matinv.f90:22)
//   k_ctilde         c~(i,m) = sum_j slmi(j,i) coef(m,occ_j): ratio vectors of
//                    nonlocd_quad (vmc/nonloc.f90:462) contracted once per electron
//   k_ecp            getvps_gauss + nonloc quadrature (vmc/nonloc_pot.f90:3,
//                    vmc/nonloc.f90:5, nonlocj_quad4 :656)
//   k_energy         E_L assembly (vmc/hpsi.f90:176-246) and metrop6 sums
#pragma once
#include <type_traits>

#include "common.cuh"

namespace cw {

struct HBuf {
  double *d2o;      // [W]
  double *pe_ee;    // [W]   sum 1/r_ij
  double *pe_ecp;   // [W]   local ECP part (or -Z/r for nloc=0)
  double *vpsp;     // [W][2]
  double *ddx;      // [W][N][4]  ddx(3), d2dx2
  double *ddorbs;   // [W][N][nmax]
  double *phi;      // [rows][K] chunk basis
  double *orball;   // [rows][Oa] chunk orbitals
  double *ctilde;   // [W][N][K]
  double *entab;    // [W][5][M][N] e-n table of the full Jastrow (k_jastrow_full)
  float *entabf;    // [W][5][M][N] its FP32 copy, partner side of the mixed path (null in FP64)
  int chunk;        // electrons per chunk
  float *phi_hi, *phi_lo;  // mixed precision: [rows][kp] split chunk basis (null in FP64)
  int kp;
  double *tvpsp;           // [W][N][nquad][M] T-move matrix elements (null without T-moves)
  double *ecp_rr;          // [W][N][M|1] k_ecp's scaled e-n distances where they do not fit shared memory (else null)
  double *tvtrj;           // [W][N][nquad][M] radial x Jastrow factor of each T-move element (multideterminant T-moves, else null)
  // multideterminant (null for one determinant)
  double *md_P;            // [W][N][K] pseudopotential quadrature basis sums
  const double *md_den;    // [W][2] energy / kinetic corrections
  const double *md_S;      // [W]    psi_D / (D_ref^up D_ref^dn)
  // several states (null for one): per state S, corrections, and outputs
  const double *md_S_ms;   // [W][nstates]
  const double *md_den_ms; // [W][nstates][2]
  double *e_ms, *psid_ms;  // [W][nstates] local energy and psi_D of the last hpsi
  double *sums_ms;         // [W][nstates][4] block sums: w, w E, w (E - T), w T
};

__device__ __forceinline__ void pair_of(long p, int &i, int &j) {
  // p = i*(i-1)/2 + j, 0 <= j < i
  int ii = (int)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
  while ((long)ii * (ii - 1) / 2 > p) ii--;
  while ((long)(ii + 1) * ii / 2 <= p) ii++;
  i = ii;
  j = (int)(p - (long)ii * (ii - 1) / 2);
}

template <int BS>
__device__ __forceinline__ double block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int k = 0; k < BS / 32; k++) r += red[k];
  return r;  // valid on thread 0
}

// ---------------------------------------------------------------------------
// jastrow_factor4 (vmc/jastrow4.f90:3): CTA per walker.
//  1. thread per electron over the centres: the e-n table (scaled distance,
//     its derivative factors, r^2) in structure-of-arrays form, the move
//     kernels' e-n table, and the e-n terms;
//  2. pair rows i and N-1-i together (N-1 pairs per batch): the row
//     electron's e-e-n coefficients are folded per centre (value, d/dx,
//     d2/dx2) into shared memory with its table entries, then threads over
//     the batch's pairs evaluate every centre from the folded coefficients;
//     the table stores d rr/dr divided by r, so the pair-centre loop has no
//     division;
//  3. per-electron gradient sums (warp per row) and block sums.
// ---------------------------------------------------------------------------
// e-n table fields ([W][kEnFields][M][N]): scaled distance rr, -kappa rr',
// -kappa rr'', -kappa rr'/r, r^2
constexpr int kEnFields = 5;

// T is the arithmetic of the pair and e-e-n terms (double: parity path,
// float: mixed path); distances, 1/r_ij, the tables and the sums over
// pairs stay FP64.  Four CTAs per SM in both arithmetics (the FP32 build at
// five spilled and ran 9% slower).
template <int NORD, typename T>
// blocks per SM: six for FP32 (80 registers, 26.2 -> 24.3 ms per 8192-walker
// sweep against four); FP64 keeps four (bounded to five it spills and took
// 37.1 against 32.1 ms)
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 6 : 4) k_jastrow_full(const __grid_constant__ CSys cs, WState st, HBuf hb) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  const int N = cs.N, M = cs.M, MN = M * N;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  constexpr int NB = een_nb(NORD);
  extern __shared__ __align__(16) double smem[];
  double *sx = smem;                      // [3][N]
  double *sI = sx + 3 * N + (3 * N & 1);  // [2][M][8] table entries and e-n vectors of the batch's rows
  T *sB = reinterpret_cast<T *>(sI + 2 * M * 8);  // [2][M][4*NB] folded rows (16-byte aligned)
  // FP32 path: the rows' fields in FP32 [2][M][8] after the folded rows
  // (used only for NORD > 1)
  float *sIf = reinterpret_cast<float *>(sB + 2 * M * 4 * NB);
  __shared__ double red[4];
  for (int t = threadIdx.x; t < 3 * N; t += blockDim.x) sx[t] = st.x[(size_t)w * 3 * N + t];
  __syncthreads();
  const double kap = cs.scalek, asym = cs.asymp_r;
  double *tab = hb.entab + (size_t)w * kEnFields * MN;
  float *tabf = hb.entabf ? hb.entabf + (size_t)w * kEnFields * MN : nullptr;
  double *fso = st.fso + (size_t)w * N * N;
  double *fij0 = st.fijo + ((size_t)w * 3 + 0) * N * N;
  double *fij1 = st.fijo + ((size_t)w * 3 + 1) * N * N;
  double *fij2 = st.fijo + ((size_t)w * 3 + 2) * N * N;
  double fsum = 0, d2sum = 0, pee = 0;
  // 1. e-n table and e-n terms
  for (int e = threadIdx.x; e < N; e += blockDim.x) {
    double fs = 0, d2 = 0, g[3] = {0, 0, 0};
    for (int ic = 0; ic < M; ic++) {
      const double v0 = sx[e] - cs.cent[3 * ic], v1 = sx[N + e] - cs.cent[3 * ic + 1], v2 = sx[2 * N + e] - cs.cent[3 * ic + 2];
      const double r2 = v0 * v0 + v1 * v1 + v2 * v2, r = sqrt(r2);
      double rr, dd1, dd2;
      scale2<double>(cs, r, rr, dd1, dd2);
      const int t = ic * N + e;
      tab[t] = rr;
      tab[MN + t] = -kap * dd1;
      tab[2 * MN + t] = -kap * dd2;
      tab[3 * MN + t] = -kap * dd1 / r;
      tab[4 * MN + t] = r2;
      if (sizeof(T) == 4 && tabf) {
        tabf[t] = (float)rr;
        tabf[MN + t] = (float)(-kap * dd1);
        tabf[2 * MN + t] = (float)(-kap * dd2);
        tabf[3 * MN + t] = (float)(-kap * dd1 / r);
        tabf[4 * MN + t] = (float)r2;
      }
      st.enm[(size_t)w * 2 * MN + t] = rr;
      st.enm[((size_t)w * 2 + 1) * MN + t] = dd1 / r;
      if (st.enmf) {
        st.enmf[(size_t)w * 2 * MN + t] = (float)rr;
        st.enmf[((size_t)w * 2 + 1) * MN + t] = (float)(dd1 / r);
      }
      if (rr == asym) continue;
      double fen, feni, fenii;
      en_term<2, double>(cs, cs.iwctype[ic], rr, fen, feni, fenii);
      fenii = fenii * dd1 * dd1 + feni * dd2;
      feni = feni * dd1 / r;
      fs += fen;
      g[0] += feni * v0;
      g[1] += feni * v1;
      g[2] += feni * v2;
      d2 += fenii + 2 * feni;
    }
    fso[(size_t)e * N + e] = fs;
    fij0[(size_t)e * N + e] = g[0];
    fij1[(size_t)e * N + e] = g[1];
    fij2[(size_t)e * N + e] = g[2];
    fsum += fs;
    d2sum += d2;
  }
  // 2. pairs
  const T kT = (T)kap, asymT = (T)asym;
  for (int bt = 0; bt < (N + 1) / 2; bt++) {
    const int ia = bt, ib = N - 1 - bt;  // ia == ib only for the middle row of odd N
    const int npa = ia, npb = (ib != ia) ? ib : 0;
    __syncthreads();  // previous batch done with sB / sI; table written
    for (int t = threadIdx.x; t < 2 * M; t += blockDim.x) {
      const int row = t / M, ic = t % M;
      const int i = row == 0 ? ia : ib;
      double *q = sI + (size_t)t * 8;
#pragma unroll
      for (int f = 0; f < kEnFields; f++) q[f] = tab[f * MN + ic * N + i];
      for (int k = 0; k < 3; k++) q[kEnFields + k] = sx[k * N + i] - cs.cent[3 * ic + k];
      if (sizeof(T) == 4 && NORD > 1)
        for (int f = 0; f < 8; f++) sIf[(size_t)t * 8 + f] = (float)q[f];
      if (NORD > 1) een_fold2<NORD, T>(een_coef<T>(cs, cs.iwctype[ic]), T(1 - kap * q[0]), sB + (size_t)t * 4 * NB);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < npa + npb; t += blockDim.x) {
      const int row = t < npa ? 0 : 1;
      const int i = row == 0 ? ia : ib, j = row == 0 ? t : t - npa;
      int isb, ipar;
      double sspinn;
      pair_spin(cs, i, j, isb, ipar, sspinn);
      const double xj[3] = {sx[j], sx[N + j], sx[2 * N + j]};
      const double rv[3] = {sx[i] - xj[0], sx[N + i] - xj[1], sx[2 * N + i] - xj[2]};
      const double rij2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2], rij = sqrt(rij2);
      const double irij = 1 / rij;
      pee += irij;
      const T rijT = (T)rij, irijT = (T)irij, rij2T = (T)rij2;
      const T rvT[3] = {(T)rv[0], (T)rv[1], (T)rv[2]};
      T u, dd1, dd2;
      scale2<T>(cs, rijT, u, dd1, dd2);
      T fs = 0, d2 = 0, gi[3] = {0, 0, 0}, gj[3] = {0, 0, 0};
      if (u != (T)cs.asymp_r) {
        T fee, feeu, feeuu;
        ee_term<2, T>(cs, isb, ipar, (T)sspinn, u, fee, feeu, feeuu);
        feeuu = feeuu * dd1 * dd1 + feeu * dd2;
        feeu = feeu * dd1 * irijT;
        fs += fee;
        for (int k = 0; k < 3; k++) {
          gi[k] += feeu * rvT[k];
          gj[k] -= feeu * rvT[k];
        }
        d2 += 2 * (feeuu + 2 * feeu);
      }
      if (NORD > 1) {
        const T z = 1 - kT * u, du1 = -kT * dd1, du2 = -kT * dd2, du1r = du1 * irijT;
        const T *Brow = sB + (size_t)row * M * 4 * NB;
        const double *Irow = sI + (size_t)row * M * 8;
        const float *IrowF = sIf + (size_t)row * M * 8;
        // the partner's table entries of the next centre are loaded one iteration
        // ahead; the mixed path reads them from the FP32 copy
        using TT = typename std::conditional<sizeof(T) == 4, float, double>::type;
        const TT *tj = (sizeof(T) == 4 ? (const TT *)(const void *)tabf : (const TT *)(const void *)tab) + j;
        TT nr = tj[0], nA = tj[MN], nB = tj[2 * MN], nG = tj[3 * MN], nS = tj[4 * MN];
        for (int ic = 0; ic < M; ic++) {
          const TT rrj = nr;
          const T Aj = (T)nA, Bj = (T)nB, Gj = (T)nG, Sj = (T)nS;
          if (ic + 1 < M) {
            const int o = (ic + 1) * N;
            nr = tj[o]; nA = tj[MN + o]; nB = tj[2 * MN + o]; nG = tj[3 * MN + o]; nS = tj[4 * MN + o];
          }
          const double *qi = Irow + ic * 8;
          const double rri = qi[0];
          if (rri == asym && rrj == (TT)asym) continue;
          // the row's fields in T (the mixed path reads the FP32 copy made at
          // the batch's start instead of converting each one here)
          T Ai, Bi, Gi, Si, vi0, vi1, vi2;
          if constexpr (sizeof(T) == 4) {
            const float4 f0 = *reinterpret_cast<const float4 *>(IrowF + ic * 8);
            const float4 f1 = *reinterpret_cast<const float4 *>(IrowF + ic * 8 + 4);
            Ai = f0.y; Bi = f0.z; Gi = f0.w; Si = f1.x; vi0 = f1.y; vi1 = f1.z; vi2 = f1.w;
          } else {
            Ai = (T)qi[1]; Bi = (T)qi[2]; Gi = (T)qi[3]; Si = (T)qi[4];
            vi0 = (T)qi[5]; vi1 = (T)qi[6]; vi2 = (T)qi[7];
          }
          const EenOut<T> e = een_apply2<NORD, T>(Brow + (size_t)ic * 4 * NB, T(1 - (TT)kap * rrj), z);
          const T dS = Si - Sj;
          const T fuu = e.fuu * du1 * du1 + e.fu * du2;
          const T fu = e.fu * du1r;
          const T fii = e.fii * Ai * Ai + e.fi * Bi, fjj = e.fjj * Aj * Aj + e.fj * Bj;
          const T fi = e.fi * Gi, fj = e.fj * Gj;
          fs += e.fc;
          const T vj0 = (T)(xj[0] - cs.cent[3 * ic]), vj1 = (T)(xj[1] - cs.cent[3 * ic + 1]),
                  vj2 = (T)(xj[2] - cs.cent[3 * ic + 2]);
          gi[0] += fi * vi0 + fu * rvT[0];
          gi[1] += fi * vi1 + fu * rvT[1];
          gi[2] += fi * vi2 + fu * rvT[2];
          gj[0] += fj * vj0 - fu * rvT[0];
          gj[1] += fj * vj1 - fu * rvT[1];
          gj[2] += fj * vj2 - fu * rvT[2];
          d2 += 2 * (fuu + 2 * fu) + du1r * (e.fui * Gi * (rij2T + dS) + e.fuj * Gj * (rij2T - dS)) + fii + 2 * fi +
                fjj + 2 * fj;
        }
      }
      fso[(size_t)i * N + j] = fs;
      fso[(size_t)j * N + i] = fs;
      fij0[(size_t)i * N + j] = gi[0]; fij0[(size_t)j * N + i] = gj[0];
      fij1[(size_t)i * N + j] = gi[1]; fij1[(size_t)j * N + i] = gj[1];
      fij2[(size_t)i * N + j] = gi[2]; fij2[(size_t)j * N + i] = gj[2];
      fsum += fs;
      d2sum += d2;
    }
  }
  (void)asymT;
  __syncthreads();
  // 3. per-electron gradient sums: warp per row, lanes over the partners
  for (int i = wid; i < N; i += blockDim.x >> 5) {
    double a0 = 0, a1 = 0, a2 = 0;
    for (int j = lane; j < N; j += 32) {
      a0 += fij0[(size_t)i * N + j];
      a1 += fij1[(size_t)i * N + j];
      a2 += fij2[(size_t)i * N + j];
    }
    a0 = warp_sum(a0);
    a1 = warp_sum(a1);
    a2 = warp_sum(a2);
    if (lane == 0) {
      st.fjo[((size_t)w * 3 + 0) * N + i] = a0;
      st.fjo[((size_t)w * 3 + 1) * N + i] = a1;
      st.fjo[((size_t)w * 3 + 2) * N + i] = a2;
    }
  }
  const double tf = block_sum<128>(fsum, red);
  const double td = block_sum<128>(d2sum, red);
  const double tp = block_sum<128>(pee, red);
  if (threadIdx.x == 0) {
    st.fsumo[w] = tf;
    hb.d2o[w] = td;
    hb.pe_ee[w] = tp;
  }
}

// ---------------------------------------------------------------------------
// basis functions with Laplacian for electrons [e0, e0+ne): warp per
// (walker, electron); rows ((w*ne + e)*5 + d).
// ---------------------------------------------------------------------------
__global__ void k_basis_all(const __grid_constant__ CSys cs, WState st, HBuf hb, GSys g, int e0, int ne) {
  extern __shared__ __align__(16) double smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const long gw = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int K = cs.K, N = cs.N;
  if (gw >= (long)st.W * ne) return;
  const int el = (int)(gw % ne), w = (int)(gw / ne), e = e0 + el;
  const double x[3] = {st.x[((size_t)w * 3 + 0) * N + e], st.x[((size_t)w * 3 + 1) * N + e],
                       st.x[((size_t)w * 3 + 2) * N + e]};
  double *rec = smem + (size_t)wib * cs.M * kCenRec;
  warp_basis_prepass<2>(cs, g, x, rec, lane);
  __syncwarp();
  if (hb.phi_hi) {
    const int kp = hb.kp;
    float *hi = hb.phi_hi + ((size_t)gw * 5) * kp, *lo = hb.phi_lo + ((size_t)gw * 5) * kp;
    for (int m = lane; m < K; m += 32)
      warp_basis_ao<2>(cs, g, rec, m, [&](int a, int d, double v) {
        float h, l;
        split_tf32(v, h, l);
        hi[(size_t)d * kp + a] = h;
        lo[(size_t)d * kp + a] = l;
      });
    return;
  }
  double *phi = hb.phi + ((size_t)gw * 5) * K;
  for (int m = lane; m < K; m += 32)
    warp_basis_ao<2>(cs, g, rec, m, [&](int a, int d, double v) { phi[(size_t)d * K + a] = v; });
}

__global__ void k_scatter_orbs(const __grid_constant__ CSys cs, WState st, HBuf hb, GSys g, int e0, int ne) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int N = cs.N, nmax = cs.nmax, Oa = cs.Oa;
  if (t >= (long)st.W * ne * nmax) return;
  const int j = (int)(t % nmax);
  const long we = t / nmax;
  const int el = (int)(we % ne), w = (int)(we / ne), e = e0 + el;
  const int iab = e < cs.nup ? 0 : 1;
  const int nel = iab == 0 ? cs.nup : cs.ndn;
  if (j >= nel) return;
  const int o = g.slot_orb[iab * nmax + j];
  const double *ob = hb.orball + (size_t)we * 5 * Oa;
  st.orbs[((size_t)w * N + e) * nmax + j] = ob[o];
  for (int k = 0; k < 3; k++) st.dorbs[(((size_t)w * 3 + k) * N + e) * nmax + j] = ob[(1 + k) * Oa + o];
  hb.ddorbs[((size_t)w * N + e) * nmax + j] = ob[4 * Oa + o];
}

// ---------------------------------------------------------------------------
// matinv + ddx/d2dx2: CTA per (walker, spin); matrix in shared memory.
// ---------------------------------------------------------------------------
// in_place: the factorisation runs in the walker's slmi block in global
// memory (L2-resident) instead of shared memory, for spins too large for
// shared memory (same arithmetic; shared memory then holds col only).
__global__ void k_slater_inv(const __grid_constant__ CSys cs, WState st, HBuf hb, int in_place) {
  const int w = blockIdx.x >> 1, iab = blockIdx.x & 1;
  if (w >= st.W) return;
  const int N = cs.N, nmax = cs.nmax;
  const int nel = iab == 0 ? cs.nup : cs.ndn, ish = iab == 0 ? 0 : cs.nup;
  const int n = nel;
  extern __shared__ __align__(16) double smem[];
  __shared__ int ipvt[256];
  __shared__ int s_p, s_sing;
  double *slmi = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax;
  double *A = in_place ? slmi : smem;            // n*n column-major: A(e,j) = orb of slot j at electron e
  double *col = in_place ? smem : smem + n * n;  // n
  if (n == 0) {
    if (threadIdx.x == 0) st.detiab[2 * w + iab] = 1.0;
    return;
  }
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
    const int e = t % n, j = t / n;
    A[t] = st.orbs[((size_t)w * N + ish + e) * nmax + j];
  }
  if (threadIdx.x == 0) s_sing = 0;
  __syncthreads();
  double det = 0;
  if (n == 1) {
    if (threadIdx.x == 0) {
      det = A[0];
      A[0] = 1.0 / A[0];
      if (det == 0.0) s_sing = 1;
    }
  } else if (n == 2) {
    if (threadIdx.x == 0) {
      det = A[0] * A[3] - A[2] * A[1];
      const double deti = 1.0 / det, aux = A[0];
      A[0] = A[3] * deti;
      A[3] = aux * deti;
      A[1] = -A[1] * deti;
      A[2] = -A[2] * deti;
      if (det == 0.0) s_sing = 1;
    }
  } else {
    // LU with partial pivoting (first entry of maximal |a|, as idamax)
    for (int k = 0; k < n; k++) {
      if (threadIdx.x < 32) {
        double best = -1.0;
        int bi = k;
        for (int i = k + threadIdx.x; i < n; i += 32) {
          const double v = fabs(A[i + n * k]);
          if (v > best) { best = v; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
          const double ob = __shfl_xor_sync(0xffffffffu, best, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if (threadIdx.x == 0) {
          s_p = bi;
          ipvt[k] = bi;
          if (A[bi + n * k] == 0.0) s_sing = 1;
        }
      }
      __syncthreads();
      if (s_sing) break;
      const int p = s_p;
      if (p != k)
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
          const double tmp = A[k + n * j];
          A[k + n * j] = A[p + n * j];
          A[p + n * j] = tmp;
        }
      __syncthreads();
      const double piv = 1.0 / A[k + n * k];
      for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) A[i + n * k] *= piv;
      __syncthreads();
      const int m = n - k - 1;
      for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
        const int i = k + 1 + t % m, j = k + 1 + t / m;
        A[i + n * j] -= A[i + n * k] * A[k + n * j];
      }
      __syncthreads();
    }
    if (!s_sing) {
      if (threadIdx.x == 0) {
        double det1 = 1.0, det2 = 0.0;
        for (int i = 0; i < n; i++) {
          if (ipvt[i] != i) det1 = -det1;
          det1 = A[i + n * i] * det1;
          if (det1 == 0.0) break;
          while (fabs(det1) < 1.0) { det1 = 10.0 * det1; det2 = det2 - 1.0; }
          while (fabs(det1) >= 10.0) { det1 = det1 / 10.0; det2 = det2 + 1.0; }
        }
        det = det1 * pow(10.0, det2);
      }
      // inv(U) in place, column by column
      for (int j = 0; j < n; j++) {
        if (threadIdx.x == 0) A[j + n * j] = 1.0 / A[j + n * j];
        __syncthreads();
        const double ajj = -A[j + n * j];
        for (int i = threadIdx.x; i < j; i += blockDim.x) {
          double s = 0;
          for (int kk = i; kk < j; kk++) s += A[i + n * kk] * A[kk + n * j];
          col[i] = s;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < j; i += blockDim.x) A[i + n * j] = col[i] * ajj;
        __syncthreads();
      }
      // solve inv(A) * L = inv(U)
      for (int j = n - 2; j >= 0; j--) {
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
          col[i] = A[i + n * j];
          A[i + n * j] = 0.0;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
          double s = 0;
          for (int kk = j + 1; kk < n; kk++) s += A[i + n * kk] * col[kk];
          A[i + n * j] -= s;
        }
        __syncthreads();
      }
      for (int j = n - 2; j >= 0; j--) {
        const int jp = ipvt[j];
        if (jp != j)
          for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const double tmp = A[i + n * j];
            A[i + n * j] = A[i + n * jp];
            A[i + n * jp] = tmp;
          }
        __syncthreads();
      }
    }
  }
  __syncthreads();
  if (s_sing) {
    if (threadIdx.x == 0) st.status[w] = 1;
    return;
  }
  if (threadIdx.x == 0) st.detiab[2 * w + iab] = det;
  if (!in_place)
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) slmi[t] = A[t];
  else
    __syncthreads();  // every thread's last writes to the block before the reads below
  // ddx, d2dx2 (determinant.f90 ddot loops)
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    const int eg = ish + e;
    for (int j = 0; j < n; j++) {
      const double s = A[j + n * e];
      a0 += s * st.dorbs[(((size_t)w * 3 + 0) * N + eg) * nmax + j];
      a1 += s * st.dorbs[(((size_t)w * 3 + 1) * N + eg) * nmax + j];
      a2 += s * st.dorbs[(((size_t)w * 3 + 2) * N + eg) * nmax + j];
      a3 += s * hb.ddorbs[((size_t)w * N + eg) * nmax + j];
    }
    double *d = hb.ddx + ((size_t)w * N + eg) * 4;
    d[0] = a0; d[1] = a1; d[2] = a2; d[3] = a3;
  }
}

// ---------------------------------------------------------------------------
// c~ vectors: CTA per (walker, spin, 64-AO chunk).
// ---------------------------------------------------------------------------
// s_global: the inverse is read from global memory (L2) rather than staged
// in shared memory, for spins too large for shared memory
__global__ void k_ctilde(const __grid_constant__ CSys cs, WState st, HBuf hb, GSys g, int s_global) {
  const int nchunk = (cs.K + 63) / 64;
  const int b = blockIdx.x;
  const int chunk = b % nchunk, iab = (b / nchunk) & 1, w = b / (2 * nchunk);
  if (w >= st.W) return;
  const int nmax = cs.nmax, K = cs.K, Oa = cs.Oa, N = cs.N;
  const int nel = iab == 0 ? cs.nup : cs.ndn, ish = iab == 0 ? 0 : cs.nup;
  if (nel == 0) return;
  extern __shared__ __align__(16) double smem[];
  const double *slmi = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax;
  double *Ss = smem;                                // nel*nel (shared-memory staging)
  double *Co = s_global ? smem : smem + nel * nel;  // [nel][64]
  const double *S = s_global ? slmi : Ss;
  if (!s_global)
    for (int t = threadIdx.x; t < nel * nel; t += blockDim.x) Ss[t] = slmi[t];
  const int m0 = chunk * 64;
  for (int t = threadIdx.x; t < nel * 64; t += blockDim.x) {
    const int j = t / 64, mm = t % 64;
    Co[t] = (m0 + mm < K) ? g.coefT[(size_t)(m0 + mm) * Oa + g.slot_orb[iab * nmax + j]] : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nel * 64; t += blockDim.x) {
    const int i = t / 64, mm = t % 64;
    if (m0 + mm >= K) continue;
    double s = 0;
    for (int j = 0; j < nel; j++) s += S[j + nel * i] * Co[j * 64 + mm];
    hb.ctilde[((size_t)w * N + ish + i) * K + m0 + mm] = s;
  }
}

// ---------------------------------------------------------------------------
// Pseudopotential: CTA per walker, warps over (pair, quadrature point).
// ---------------------------------------------------------------------------
template <int NORD>
__device__ __forceinline__ double psinl_d(const CSys &cs, double u, double rri, double rrj, int it) {
  if (rri == cs.asymp_r && rrj == cs.asymp_r) return 0.0;
  const double k = cs.scalek;
  return een_poly<NORD, 0, double>(&cs.c[it * CW_MAX_TERMS], 1 - k * u, 1 - k * rri, 1 - k * rrj).fc;
}
__device__ __forceinline__ double psianl_d(const CSys &cs, double rri, int it) {
  if (rri == cs.asymp_r) return 0.0;
  const int na = cs.norda + 1;
  double v = cs.a4[it * na] * rri / (1.0 + cs.a4[it * na + 1] * rri) - cs.asymp_jasa[it];
  double rrip = rri;
  for (int i = 2; i <= cs.norda; i++) {
    rrip *= rri;
    v += cs.a4[it * na + i] * rrip;
  }
  return v;
}
template <typename T>
__device__ __forceinline__ T psibnl_t(const CSys &cs, T u, int isb, int ipar, T sspinn) {
  if (u == (T)cs.asymp_r) return 0;
  const int nb = cs.nordb + 1;
  T fee = (T)cs.b[isb * nb] * u / (1 + (T)cs.b[isb * nb + 1] * u);
  T v = sspinn * fee - (T)cs.asymp_jasb[ipar];
  T uu = u;
  for (int i = 2; i <= cs.nordb; i++) {
    uu *= u;
    v += (T)cs.b[isb * nb + i] * uu;
  }
  return v;
}
__device__ __forceinline__ double psibnl_d(const CSys &cs, double u, int isb, int ipar, double sspinn) {
  return psibnl_t<double>(cs, u, isb, ipar, sspinn);
}

// Shared-memory plan of k_ecp (in doubles, every region 16-byte aligned):
//   rr_en [N][M|1] scaled e-n distances (odd row stride: lanes over the
//   electrons read them without bank conflicts), sx [3][N], the pair list (channel
//   potentials [cap][3], packed i*M+ic [cap] ints), then per warp: the
//   point's scaled e-n distances [M], its folded e-e-n coefficients [M][NB],
//   its basis prepass [M][kCenRec] and, for multideterminant wave functions,
//   its basis values [K] (reused by the pseudopotential B matrix).
constexpr int kEcpMaxWarps = 16;
__host__ __device__ inline size_t ecp_base_doubles(int N, int M, int cap, int rr_global) {
  const size_t b = (rr_global ? 0 : (size_t)N * (M | 1)) + 3 * (size_t)N + 3 * (size_t)cap + (size_t)(cap + 1) / 2;
  return b + (b & 1);
}
__host__ __device__ inline size_t ecp_warp_doubles(int M, int nb, int tbytes, int naov) {
  size_t bq = ((size_t)M * nb * tbytes + 7) / 8;
  bq += bq & 1;
  return (size_t)(M + (M & 1)) + bq + (size_t)M * kCenRec + (size_t)(naov + (naov & 1));
}

// T: arithmetic of the quadrature points' Jastrow ratio terms (double:
// parity path, float: mixed path); the ratio sums, potentials, basis values
// and the determinant ratio stay FP64.
//
// CTA per walker.  getvps_gauss (vmc/nonloc_pot.f90:3) runs for every
// (electron, centre) pair in parallel; the pairs whose non-local channels
// pass the reference's 1e-4 test are listed in (electron, centre) order, and
// each warp then evaluates (pair, quadrature point) units round-robin: the
// point's determinant ratio (nonlocd_quad through c~), its Jastrow ratio
// (nonlocj_quad4) and the weighted Legendre sum (vmc/nonloc.f90:5).  The list
// holds at most blockDim entries; a walker with more active pairs is
// processed in several passes, in the same order.
template <int NORD, typename T, int MINB>  // MINB: blocks per SM the register budget is set for
__global__ void __launch_bounds__(32 * kEcpMaxWarps, MINB) k_ecp(const __grid_constant__ CSys cs, WState st, HBuf hb, GSys g) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  const int N = cs.N, M = cs.M, K = cs.K, NQ = cs.nquad, NM = N * M;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5, cap = blockDim.x;
  constexpr int NB = 2 * ((een_nb(NORD) + 1) / 2);
  extern __shared__ __align__(16) double smem[];
  const int MS = M | 1;                         // row stride of rr_en
  const int rrg = hb.ecp_rr != nullptr;         // rr_en in global memory (large molecules)
  double *rr_en = rrg ? hb.ecp_rr + (size_t)w * N * MS : smem;  // [N][MS]
  double *sx = smem + (rrg ? 0 : (size_t)N * MS);              // [3][N]
  double *lst_v = sx + 3 * N;                   // [cap][3] non-local channel potentials
  int *lst_ie = reinterpret_cast<int *>(lst_v + 3 * cap);  // [cap] i*M + ic
  const int naov = hb.md_P ? K : 0;
  const size_t wsd = ecp_warp_doubles(M, NB, (int)sizeof(T), naov);
  double *wsp = smem + ecp_base_doubles(N, M, cap, rrg) + (size_t)wid * wsd;
  double *rq = wsp;                             // [M]
  T *bq = reinterpret_cast<T *>(wsp + M + (M & 1));  // [M][NB]
  double *aov = wsp + wsd - (naov + (naov & 1));      // [K] basis values (multideterminant)
  double *rec = aov - (size_t)M * kCenRec;            // [M][kCenRec]
  __shared__ int s_wcnt[kEcpMaxWarps];
  __shared__ int s_total;
  __shared__ double s_red[kEcpMaxWarps][3];
  for (int t = threadIdx.x; t < 3 * N; t += blockDim.x) sx[t] = st.x[(size_t)w * 3 * N + t];
  if (threadIdx.x == 0) s_total = 0;
  __syncthreads();
  for (int t = threadIdx.x; t < NM; t += blockDim.x) {
    const int jj = t / M, jc = t % M;
    const Cen cc = cen_of(g, jc);
    const double d0 = sx[jj] - cc.x, d1 = sx[N + jj] - cc.y, d2 = sx[2 * N + jj] - cc.z;
    rr_en[jj * MS + jc] = scale0<double>(cs, sqrt(d0 * d0 + d1 * d1 + d2 * d2));
  }
  const double *xqw = st.xq + (size_t)w * 3 * NQ;
  const double *fso = st.fso + (size_t)w * N * N;
  double vp0 = 0, vp1 = 0, vloc = 0;
  int cursor = 0;
  for (;;) {
    // ---- list the active (electron, centre) pairs from `cursor` on
    while (cursor < NM) {
      const int t = cursor + threadIdx.x;
      int flag = 0;
      double v[3] = {0, 0, 0}, vl = 0;
      if (t < NM) {
        const int i = t / M, ic = t % M;
        const Cen cc = cen_of(g, ic);
        const int ict = cc.it;
        const double d0 = sx[i] - cc.x, d1 = sx[N + i] - cc.y, d2 = sx[2 * N + i] - cc.z;
        const double r = fmax(1.0e-10, sqrt(d0 * d0 + d1 * d1 + d2 * d2));
        const int lp = cs.lpot[ict];
        vl = gauss_pot_d(cs, r, lp, ict) - cs.znuc[ict] * (1.0 / r);
#pragma unroll
        for (int l = 1; l <= 3; l++) {
          if (l <= lp - 1) {
            v[l - 1] = gauss_pot_d(cs, r, l, ict);
            if (fabs(v[l - 1]) > 1.0e-4) flag = 1;
          }
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, flag);
      if (lane == 0) s_wcnt[wid] = __popc(bal);
      __syncthreads();
      int off = 0, tot = 0;
      for (int k = 0; k < nw; k++) {
        const int c = s_wcnt[k];
        off += k < wid ? c : 0;
        tot += c;
      }
      const int base = s_total;
      __syncthreads();  // s_wcnt and s_total read by every thread
      if (base + tot > cap) break;  // uniform: this chunk opens the next pass
      if (flag) {
        const int pos = base + off + __popc(bal & ((1u << lane) - 1u));
        lst_ie[pos] = t;
        lst_v[3 * pos] = v[0]; lst_v[3 * pos + 1] = v[1]; lst_v[3 * pos + 2] = v[2];
      }
      vloc += vl;
      if (threadIdx.x == 0) s_total = base + tot;
      cursor += blockDim.x;
      __syncthreads();
    }
    const int nlist = s_total;
    // ---- (pair, quadrature point) units, round-robin over warps
    for (int u = wid; u < nlist * NQ; u += nw) {
      const int a = u / NQ, q = u - a * NQ;
      const int pt = lst_ie[a], i = pt / M, ic = pt - (pt / M) * M;
      const int ict = cs.iwctype[ic];
      const double ri_v[3] = {sx[i] - cs.cent[3 * ic], sx[N + i] - cs.cent[3 * ic + 1], sx[2 * N + i] - cs.cent[3 * ic + 2]};
      const double rin = sqrt(ri_v[0] * ri_v[0] + ri_v[1] * ri_v[1] + ri_v[2] * ri_v[2]);
      const double xqq = xqw[q], yqq = xqw[NQ + q], zqq = xqw[2 * NQ + q];
      const double costh = (ri_v[0] * xqq + ri_v[1] * yqq + ri_v[2] * zqq) * (1.0 / rin);
      const double xp[3] = {rin * xqq + cs.cent[3 * ic], rin * yqq + cs.cent[3 * ic + 1], rin * zqq + cs.cent[3 * ic + 2]};
      // distance_quad (r_en_quad(iq,ic) = r_en(i,ic)) and the folded e-e-n
      // coefficients of the point
      for (int jc = lane; jc < M; jc += 32) {
        const Cen cc = cen_of(g, jc);
        double xc[3] = {xp[0] - cc.x, xp[1] - cc.y, xp[2] - cc.z};
        double r = sqrt(xc[0] * xc[0] + xc[1] * xc[1] + xc[2] * xc[2]);
        if (jc == ic) r = rin;
        rq[jc] = scale0<double>(cs, r);
        if (NORD > 1)
          een_fold0<NORD, T>(een_coef<T>(cs, cc.it), T(1 - cs.scalek * rq[jc]), bq + (size_t)jc * NB);
      }
      warp_basis_prepass<0>(cs, g, xp, rec, lane);
      __syncwarp();
      // determinant ratio (nonlocd_quad) via c~: basis values (ider=0) of the
      // point contracted on the fly
      const double *ct = hb.ctilde + ((size_t)w * N + i) * K;
      double dr = 0;
      for (int m = lane; m < K; m += 32)
        warp_basis_ao<0>(cs, g, rec, m, [&](int, int, double v) {
          dr += v * ct[m];
          if (naov) aov[m] = v;
        });
      dr = warp_sum(dr);
      // Jastrow ratio (nonlocj_quad4)
      double fsum = 0;
      for (int jj = lane; jj < N; jj += 32) {
        if (jj == i) continue;
        const int pi = jj < i ? i : jj, pj = jj < i ? jj : i;
        int isb, ipar;
        double sspinn;
        pair_spin(cs, pi, pj, isb, ipar, sspinn);
        const double dx0 = sx[jj] - xp[0], dx1 = sx[N + jj] - xp[1], dx2 = sx[2 * N + jj] - xp[2];
        const double rij = sqrt(dx0 * dx0 + dx1 * dx1 + dx2 * dx2);
        const T u = scale0<T>(cs, (T)rij);
        T f = psibnl_t<T>(cs, u, isb, ipar, (T)sspinn);
        if (NORD > 1) {
          // psinl (vmc/nonlpsi.f90:4) through the folded coefficients of the point
          const T kT = (T)cs.scalek, z = 1 - kT * u;
          for (int jc = 0; jc < M; jc++) {
            const double rrj = rr_en[jj * MS + jc];
            if (rq[jc] == cs.asymp_r && rrj == cs.asymp_r) continue;
            if constexpr (sizeof(T) == 8)
              f += een_apply0<NORD>((const double *)(bq + (size_t)jc * NB), 1 - cs.scalek * rrj, (double)z);
            else
              f += een_apply0f<NORD>((const float *)(bq + (size_t)jc * NB), 1 - kT * (T)rrj, (float)z);
          }
        }
        fsum += (double)f - fso[(size_t)i * N + jj];
      }
      double fen = 0;
      for (int jc = lane; jc < M; jc += 32) fen += psianl_d(cs, rq[jc], cs.iwctype[jc]);
      fsum = warp_sum(fsum) + (warp_sum(fen) - fso[(size_t)i * N + i]);
      double term = 0;
      for (int l = 1; l <= cs.lpot[ict] - 1; l++) term += yl0_d(l, costh) * lst_v[3 * a + (l - 1)];
      const double trj = term * cs.wq[q] * exp(fsum);
      if (i < cs.nup) vp0 += trj * dr;
      else vp1 += trj * dr;
      if (hb.tvpsp && lane == 0) {  // transition matrix element of a T-move (nonloc.f90:296)
        hb.tvpsp[(((size_t)w * N + i) * NQ + q) * M + ic] = dr * trj;
        if (hb.tvtrj) hb.tvtrj[(((size_t)w * N + i) * NQ + q) * M + ic] = trj;
      }
      if (hb.md_P) {
        // pseudopotential B matrix of every orbital (nonloc.f90:271): the
        // basis values of the point weighted by trj, contracted with coef later
        double *P = hb.md_P + ((size_t)w * N + i) * K;
        for (int m = lane; m < K; m += 32) atomicAdd(&P[m], trj * aov[m]);
      }
      __syncwarp();
    }
    __syncthreads();  // list consumed
    if (cursor >= NM) break;
    if (threadIdx.x == 0) s_total = 0;
  }
  vloc = warp_sum(vloc);
  if (lane == 0) {
    s_red[wid][0] = vp0;
    s_red[wid][1] = vp1;
    s_red[wid][2] = vloc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0, c = 0;
    for (int k = 0; k < nw; k++) { a += s_red[k][0]; b += s_red[k][1]; c += s_red[k][2]; }
    hb.vpsp[2 * w] = a;
    hb.vpsp[2 * w + 1] = b;
    hb.pe_ecp[w] = c;
  }
}

// ---------------------------------------------------------------------------
// E_L assembly + metrop6's per-step sums (warp per walker).
// mode: 0 = hpsi only (zerest, parity hook), 1 = end of a metrop6 sweep
// ---------------------------------------------------------------------------
__global__ void k_energy(const __grid_constant__ CSys cs, WState st, HBuf hb, int mode, double *out_e, double *out_ekin) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= st.W) return;
  const int N = cs.N;
  const double hb_ = 0.5;
  double ek[2] = {0, 0}, v2 = 0, pen = 0;
  for (int e = lane; e < N; e += 32) {
    const double *d = hb.ddx + ((size_t)w * N + e) * 4;
    const double vx = st.fjo[((size_t)w * 3 + 0) * N + e], vy = st.fjo[((size_t)w * 3 + 1) * N + e],
                 vz = st.fjo[((size_t)w * 3 + 2) * N + e];
    const double tmp = -hb_ * (d[3] + 2.0 * (vx * d[0] + vy * d[1] + vz * d[2]));
    ek[e < cs.nup ? 0 : 1] += tmp;
    v2 += -hb_ * (vx * vx + vy * vy + vz * vz);
    if (cs.nloc == 0) {
      for (int ic = 0; ic < cs.M; ic++) {
        const double d0 = st.x[((size_t)w * 3 + 0) * N + e] - cs.cent[3 * ic];
        const double d1 = st.x[((size_t)w * 3 + 1) * N + e] - cs.cent[3 * ic + 1];
        const double d2 = st.x[((size_t)w * 3 + 2) * N + e] - cs.cent[3 * ic + 2];
        pen += -cs.znuc[cs.iwctype[ic]] / sqrt(d0 * d0 + d1 * d1 + d2 * d2);
      }
    }
  }
  ek[0] = warp_sum(ek[0]);
  ek[1] = warp_sum(ek[1]);
  v2 = warp_sum(v2);
  pen = warp_sum(pen);
  if (lane != 0) return;
  double pe = cs.pecent + hb.pe_ee[w];
  if (cs.nloc == 0) pe += pen;
  else pe += hb.pe_ecp[w];
  const double vp0 = cs.nloc ? hb.vpsp[2 * w] : 0.0, vp1 = cs.nloc ? hb.vpsp[2 * w + 1] : 0.0;
  const double ekin_other = -hb_ * hb.d2o[w] + v2;
  const double e_other = ekin_other + pe;
  const double dener = hb.md_den ? hb.md_den[2 * w] : 0.0, dekin = hb.md_den ? hb.md_den[2 * w + 1] : 0.0;
  const double energy = dener + (ek[0] + vp0) + (ek[1] + vp1) + e_other;
  const double ekin = dekin + ek[0] + ek[1] + ekin_other;
  const double psid = hb.md_S ? st.detiab[2 * w] * st.detiab[2 * w + 1] * hb.md_S[w]
                             : st.detiab[2 * w] * st.detiab[2 * w + 1] * cs.cdet;
  const double psij = st.fsumo[w];
  st.eold[w] = energy;
  st.ekino[w] = ekin;
  st.psido[w] = psid;
  st.psijo[w] = psij;
  // guiding function (metrop6 :652-657, :732): psi2g from the S of every state
  const double psi2g = (cs.iguiding > 0 && hb.md_S_ms) ? md_psig(cs, hb.md_S_ms + (size_t)w * cs.nstates, cs.nstates) : 1.0;
  st.psi2o[w] = log(fabs(psi2g)) + 2 * (log(fabs(psid)) + psij);
  if (!isfinite(energy)) st.status[w] |= 2;
  if (out_e) out_e[w] = energy;
  if (out_ekin) out_ekin[w] = ekin;
  if (hb.md_S_ms) {
    // every state: its own correction and psi_D, weighted by
    // (psi_s/psi_1)^2 / psi2g for the sampled distribution (metrop6 :678-690)
    const int ns = cs.nstates;
    const double S1 = hb.md_S_ms[(size_t)w * ns];
    for (int s = 0; s < ns; s++) {
      const double *dn = hb.md_den_ms + ((size_t)w * ns + s) * 2;
      const double Ss = hb.md_S_ms[(size_t)w * ns + s];
      const double es = dn[0] + (ek[0] + vp0) + (ek[1] + vp1) + e_other;
      const double ks = dn[1] + ek[0] + ek[1] + ekin_other;
      hb.e_ms[(size_t)w * ns + s] = es;
      hb.psid_ms[(size_t)w * ns + s] = st.detiab[2 * w] * st.detiab[2 * w + 1] * Ss;
      if (mode == 1) {
        const double ws = Ss / S1 * exp(psij - psij) / sqrt(psi2g);
        const double wt = ws * ws;
        double *q = hb.sums_ms + ((size_t)w * ns + s) * 4;
        q[0] += wt;
        q[1] += es * wt;
        q[2] += (es - ks) * wt;
        q[3] += ks * wt;
      }
    }
  }
  if (mode == 1) {
    const double wtg_sqrt = psid / psid * exp(psij - psij) / sqrt(psi2g);
    const double wtg = wtg_sqrt * wtg_sqrt;
    double *s = st.sums + (size_t)w * 8;
    s[0] += wtg;
    s[1] += energy * wtg;
    s[2] += (energy - ekin) * wtg;
    s[3] += ekin * wtg;
    s[5] += energy * wtg;
    s[6] += energy * energy * wtg;
  }
}

// rotqua (vmc/rotqua.f90:357): random rotation frame (x, y, z axes) of the
// quadrature grid drawn from one stream.  Host and device share it: VMC draws
// per walker on the device, DMC draws once per step from the population
// stream on the host.
__host__ __device__ inline void rotqua_frame(DRng &rng, double f[9]) {
  double x1, x2, x3, xsum;
  int guard = 0;
  do {
    x1 = 1.0 - 2.0 * rng.uniform();
    x2 = 1.0 - 2.0 * rng.uniform();
    xsum = x1 * x1 + x2 * x2;
  } while (xsum >= 1.0 && ++guard < 1000000);
  double xsum2 = 2.0 * sqrt(fabs(1.0 - xsum));
  x1 = x1 * xsum2;
  x2 = x2 * xsum2;
  x3 = 1.0 - 2.0 * xsum;
  double theta = acos(x3), sthet = sin(theta), cfi, sfi;
  if (sthet < 1.0e-05) {
    cfi = 1; sfi = 0; x1 = 0; x2 = 0; x3 = 1; sthet = 0;
  } else {
    cfi = x1 / sthet;
    sfi = x2 / sthet;
  }
  const double yy1 = x3 * cfi, yy2 = x3 * sfi, yy3 = -sthet;
  const double zz1 = -sfi, zz2 = cfi, zz3 = 0.0;
  double u1, u2, usum;
  guard = 0;
  do {
    u1 = rng.uniform() * 2.0 - 1.0;
    u2 = rng.uniform() * 2.0 - 1.0;
    usum = u1 * u1 + u2 * u2;
  } while (usum >= 1.0 && ++guard < 1000000);
  const double uu = sqrt(usum);
  u1 = u1 / uu;
  u2 = u2 / uu;
  f[0] = x1; f[1] = x2; f[2] = x3;
  f[3] = yy1 * u1 + zz1 * u2; f[4] = yy2 * u1 + zz2 * u2; f[5] = yy3 * u1 + zz3 * u2;
  f[6] = yy1 * u2 - zz1 * u1; f[7] = yy2 * u2 - zz2 * u1; f[8] = yy3 * u2 - zz3 * u1;
}

__device__ __forceinline__ void rotqua_body(const CSys &cs, const WState &st, const int bid) {
  const int w = bid * blockDim.x + threadIdx.x;
  if (w >= st.W) return;
  DRng rng;
  rng.load(st.rng + 4 * (size_t)w);
  double f[9];
  rotqua_frame(rng, f);
  const int NQ = cs.nquad;
  double *xq = st.xq + (size_t)w * 3 * NQ;
  for (int iq = 0; iq < NQ; iq++) {
    xq[iq] = cs.xq0[iq] * f[0] + cs.yq0[iq] * f[3] + cs.zq0[iq] * f[6];
    xq[NQ + iq] = cs.xq0[iq] * f[1] + cs.yq0[iq] * f[4] + cs.zq0[iq] * f[7];
    xq[2 * NQ + iq] = cs.xq0[iq] * f[2] + cs.yq0[iq] * f[5] + cs.zq0[iq] * f[8];
  }
  rng.store(st.rng + 4 * (size_t)w);
}
__global__ void k_rotqua(const __grid_constant__ CSys cs, WState st) { rotqua_body(cs, st, blockIdx.x); }

// Positions between the caller's layout [W][N][3] (CHAMP's xold(3,nelec)
// per walker) and the engine's [W][3][N]: thread per (walker, electron).
__global__ void k_x_from_host(int W, int N, const double *__restrict__ src, double *__restrict__ dst) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)W * N) return;
  const long w = t / N, e = t % N;
  const double *p = src + 3 * t;
  dst[(w * 3 + 0) * N + e] = p[0];
  dst[(w * 3 + 1) * N + e] = p[1];
  dst[(w * 3 + 2) * N + e] = p[2];
}
__global__ void k_x_to_host(int W, int N, const double *__restrict__ src, double *__restrict__ dst) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)W * N) return;
  const long w = t / N, e = t % N;
  double *p = dst + 3 * t;
  p[0] = src[(w * 3 + 0) * N + e];
  p[1] = src[(w * 3 + 1) * N + e];
  p[2] = src[(w * 3 + 2) * N + e];
}

// zerest's unrotated quadrature points of every walker: thread per walker
__global__ void k_xq_unrotated(const __grid_constant__ CSys cs, WState st) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= st.W) return;
  const int NQ = cs.nquad;
  double *xq = st.xq + (size_t)w * 3 * NQ;
  for (int q = 0; q < NQ; q++) {
    xq[q] = cs.xq0[q];
    xq[NQ + q] = cs.yq0[q];
    xq[2 * NQ + q] = cs.zq0[q];
  }
}

// zerest's nearest-nucleus tables: thread per (walker, electron)
__global__ void k_nearest(const __grid_constant__ CSys cs, WState st) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int N = cs.N;
  if (t >= (long)st.W * N) return;
  const int w = (int)(t / N), i = (int)(t % N);
  double rmin = 99.0e9;
  int near = 0;
  double x[3];
  for (int k = 0; k < 3; k++) x[k] = st.x[((size_t)w * 3 + k) * N + i];
  for (int ic = 0; ic < cs.M; ic++) {
    double r2 = 0;
    for (int k = 0; k < 3; k++) {
      const double d = x[k] - cs.cent[3 * ic + k];
      r2 += d * d;
    }
    const double r = sqrt(r2);
    if (r < rmin) { rmin = r; near = ic; }
  }
  st.rmino[(size_t)w * N + i] = rmin;
  st.nearesto[(size_t)w * N + i] = near;
  for (int k = 0; k < 3; k++) st.rvmino[((size_t)w * 3 + k) * N + i] = x[k] - cs.cent[3 * near + k];
}

}  // namespace cw
