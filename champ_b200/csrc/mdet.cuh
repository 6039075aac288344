// mdet.cuh — multideterminant wave functions, psi_D = sum_k c_k D_k^up D_k^dn
// with determinants given as excitations of a reference (CHAMP's compact
// table method: vmc/multideterminant.f90, vmc/multideterminante.f90,
// vmc/set_input_data.f90:46).
//
// Per spin s, with A the reference Slater matrix and Phi the values of all
// orbitals at the electrons of spin s:
//   aa = A^-1 Phi                        (n x O, only columns >= ivirt used)
//   d_s[kk] = det(aa[irepcol_kk, ireporb_kk])   excitation ratio of unique
//                                        spin-determinant kk
//   S = sum_k c_k d_up(k) d_dn(k)        (d = 1 for a kref-equivalent part)
//   psi_D = D_ref^up D_ref^dn S
// Y matrix of spin s: Y[irep][v] = sum_kk ceq[kk] (M_kk^-1)[jr][ir] at
// (v, irep) = (ireporb[jr], irepcol[ir]), ceq[kk] = d_s[kk] G_s[kk] with
//   G_s[kk] = sum_{k: spin-s part of k is kk} c_k d_other(k),
// which depends only on the other spin.  During the moves of spin s the
// other spin is frozen, so G_s is formed once per spin phase and each move
// costs O(unique spin-determinants), not O(ndet).
//
//   k_md_scatter    orbital values / gradients of every orbital and the
//                   kinetic B matrix (compute_bmatrices_kin) from hpsi's LCAO
//   k_md_ecp_b      pseudopotential B matrix: quadrature basis sums x coef
//   k_md_hpsi       aa, excitation ratios, S, Y of both spins, the energy
//                   corrections (multideterminant_hpsi + hpsi :220-238)
//   k_md_phase      G_s at the start of the moves of spin s (the role of
//                   update_ymat, vmc/multideterminant.f90:562)
//   k_md_drift_old  multideterminante_grad at the old position
//   k_md_move       multideterminante at the proposed position: rank-1
//                   update of aa, ratios, S, psi_D, drift
// The moves never form Y: the drift needs only its contraction with one
// inverse column, sum_{v,irep} Y[irep][v] t[v] c[irep], which regrouped per
// excitation is sum_kk d_kk G_kk t[ro_kk] . M_kk^-1 c[rc_kk]; Y itself is
// built once per sweep for the energy (k_md_hpsi) and the post-hpsi drifts.
#pragma once
#include "common.cuh"

namespace cw {

#define CW_MD_MEX 4   // largest excitation order handled on the GPU

struct MdTab {
  const int *exc;     // [2][nuniq_max][1 + 2*CW_MD_MEX]: numrep, irepcol[], ireporb[]
  const int *kw;      // [ndet][2] unique index of each spin part, -1 = kref-equivalent
  const double *cdet; // [ndet] sign-adjusted coefficients
  int numax;          // nuniq_max
};

struct MdBuf {
  double *aa;     // [W][2][nmax][O]
  double *ymat;   // [W][2][nmax][O]  Y(v, irep) at [irep][v]
  double *dd;     // [W][2][numax]
  double *G;      // [W][numax + 1]  phase weights of the moving spin, [numax] = kref-equivalent part
  double *S;      // [W]
  double *orbA;   // [W][N][O]
  double *dorbA;  // [W][3][N][O]
  double *bkin;   // [W][N][O]
  double *bnl;    // [W][N][O]
  double *P;      // [W][N][K] quadrature basis sums of the pseudopotential
  double *den;    // [W][2]  denergy, dekin
  double *S_ms;   // [W][nstates] S of every state (null for one state)
  double *den_ms; // [W][nstates][2] denergy, dekin of every state
  // guiding function (null without): S of every state at the proposed point,
  // psi2g there
  double *Sn_ms;  // [W][nstates]
  double *psi2gn; // [W]
  // move outputs (spin of the moved electron)
  double *cvec;   // [W][nmax] inverse column of the moved electron (before the move)
  double *wvec;   // [W][O]    rank-1 factor of aa
  double *ddn;    // [W][numax]
  double *Sn;     // [W]
  double *psidn;  // [W]
  double *veln;   // [W][3]
  double *velo;   // [W][3]
};

__device__ __forceinline__ const int *md_exc(const MdTab &t, int s, int kk) {
  return t.exc + ((size_t)s * t.numax + kk) * (1 + 2 * CW_MD_MEX);
}

// One excitation entry and its phase weight G held in registers, so that a
// loop over the unique spin-determinants loads the next entry while it
// solves the current one (the table and G come from L2 / DRAM).
struct MdExcPf {
  int e[1 + 2 * CW_MD_MEX];
  double g;
  __device__ __forceinline__ void load(const MdTab &tab, int s, int kk, const double *G) {
    const int *p = md_exc(tab, s, kk);
#pragma unroll
    for (int i = 0; i < 1 + 2 * CW_MD_MEX; i++) e[i] = __ldg(p + i);
    g = G[kk];
  }
};

// Gauss-Jordan with partial pivoting on the NR x NR excitation matrix
// a[ir][jr] = aa[rc[ir]][ro[jr]] held in registers (row swaps by select, no
// dynamic indexing); with INV the inverse is left in b (b[r][k] =
// (M^-1)(r, k)).  Same operations in the same order as md_small_inv's
// general path, so the same determinant bit for bit.
template <int NR, bool INV>
__device__ __forceinline__ double md_gj_nr(const double *aa, int ld, const int *rc, const int *ro, double (&b)[NR][NR]) {
  double a[NR][NR];
#pragma unroll
  for (int ir = 0; ir < NR; ir++)
#pragma unroll
    for (int jr = 0; jr < NR; jr++) {
      a[ir][jr] = aa[(size_t)rc[ir] * ld + ro[jr]];
      if (INV) b[ir][jr] = (ir == jr) ? 1.0 : 0.0;
    }
  double det = 1.0;
#pragma unroll
  for (int c = 0; c < NR; c++) {
    // first row of largest |a[r][c]| (the running maximum kept in a register:
    // indexing a by p would move the matrix to local memory)
    int p = c;
    double amax = fabs(a[c][c]);
#pragma unroll
    for (int r = c + 1; r < NR; r++)
      if (fabs(a[r][c]) > amax) {
        amax = fabs(a[r][c]);
        p = r;
      }
    if (p != c) {
      det = -det;
#pragma unroll
      for (int k = 0; k < NR; k++) {
        double ta = a[c][k], pa = 0, tb = INV ? b[c][k] : 0.0, pb = 0;
#pragma unroll
        for (int r = c + 1; r < NR; r++)
          if (r == p) {
            pa = a[r][k];
            if (INV) pb = b[r][k];
          }
        a[c][k] = pa;
        if (INV) b[c][k] = pb;
#pragma unroll
        for (int r = c + 1; r < NR; r++)
          if (r == p) {
            a[r][k] = ta;
            if (INV) b[r][k] = tb;
          }
      }
    }
    const double piv = a[c][c];
    det *= piv;
    const double pinv = 1.0 / piv;
#pragma unroll
    for (int k = 0; k < NR; k++) {
      a[c][k] *= pinv;
      if (INV) b[c][k] *= pinv;
    }
#pragma unroll
    for (int r = 0; r < NR; r++) {
      if (r == c) continue;
      const double f = a[r][c];
      if (f == 0.0) continue;
#pragma unroll
      for (int k = 0; k < NR; k++) {
        a[r][k] -= f * a[c][k];
        if (INV) b[r][k] -= f * b[c][k];
      }
    }
  }
  return det;
}

// determinant of the excitation matrix of e (register-resident for every
// excitation order)
__device__ __forceinline__ double md_small_det(const double *aa, int ld, const int *e) {
  const int nr = e[0];
  const int *rc = e + 1, *ro = e + 1 + CW_MD_MEX;
  if (nr == 1) return aa[(size_t)rc[0] * ld + ro[0]];
  if (nr == 2) {
    const double w0 = aa[(size_t)rc[0] * ld + ro[0]], w1 = aa[(size_t)rc[1] * ld + ro[0]];
    const double w2 = aa[(size_t)rc[0] * ld + ro[1]], w3 = aa[(size_t)rc[1] * ld + ro[1]];
    return w0 * w3 - w2 * w1;
  }
  if (nr == 3) {
    double b[3][3];
    return md_gj_nr<3, false>(aa, ld, rc, ro, b);
  }
  double b[4][4];
  return md_gj_nr<4, false>(aa, ld, rc, ro, b);
}

// ceq * M^-1 of excitation e added into Y[rc][ro] (atomics), M^-1 in
// registers
template <int NR>
__device__ __forceinline__ void md_y_add_nr(const double *aa, int ld, const int *e, double ceq, double *Y) {
  const int *rc = e + 1, *ro = e + 1 + CW_MD_MEX;
  double b[NR][NR];
  md_gj_nr<NR, true>(aa, ld, rc, ro, b);
#pragma unroll
  for (int ir = 0; ir < NR; ir++)
#pragma unroll
    for (int jr = 0; jr < NR; jr++) atomicAdd(&Y[rc[ir] * ld + ro[jr]], ceq * b[jr][ir]);
}

// determinant and inverse of the excitation matrix M[ir][jr] =
// aa[rc[ir]][ro[jr]] (aa row stride ld); inverse stored column-major as
// CHAMP's wfmat: inv[jr + nr*ir] = (M^-1)(jr, ir)
__device__ __forceinline__ double md_small_inv(const double *aa, int ld, const int *e, double *inv) {
  const int nr = e[0];
  const int *rc = e + 1, *ro = e + 1 + CW_MD_MEX;
  if (nr == 1) {
    const double d = aa[(size_t)rc[0] * ld + ro[0]];
    inv[0] = 1.0 / d;
    return d;
  }
  if (nr == 2) {
    const double w0 = aa[(size_t)rc[0] * ld + ro[0]], w1 = aa[(size_t)rc[1] * ld + ro[0]];
    const double w2 = aa[(size_t)rc[0] * ld + ro[1]], w3 = aa[(size_t)rc[1] * ld + ro[1]];
    const double d = w0 * w3 - w2 * w1, di = 1.0 / d;
    inv[0] = w3 * di;
    inv[1] = -w1 * di;
    inv[2] = -w2 * di;
    inv[3] = w0 * di;
    return d;
  }
  // Gauss-Jordan with partial pivoting on the column-major copy
  double a[CW_MD_MEX * CW_MD_MEX], b[CW_MD_MEX * CW_MD_MEX];
  for (int jr = 0; jr < nr; jr++)
    for (int ir = 0; ir < nr; ir++) {
      a[ir + nr * jr] = aa[(size_t)rc[ir] * ld + ro[jr]];
      b[ir + nr * jr] = (ir == jr) ? 1.0 : 0.0;
    }
  double det = 1.0;
  for (int c = 0; c < nr; c++) {
    int p = c;
    for (int r = c + 1; r < nr; r++)
      if (fabs(a[r + nr * c]) > fabs(a[p + nr * c])) p = r;
    if (p != c) {
      det = -det;
      for (int k = 0; k < nr; k++) {
        double t = a[c + nr * k]; a[c + nr * k] = a[p + nr * k]; a[p + nr * k] = t;
        t = b[c + nr * k]; b[c + nr * k] = b[p + nr * k]; b[p + nr * k] = t;
      }
    }
    const double piv = a[c + nr * c];
    det *= piv;
    const double pinv = 1.0 / piv;
    for (int k = 0; k < nr; k++) {
      a[c + nr * k] *= pinv;
      b[c + nr * k] *= pinv;
    }
    for (int r = 0; r < nr; r++) {
      if (r == c) continue;
      const double f = a[r + nr * c];
      if (f == 0.0) continue;
      for (int k = 0; k < nr; k++) {
        a[r + nr * k] -= f * a[c + nr * k];
        b[r + nr * k] -= f * b[c + nr * k];
      }
    }
  }
  for (int t = 0; t < nr * nr; t++) inv[t] = b[t];
  return det;
}

// det(M) and z = M^-1 b for the excitation matrix M[ir][jr] =
// aa[rc[ir]][ro[jr]] and b[ir] = cvec[rc[ir]]: Gaussian elimination with
// partial pivoting, fully unrolled in registers for NR <= 4.
template <int NR>
__device__ __forceinline__ double md_solve_nr(const double *aa, int ld, const int *rc, const int *ro,
                                             const double *cvec, double *z) {
  double a[NR][NR], b[NR];
#pragma unroll
  for (int ir = 0; ir < NR; ir++) {
#pragma unroll
    for (int jr = 0; jr < NR; jr++) a[ir][jr] = aa[(size_t)rc[ir] * ld + ro[jr]];
    b[ir] = cvec[rc[ir]];
  }
  // M z = b with M[ir][jr]: eliminate over columns jr (unknown z[jr])
  double det = 1.0;
#pragma unroll
  for (int c = 0; c < NR; c++) {
    // first row of largest |a[r][c]| (the running maximum kept in a register:
    // indexing a by p would move the matrix to local memory)
    int p = c;
    double amax = fabs(a[c][c]);
#pragma unroll
    for (int r = c + 1; r < NR; r++)
      if (fabs(a[r][c]) > amax) {
        amax = fabs(a[r][c]);
        p = r;
      }
    if (p != c) {
      det = -det;
#pragma unroll
      for (int k = 0; k < NR; k++) {
        // swap rows p and c without dynamic indexing: select per element
        double tc = a[c][k], tp = 0;
#pragma unroll
        for (int r = c + 1; r < NR; r++)
          if (r == p) tp = a[r][k];
        a[c][k] = tp;
#pragma unroll
        for (int r = c + 1; r < NR; r++)
          if (r == p) a[r][k] = tc;
      }
      double tc = b[c], tp = 0;
#pragma unroll
      for (int r = c + 1; r < NR; r++)
        if (r == p) tp = b[r];
      b[c] = tp;
#pragma unroll
      for (int r = c + 1; r < NR; r++)
        if (r == p) b[r] = tc;
    }
    det *= a[c][c];
    const double pinv = 1.0 / a[c][c];
#pragma unroll
    for (int r = c + 1; r < NR; r++) {
      const double f = a[r][c] * pinv;
#pragma unroll
      for (int k = c; k < NR; k++) a[r][k] -= f * a[c][k];
      b[r] -= f * b[c];
    }
  }
#pragma unroll
  for (int c = NR - 1; c >= 0; c--) {
    double v = b[c];
#pragma unroll
    for (int k = c + 1; k < NR; k++) v -= a[c][k] * z[k];
    z[c] = v / a[c][c];
  }
  return det;
}

// excitation ratio d = det(M) and the drift contraction sum_jr t[ro[jr]] z[jr]
// with z = M^-1 cvec[rc] (t: 3 components, row stride tstride)
__device__ __forceinline__ double md_ratio_contract(const double *aa, int ld, const int *e, const double *cvec,
                                                    const double *t, int tstride, double g[3]) {
  const int nr = e[0];
  const int *rc = e + 1, *ro = e + 1 + CW_MD_MEX;
  double z[CW_MD_MEX], d;
  switch (nr) {
    case 1: d = md_solve_nr<1>(aa, ld, rc, ro, cvec, z); break;
    case 2: d = md_solve_nr<2>(aa, ld, rc, ro, cvec, z); break;
    case 3: d = md_solve_nr<3>(aa, ld, rc, ro, cvec, z); break;
    default: d = md_solve_nr<4>(aa, ld, rc, ro, cvec, z); break;
  }
  g[0] = g[1] = g[2] = 0;
#pragma unroll
  for (int jr = 0; jr < CW_MD_MEX; jr++) {
    if (jr >= nr) break;
    const int v = ro[jr];
    g[0] += t[v] * z[jr];
    g[1] += t[tstride + v] * z[jr];
    g[2] += t[2 * tstride + v] * z[jr];
  }
  return d;
}

template <int BS>
__device__ __forceinline__ double md_block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double r = 0;
  for (int k = 0; k < BS / 32; k++) r += red[k];
  __syncthreads();
  return r;  // valid on every thread
}

// orbital rows of every orbital and the kinetic B of one electron chunk
__global__ void k_md_scatter(const __grid_constant__ CSys cs, WState st, MdBuf md, const double *orball, int e0, int ne) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int N = cs.N, O = cs.Oa;
  if (t >= (long)st.W * ne * O) return;
  const int o = (int)(t % O);
  const long we = t / O;
  const int el = (int)(we % ne), w = (int)(we / ne), e = e0 + el;
  const double *ob = orball + (size_t)we * 5 * O;
  const double v = ob[o], d0 = ob[O + o], d1 = ob[2 * O + o], d2 = ob[3 * O + o], lap = ob[4 * O + o];
  md.orbA[((size_t)w * N + e) * O + o] = v;
  md.dorbA[(((size_t)w * 3 + 0) * N + e) * O + o] = d0;
  md.dorbA[(((size_t)w * 3 + 1) * N + e) * O + o] = d1;
  md.dorbA[(((size_t)w * 3 + 2) * N + e) * O + o] = d2;
  const double vx = st.fjo[((size_t)w * 3 + 0) * N + e], vy = st.fjo[((size_t)w * 3 + 1) * N + e],
               vz = st.fjo[((size_t)w * 3 + 2) * N + e];
  md.bkin[((size_t)w * N + e) * O + o] = -0.5 * (lap + 2 * (vx * d0 + vy * d1 + vz * d2));
}

// G_s (and its kref-equivalent part) from the other spin's ratios; smem-free
__device__ void md_form_G(const CSys &cs, const MdTab &tab, const MdBuf &md, int w, int s, double *G, double *red,
                          const double *cdet) {
  const int NU = cs.md_nuniq[s];
  for (int kk = threadIdx.x; kk <= NU; kk += blockDim.x) G[kk] = 0.0;
  __syncthreads();
  const double *dother = md.dd + ((size_t)w * 2 + (1 - s)) * tab.numax;
  double gref = 0.0;
  for (int k = threadIdx.x; k < cs.ndet; k += blockDim.x) {
    const int kws = tab.kw[2 * k + s], kwo = tab.kw[2 * k + (1 - s)];
    const double v = cdet[k] * (kwo >= 0 ? dother[kwo] : 1.0);
    if (kws >= 0) atomicAdd(&G[kws], v);
    else gref += v;
  }
  gref = md_block_sum<128>(gref, red);
  if (threadIdx.x == 0) G[NU] = gref;
  __syncthreads();
}

// Y_s into shared memory Y[n][O] from aa (row stride O), ratios dd and G
__device__ void md_form_Y(const CSys &cs, const MdTab &tab, int s, const double *aa, const double *dd, const double *G, double *Y) {
  const int n = s == 0 ? cs.nup : cs.ndn, O = cs.Oa, NU = cs.md_nuniq[s];
  for (int t = threadIdx.x; t < n * O; t += blockDim.x) Y[t] = 0.0;
  __syncthreads();
  for (int kk = threadIdx.x; kk < NU; kk += blockDim.x) {
    const int *e = md_exc(tab, s, kk);
    const double ceq = dd[kk] * G[kk];
    switch (e[0]) {
      case 1: md_y_add_nr<1>(aa, O, e, ceq, Y); break;
      case 2: {
        double inv[4];
        md_small_inv(aa, O, e, inv);
#pragma unroll
        for (int ir = 0; ir < 2; ir++)
#pragma unroll
          for (int jr = 0; jr < 2; jr++) atomicAdd(&Y[e[1 + ir] * O + e[1 + CW_MD_MEX + jr]], ceq * inv[jr + 2 * ir]);
        break;
      }
      case 3: md_y_add_nr<3>(aa, O, e, ceq, Y); break;
      default: md_y_add_nr<4>(aa, O, e, ceq, Y); break;
    }
  }
  __syncthreads();
}

// multideterminante_grad: velocity of electron e (spin s, slot jel) from
// the drift operands: column c of A^-1 (c[irep] = slmi[irep + n*jel]),
// gradients b_k[v] of every orbital at the electron, aa and Y (row stride
// O); lanes of one warp over the virtual orbitals.  Returns the
// detratio-scaled sum on every lane.
__device__ void md_velocity_warp(const CSys &cs, int s, const double *c, const double *b0, const double *b1, const double *b2,
                                 int bstride_slot /*1*/, const double *aa, const double *Y, const int *slot_orb,
                                 double detratio, double vel[3]) {
  const int n = s == 0 ? cs.nup : cs.ndn, O = cs.Oa;
  const int ivirt = cs.md_ivirt[s], iactv = cs.md_iactv[s];
  const int lane = threadIdx.x & 31;
  double a0 = 0, a1 = 0, a2 = 0;
  for (int v = ivirt + lane; v < O; v += 32) {
    double u = 0;
    for (int irep = iactv; irep < n; irep++) u += Y[irep * O + v] * c[irep];
    double t0 = 0, t1 = 0, t2 = 0;
    for (int j = 0; j < n; j++) {
      const double a = aa[j * O + v];
      const int oj = slot_orb[j];
      t0 += b0[oj] * a;
      t1 += b1[oj] * a;
      t2 += b2[oj] * a;
    }
    a0 += (b0[v] - t0) * u;
    a1 += (b1[v] - t1) * u;
    a2 += (b2[v] - t2) * u;
  }
  (void)bstride_slot;
  vel[0] = warp_sum(a0) * detratio;
  vel[1] = warp_sum(a1) * detratio;
  vel[2] = warp_sum(a2) * detratio;
}

// ---------------------------------------------------------------------------
// hpsi part: CTA (128 threads) per walker.  Shared: slmi of one spin (n*n),
// X and X_kin (n*n each), Y (n*O), G (numax+1), reduction scratch.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_md_hpsi(const __grid_constant__ CSys cs, WState st, MdBuf md, MdTab tab, GSys g) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  const int N = cs.N, O = cs.Oa, nmax = cs.nmax;
  extern __shared__ __align__(16) double smem[];
  double *Sl = smem;                       // nmax*nmax
  double *X = Sl + nmax * nmax;            // nmax*nmax
  double *Xk = X + nmax * nmax;            // nmax*nmax
  double *T = Xk + nmax * nmax;            // nmax*nmax work
  double *Y = T + nmax * nmax;             // nmax*O
  double *G = Y + (size_t)nmax * O;        // numax+1
  double *Tm = G + tab.numax + 1;          // nmax*O tildem of B = bkin + bnl (several states only)
  double *Tk = Tm + (size_t)nmax * O;      // nmax*O tildem of bkin
  __shared__ double red[4];
  // 1. aa and excitation ratios of both spins
  for (int s = 0; s < 2; s++) {
    const int n = s == 0 ? cs.nup : cs.ndn, ish = s == 0 ? 0 : cs.nup;
    if (n == 0) continue;
    const double *slmi = st.slmi + ((size_t)w * 2 + s) * nmax * nmax;
    __syncthreads();
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) Sl[t] = slmi[t];
    __syncthreads();
    double *aa = md.aa + ((size_t)w * 2 + s) * nmax * O;
    for (int t = threadIdx.x; t < n * O; t += blockDim.x) {
      const int irep = t / O, v = t % O;
      double d = 0;
      for (int e = 0; e < n; e++) d += Sl[irep + n * e] * md.orbA[((size_t)w * N + ish + e) * O + v];
      aa[t] = d;
    }
    __syncthreads();
    double *dd = md.dd + ((size_t)w * 2 + s) * tab.numax;
    for (int kk = threadIdx.x; kk < cs.md_nuniq[s]; kk += blockDim.x) dd[kk] = md_small_det(aa, O, md_exc(tab, s, kk));
  }
  __syncthreads();
  // 2. S of every state (state 0 drives the walk)
  const int ns = cs.nstates;
  __shared__ double s_S[CW_MAX_STATES], s_den[CW_MAX_STATES], s_dek[CW_MAX_STATES];
  for (int stt = 0; stt < ns; stt++) {
    const double *cd = tab.cdet + (size_t)stt * cs.ndet;
    double sp = 0;
    for (int k = threadIdx.x; k < cs.ndet; k += blockDim.x) {
      const int k0 = tab.kw[2 * k], k1 = tab.kw[2 * k + 1];
      const double d0 = k0 >= 0 ? md.dd[((size_t)w * 2 + 0) * tab.numax + k0] : 1.0;
      const double d1 = k1 >= 0 ? md.dd[((size_t)w * 2 + 1) * tab.numax + k1] : 1.0;
      sp += d0 * d1 * cd[k];
    }
    sp = md_block_sum<128>(sp, red);
    if (threadIdx.x == 0) {
      s_S[stt] = sp;
      s_den[stt] = 0;
      s_dek[stt] = 0;
    }
  }
  // 3. per spin: tildem = A^-1 B - X Phi (state-independent), then per state
  //    G, Y and the energy corrections sum_{irep>=iactv, v>=ivirt} Y tildem
  for (int s = 0; s < 2; s++) {
    const int n = s == 0 ? cs.nup : cs.ndn, ish = s == 0 ? 0 : cs.nup;
    if (n == 0) continue;
    const double *aa = md.aa + ((size_t)w * 2 + s) * nmax * O;
    const double *dd = md.dd + ((size_t)w * 2 + s) * tab.numax;
    // X = A^-1 B_occ A^-1 (bxmatrix) for B = bkin + bnl and for bkin
    const double *slmi = st.slmi + ((size_t)w * 2 + s) * nmax * nmax;
    __syncthreads();
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) Sl[t] = slmi[t];
    __syncthreads();
    for (int pass = 0; pass < 2; pass++) {
      double *Xo = pass == 0 ? X : Xk;
      // T[j][m] = sum_i B(occ_i, e_j) slmi[i + n m]
      for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
        const int j = t / n, m = t % n;
        double a = 0;
        for (int i = 0; i < n; i++) {
          const int oi = g.slot_orb[s * nmax + i];
          const size_t bi = ((size_t)w * N + ish + j) * O + oi;
          const double bv = pass == 0 ? md.bkin[bi] + md.bnl[bi] : md.bkin[bi];
          a += bv * Sl[i + n * m];
        }
        T[t] = a;
      }
      __syncthreads();
      // X[m][np] (CHAMP xmat(m + n*np)) = sum_j T[j][m] slmi[np + n j]
      for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
        const int m = t / n, np = t % n;
        double a = 0;
        for (int j = 0; j < n; j++) a += T[j * n + m] * Sl[np + n * j];
        Xo[m * n + np] = a;
      }
      __syncthreads();
    }
    const int ivirt = cs.md_ivirt[s], iactv = cs.md_iactv[s];
    const int nv = O - ivirt, na = n - iactv;
    if (ns == 1) {
      // one state: Y first, then tildem contracted with it on the fly
      md_form_G(cs, tab, md, w, s, G, red, tab.cdet);
      md_form_Y(cs, tab, s, aa, dd, G, Y);
      double *yg = md.ymat + ((size_t)w * 2 + s) * nmax * O;
      for (int t = threadIdx.x; t < n * O; t += blockDim.x) yg[t] = Y[t];
    }
    double den1 = 0, dek1 = 0;
    for (int t = threadIdx.x; t < nv * na; t += blockDim.x) {
      const int irep = iactv + t / nv, v = ivirt + t % nv;
      double d2 = 0, d3 = 0, d4 = 0, d5 = 0;
      for (int e = 0; e < n; e++) {
        const size_t bi = ((size_t)w * N + ish + e) * O + v;
        const double ov = md.orbA[bi];
        const double sl = Sl[irep + n * e];
        d2 += sl * (md.bkin[bi] + md.bnl[bi]);
        d3 += X[e * n + irep] * ov;
        d4 += sl * md.bkin[bi];
        d5 += Xk[e * n + irep] * ov;
      }
      if (ns == 1) {
        const double y = Y[irep * O + v];
        den1 += y * (d2 - d3);
        dek1 += y * (d4 - d5);
      } else {
        Tm[t] = d2 - d3;
        Tk[t] = d4 - d5;
      }
    }
    if (ns == 1) {
      den1 = md_block_sum<128>(den1, red);
      dek1 = md_block_sum<128>(dek1, red);
      if (threadIdx.x == 0) {
        s_den[0] += den1;
        s_dek[0] += dek1;
      }
      __syncthreads();
      continue;
    }
    for (int stt = 0; stt < ns; stt++) {
      md_form_G(cs, tab, md, w, s, G, red, tab.cdet + (size_t)stt * cs.ndet);
      md_form_Y(cs, tab, s, aa, dd, G, Y);
      if (stt == 0) {
        double *yg = md.ymat + ((size_t)w * 2 + s) * nmax * O;
        for (int t = threadIdx.x; t < n * O; t += blockDim.x) yg[t] = Y[t];
      }
      double den = 0, dek = 0;
      for (int t = threadIdx.x; t < nv * na; t += blockDim.x) {
        const double y = Y[(iactv + t / nv) * O + ivirt + t % nv];
        den += y * Tm[t];
        dek += y * Tk[t];
      }
      den = md_block_sum<128>(den, red);
      dek = md_block_sum<128>(dek, red);
      if (threadIdx.x == 0) {
        s_den[stt] += den;
        s_dek[stt] += dek;
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    md.S[w] = s_S[0];
    md.den[2 * w] = s_den[0] / s_S[0];
    md.den[2 * w + 1] = s_dek[0] / s_S[0];
    if (md.S_ms)
      for (int stt = 0; stt < ns; stt++) {
        md.S_ms[(size_t)w * ns + stt] = s_S[stt];
        md.den_ms[((size_t)w * ns + stt) * 2] = s_den[stt] / s_S[stt];
        md.den_ms[((size_t)w * ns + stt) * 2 + 1] = s_dek[stt] / s_S[stt];
      }
  }
}

// optci_deloc (vmc/optci.f90:49-51): d ln psi / d c_k = sgn_k D_k / psi_D of
// every determinant (sgn_k: the orbital-order sign folded into the internal
// coefficients, so the derivative is taken for the input coefficients), in
// both walker-major and determinant-major layouts (the latter feeds the
// overlap GEMM).  CTA per walker.
// (columns off .. off+ndet-1 of the optimisation vector o, row stride np,
// and the same rows of its transpose ot [np][W])
__global__ void k_md_ci_o(const __grid_constant__ CSys cs, WState st, MdBuf md, MdTab tab, const double *sgn, double *o, double *ot, int np,
                          int off) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  const double iS = 1.0 / md.S[w];
  for (int k = threadIdx.x; k < cs.ndet; k += blockDim.x) {
    const int k0 = tab.kw[2 * k], k1 = tab.kw[2 * k + 1];
    const double d0 = k0 >= 0 ? md.dd[((size_t)w * 2 + 0) * tab.numax + k0] : 1.0;
    const double d1 = k1 >= 0 ? md.dd[((size_t)w * 2 + 1) * tab.numax + k1] : 1.0;
    const double v = sgn[k] * (d0 * d1 * iS);
    o[(size_t)w * np + off + k] = v;
    ot[(size_t)(off + k) * st.W + w] = v;
  }
}

// SR sums (optwf_store's sr_o contracted per sample): sum_w O_k and
// sum_w E_w O_k over the np entries of the optimisation vector, thread per
// entry, walkers in order
__global__ void k_sr_accum(WState st, const double *o, int np, double *sr_o, double *sr_eo) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np) return;
  double a = 0, b = 0;
  for (int w = 0; w < st.W; w++) {
    const double v = o[(size_t)w * np + k];
    a += v;
    b += st.eold[w] * v;
  }
  sr_o[k] += a;
  sr_eo[k] += b;
}

__global__ void k_add_inplace(double *dst, const double *src, size_t n) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] += src[t];
}

// pseudopotential B matrix: bnl[w][e][o] = sum_m P[w][e][m] coef(m, o) is
// a GEMM launched by the host; this kernel only clears P before k_ecp
__global__ void k_md_zero(double *p, size_t n) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[t] = 0.0;
}

// drift operands t_k[v] = b_k[v] - sum_j b_k[occ_j] aa[j][v] of one
// electron (multideterminante_grad's gmat without the slmi factor), shared.
// The occupied orbitals' values b_k[occ_j] are staged in bo [3][n] first, so
// the column sums read shared memory only.  Ends with a block barrier.
__device__ __forceinline__ void md_form_t(const CSys &cs, int s, const double *b0, const double *b1, const double *b2,
                                          const double *aa, const int *slot_orb, double *t, double *bo) {
  const int n = s == 0 ? cs.nup : cs.ndn, O = cs.Oa, ivirt = cs.md_ivirt[s];
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const int oj = slot_orb[j];
    bo[j] = b0[oj];
    bo[n + j] = b1[oj];
    bo[2 * n + j] = b2[oj];
  }
  __syncthreads();
  for (int v = ivirt + threadIdx.x; v < O; v += blockDim.x) {
    double t0 = 0, t1 = 0, t2 = 0;
    for (int j = 0; j < n; j++) {
      const double a = aa[j * O + v];
      t0 += bo[j] * a;
      t1 += bo[n + j] * a;
      t2 += bo[2 * n + j] * a;
    }
    t[v] = b0[v] - t0;
    t[O + v] = b1[v] - t1;
    t[2 * O + v] = b2[v] - t2;
  }
  __syncthreads();
}

// drift correction of every electron at the current configuration right
// after hpsi (dmc_ps :516), from the Y matrix hpsi just built: warp per
// (walker, electron); vall [W][N][3]
__global__ void k_md_drift_all(const __grid_constant__ CSys cs, WState st, MdBuf md, GSys g, double *vall) {
  const long gw = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int N = cs.N, O = cs.Oa, nmax = cs.nmax;
  if (gw >= (long)st.W * N) return;
  const int w = (int)(gw / N), e = (int)(gw % N);
  const int s = e < cs.nup ? 0 : 1, n = s == 0 ? cs.nup : cs.ndn, ish = s == 0 ? 0 : cs.nup;
  const double *c = st.slmi + ((size_t)w * 2 + s) * nmax * nmax + (size_t)n * (e - ish);
  const double *b0 = md.dorbA + (((size_t)w * 3 + 0) * N + e) * O;
  const double *b1 = md.dorbA + (((size_t)w * 3 + 1) * N + e) * O;
  const double *b2 = md.dorbA + (((size_t)w * 3 + 2) * N + e) * O;
  const double detratio = st.detiab[2 * w] * st.detiab[2 * w + 1] / st.psido[w];
  double vel[3];
  md_velocity_warp(cs, s, c, b0, b1, b2, 1, md.aa + ((size_t)w * 2 + s) * nmax * O,
                   md.ymat + ((size_t)w * 2 + s) * nmax * O, g.slot_orb + s * nmax, detratio, vel);
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; k++) vall[((size_t)w * N + e) * 3 + k] = vel[k];
}

// G_s before the moves of spin s: CTA (128) per walker.  s < 0: the spin of
// each walker's T-move electron (ms[w].tel; walkers without one are skipped)
__global__ void __launch_bounds__(128) k_md_phase(const __grid_constant__ CSys cs, WState st, MdBuf md, MdTab tab, int s,
                                                  const MoveScratch *ms) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  if (s < 0) {
    if (ms[w].igeo) return;
    s = ms[w].tel < cs.nup ? 0 : 1;
  }
  extern __shared__ __align__(16) double smem[];
  double *G = smem;  // numax+1
  __shared__ double red[4];
  const int ng = cs.iguiding > 0 ? cs.nstates : 1;  // states whose G the moves need
  for (int stt = 0; stt < ng; stt++) {
    md_form_G(cs, tab, md, w, s, G, red, tab.cdet + (size_t)stt * cs.ndet);
    double *gG = md.G + ((size_t)w * ng + stt) * (tab.numax + 1);
    for (int kk = threadIdx.x; kk <= cs.md_nuniq[s]; kk += blockDim.x) gG[kk] = G[kk];
    __syncthreads();
  }
}

// multideterminante_grad at the old position of electron iel, without the Y
// matrix: vel = detratio * sum_kk d_kk G_kk sum_jr t[ro_jr] (M_kk^-1 c)[jr]
// with c the column of A^-1 of the electron (the Y contraction regrouped per
// excitation).  CTA (128) per walker; shared: c (nmax), t (3*O), aa (nmax*O).
__global__ void __launch_bounds__(128, 5) k_md_drift_old(const __grid_constant__ CSys cs, WState st, MdBuf md, MdTab tab, GSys g, int iel) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  const int N = cs.N, O = cs.Oa, nmax = cs.nmax;
  const int s = iel < cs.nup ? 0 : 1, n = s == 0 ? cs.nup : cs.ndn, ish = s == 0 ? 0 : cs.nup;
  extern __shared__ __align__(16) double smem[];
  double *c = smem;              // nmax
  double *t = c + nmax;          // 3*O
  double *A = t + 3 * O;         // nmax*O
  double *bo = A + (size_t)nmax * O;  // 3*nmax
  __shared__ double red[4];
  const double *sl = st.slmi + ((size_t)w * 2 + s) * nmax * nmax + (size_t)n * (iel - ish);
  const double *aa = md.aa + ((size_t)w * 2 + s) * nmax * O;
  for (int q = threadIdx.x; q < n * O; q += blockDim.x) cp_async8(A + q, aa + q);
  for (int j = threadIdx.x; j < n; j += blockDim.x) c[j] = sl[j];
  cp_async8_wait();
  __syncthreads();
  md_form_t(cs, s, md.dorbA + (((size_t)w * 3 + 0) * N + iel) * O, md.dorbA + (((size_t)w * 3 + 1) * N + iel) * O,
            md.dorbA + (((size_t)w * 3 + 2) * N + iel) * O, A, g.slot_orb + s * nmax, t, bo);
  __syncthreads();
  const double *G = md.G + (size_t)w * (cs.iguiding > 0 ? cs.nstates : 1) * (tab.numax + 1);
  if (cs.iguiding > 0) {
    // guiding (determinante.f90:150-171): sum_i w_i (S_i/S_1)^2 v_i / psi2g,
    // v_i the velocity of state i (its own G, 1/S_i)
    const int ns = cs.nstates;
    const double *S = md.S_ms + (size_t)w * ns;
    double vg[3] = {0, 0, 0};
    for (int stt = 0; stt < ns; stt++) {
      const double *Gs = G + (size_t)stt * (tab.numax + 1);
      double a0 = 0, a1 = 0, a2 = 0;
      for (int kk = threadIdx.x; kk < cs.md_nuniq[s]; kk += blockDim.x) {
        double gv[3];
        const double d = md_ratio_contract(A, O, md_exc(tab, s, kk), c, t, O, gv);
        const double ce = d * Gs[kk];
        a0 += ce * gv[0];
        a1 += ce * gv[1];
        a2 += ce * gv[2];
      }
      a0 = md_block_sum<128>(a0, red);
      a1 = md_block_sum<128>(a1, red);
      a2 = md_block_sum<128>(a2, red);
      const double r = S[stt] / S[0], f = cs.wg[stt] * r * r / S[stt];
      vg[0] += f * a0;
      vg[1] += f * a1;
      vg[2] += f * a2;
    }
    if (threadIdx.x == 0) {
      const double gi = 1.0 / md_psig(cs, S, ns);
      md.velo[3 * w] = vg[0] * gi;
      md.velo[3 * w + 1] = vg[1] * gi;
      md.velo[3 * w + 2] = vg[2] * gi;
    }
    return;
  }
  double v0 = 0, v1 = 0, v2 = 0;
  const int NU = cs.md_nuniq[s];
  MdExcPf nx;
  if ((int)threadIdx.x < NU) nx.load(tab, s, threadIdx.x, G);
  for (int kk = threadIdx.x; kk < NU; kk += blockDim.x) {
    const MdExcPf cur = nx;
    if (kk + (int)blockDim.x < NU) nx.load(tab, s, kk + blockDim.x, G);
    double gv[3];
    const double d = md_ratio_contract(A, O, cur.e, c, t, O, gv);
    const double ce = d * cur.g;
    v0 += ce * gv[0];
    v1 += ce * gv[1];
    v2 += ce * gv[2];
  }
  v0 = md_block_sum<128>(v0, red);
  v1 = md_block_sum<128>(v1, red);
  v2 = md_block_sum<128>(v2, red);
  if (threadIdx.x == 0) {
    const double detratio = st.detiab[2 * w] * st.detiab[2 * w + 1] / st.psido[w];
    md.velo[3 * w] = v0 * detratio;
    md.velo[3 * w + 1] = v1 * detratio;
    md.velo[3 * w + 2] = v2 * detratio;
  }
}

// multideterminante at the proposed position of electron iel: CTA (128)
// per walker.  aa_new = aa + c (x) w with w[v] = (psi_new[v] - sum_i
// phi_new(occ_i) aa[i][v]) / R (the Sherman-Morrison form of
// slmin * orb_new), the excitation ratios, S, psi_D and the drift at the new
// point.  Shared: c, slot values (nmax each), w (O), t (3*O), aa_new (nmax*O).
__global__ void __launch_bounds__(128, 5) k_md_move(const __grid_constant__ CSys cs, WState st, MoveBuf mb, MdBuf md, MdTab tab, GSys g, int iel) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  if (iel < 0) iel = mb.ms[w].tel;  // T-move: each walker's own electron
  const int O = cs.Oa, nmax = cs.nmax;
  const int s = iel < cs.nup ? 0 : 1, n = s == 0 ? cs.nup : cs.ndn, ish = s == 0 ? 0 : cs.nup;
  const int ivirt = cs.md_ivirt[s], NU = cs.md_nuniq[s];
  extern __shared__ __align__(16) double smem[];
  double *c = smem;                       // nmax
  double *ps = c + nmax;                  // nmax
  double *wv = ps + nmax;                 // O
  double *t = wv + O;                     // 3*O
  double *An = t + 3 * O;                 // nmax*O
  double *bo = An + (size_t)nmax * O;     // 3*nmax
  __shared__ double red[4];
  __shared__ double s_R;
  if (mb.ms[w].igeo) {
    if (threadIdx.x == 0) md.psidn[w] = 0.0;
    return;
  }
  const double *orbn = mb.orbn + (size_t)w * 4 * O;
  const double *sl = st.slmi + ((size_t)w * 2 + s) * nmax * nmax + (size_t)n * (iel - ish);
  // the spin's aa block lands in shared memory while the ratio is formed
  const double *aa = md.aa + ((size_t)w * 2 + s) * nmax * O;
  for (int q = threadIdx.x; q < n * O; q += blockDim.x) cp_async8(An + q, aa + q);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    c[j] = sl[j];
    ps[j] = orbn[g.slot_orb[s * nmax + j]];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0;
    for (int j = 0; j < n; j++) r += c[j] * ps[j];
    s_R = r;
  }
  cp_async8_wait();
  __syncthreads();
  const double R = s_R;
  if (R == 0.0) {
    if (threadIdx.x == 0) md.psidn[w] = 0.0;
    return;
  }
  for (int v = ivirt + threadIdx.x; v < O; v += blockDim.x) {
    double tt = 0;
    for (int i = 0; i < n; i++) tt += ps[i] * An[i * O + v];
    wv[v] = (orbn[v] - tt) / R;
  }
  __syncthreads();
  for (int i = threadIdx.x >> 5; i < n; i += blockDim.x >> 5)  // warps over rows, lanes over columns
    for (int v = threadIdx.x & 31; v < O; v += 32)
      An[i * O + v] = v >= ivirt ? An[i * O + v] + c[i] * wv[v] : 0.0;
  __syncthreads();
  // column iel of the updated inverse is c / R; drift operands at the new point
  md_form_t(cs, s, orbn + O, orbn + 2 * O, orbn + 3 * O, An, g.slot_orb + s * nmax, t, bo);
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) c[j] = c[j] / R;
  __syncthreads();
  const double *G = md.G + (size_t)w * (cs.iguiding > 0 ? cs.nstates : 1) * (tab.numax + 1);
  double *ddn = md.ddn + (size_t)w * tab.numax;
  if (cs.iguiding > 0) {
    // guiding: S and velocity of every state at the proposed point, psi2g there
    const int ns = cs.nstates;
    __shared__ double s_Sn[CW_MAX_STATES], s_v[CW_MAX_STATES][3];
    for (int stt = 0; stt < ns; stt++) {
      const double *Gs = G + (size_t)stt * (tab.numax + 1);
      double sp = 0, a0 = 0, a1 = 0, a2 = 0;
      for (int kk = threadIdx.x; kk < NU; kk += blockDim.x) {
        double gv[3];
        const double d = md_ratio_contract(An, O, md_exc(tab, s, kk), c, t, O, gv);
        if (stt == 0) ddn[kk] = d;
        const double ce = d * Gs[kk];
        sp += ce;
        a0 += ce * gv[0];
        a1 += ce * gv[1];
        a2 += ce * gv[2];
      }
      sp = md_block_sum<128>(sp, red) + Gs[NU];
      a0 = md_block_sum<128>(a0, red);
      a1 = md_block_sum<128>(a1, red);
      a2 = md_block_sum<128>(a2, red);
      if (threadIdx.x == 0) {
        s_Sn[stt] = sp;
        s_v[stt][0] = a0;
        s_v[stt][1] = a1;
        s_v[stt][2] = a2;
      }
    }
    if (threadIdx.x == 0) {
      const double detn_ref = st.detiab[2 * w + s] * R;
      const double dpair = s == 0 ? detn_ref * st.detiab[2 * w + 1] : st.detiab[2 * w] * detn_ref;
      const double g = md_psig(cs, s_Sn, ns), gi = 1.0 / g;
      double vg[3] = {0, 0, 0};
      for (int stt = 0; stt < ns; stt++) {
        const double r = s_Sn[stt] / s_Sn[0], f = cs.wg[stt] * r * r / s_Sn[stt];
        for (int k = 0; k < 3; k++) vg[k] += f * s_v[stt][k];
        md.Sn_ms[(size_t)w * ns + stt] = s_Sn[stt];
      }
      for (int k = 0; k < 3; k++) md.veln[3 * w + k] = vg[k] * gi;
      md.psidn[w] = dpair * s_Sn[0];
      md.Sn[w] = s_Sn[0];
      md.psi2gn[w] = g;
    }
    double *cv = md.cvec + (size_t)w * nmax;
    double *wgv = md.wvec + (size_t)w * O;
    for (int j = threadIdx.x; j < n; j += blockDim.x) cv[j] = c[j] * R;
    for (int v = ivirt + threadIdx.x; v < O; v += blockDim.x) wgv[v] = wv[v];
    return;
  }
  double sp = 0, v0 = 0, v1 = 0, v2 = 0;
  MdExcPf nx;
  if ((int)threadIdx.x < NU) nx.load(tab, s, threadIdx.x, G);
  for (int kk = threadIdx.x; kk < NU; kk += blockDim.x) {
    const MdExcPf cur = nx;
    if (kk + (int)blockDim.x < NU) nx.load(tab, s, kk + blockDim.x, G);
    double gv[3];
    const double d = md_ratio_contract(An, O, cur.e, c, t, O, gv);
    ddn[kk] = d;
    const double ce = d * cur.g;
    sp += ce;
    v0 += ce * gv[0];
    v1 += ce * gv[1];
    v2 += ce * gv[2];
  }
  const double Sn = md_block_sum<128>(sp, red) + G[NU];
  v0 = md_block_sum<128>(v0, red);
  v1 = md_block_sum<128>(v1, red);
  v2 = md_block_sum<128>(v2, red);
  if (threadIdx.x == 0) {
    const double detn_ref = st.detiab[2 * w + s] * R;
    const double dpair = s == 0 ? detn_ref * st.detiab[2 * w + 1] : st.detiab[2 * w] * detn_ref;
    const double psidn = dpair * Sn;
    const double detratio = dpair / psidn;
    md.veln[3 * w] = v0 * detratio;
    md.veln[3 * w + 1] = v1 * detratio;
    md.veln[3 * w + 2] = v2 * detratio;
    md.psidn[w] = psidn;
    md.Sn[w] = Sn;
  }
  // rank-1 factors for the commit (the inverse column before the move)
  double *cv = md.cvec + (size_t)w * nmax;
  double *wg = md.wvec + (size_t)w * O;
  for (int j = threadIdx.x; j < n; j += blockDim.x) cv[j] = c[j] * R;
  for (int v = ivirt + threadIdx.x; v < O; v += blockDim.x) wg[v] = wv[v];
}

// commit of an accepted move (after k_commit): aa += c (x) w on the
// virtual columns, ratios, S, and the gradient row of the moved electron
__global__ void k_md_commit(const __grid_constant__ CSys cs, WState st, MoveBuf mb, MdBuf md, MdTab tab, int iel) {
  const int w = blockIdx.x;
  if (w >= st.W || !mb.ms[w].acc) return;
  if (iel < 0) iel = mb.ms[w].tel;  // T-move: each walker's own electron
  const int N = cs.N, O = cs.Oa, nmax = cs.nmax;
  const int s = iel < cs.nup ? 0 : 1, n = s == 0 ? cs.nup : cs.ndn;
  const int ivirt = cs.md_ivirt[s];
  double *aa = md.aa + ((size_t)w * 2 + s) * nmax * O;
  const double *cv = md.cvec + (size_t)w * nmax;
  const double *wg = md.wvec + (size_t)w * O;
  for (int i = threadIdx.x >> 5; i < n; i += blockDim.x >> 5) {  // warps over rows, lanes over columns
    const double ci = cv[i];
    for (int v = ivirt + (threadIdx.x & 31); v < O; v += 32) aa[i * O + v] = aa[i * O + v] + ci * wg[v];
  }
  double *dd = md.dd + ((size_t)w * 2 + s) * tab.numax;
  for (int kk = threadIdx.x; kk < cs.md_nuniq[s]; kk += blockDim.x) dd[kk] = md.ddn[(size_t)w * tab.numax + kk];
  const double *orbn = mb.orbn + (size_t)w * 4 * O;
  for (int o = threadIdx.x; o < O; o += blockDim.x)
    for (int k = 0; k < 3; k++) md.dorbA[(((size_t)w * 3 + k) * N + iel) * O + o] = orbn[(1 + k) * O + o];
  if (threadIdx.x == 0) md.S[w] = md.Sn[w];
  if (md.Sn_ms)
    for (int stt = threadIdx.x; stt < cs.nstates; stt += blockDim.x)
      md.S_ms[(size_t)w * cs.nstates + stt] = md.Sn_ms[(size_t)w * cs.nstates + stt];
}

// multideterminant_tmove (dmc/multideterminant_tmove.f90:3): the
// excitations' part of every T-move element, after hpsi has built Y.  The
// element of electron i at quadrature point x_q gains
//   detratio * trj * sum_jrep (b(jrep) - sum_j b(occ_j) aa(j,jrep)) * Yc(jrep),
//   Yc(jrep) = sum_{irep >= iactv} Y(jrep, irep) slmi(irep, i),
// b the orbital values at x_q, trj the element's radial x Jastrow factor
// (tvtrj, written by k_ecp).  Regrouped per electron as a vector over the
// basis, Zb = coef Z with Z(v) = Yc(v) on the virtual columns minus, on each
// occupied orbital occ_j, sum_v aa(j,v) Yc(v), each point costs one basis
// evaluation and a dot product with Zb.  CTA (128) per walker; shared: Yc,
// Z (O each), the aa factors (nmax), Zb (K), per warp the basis prepass.
__global__ void __launch_bounds__(128) k_md_tmove(const __grid_constant__ CSys cs, WState st, MdBuf md, HBuf hb, GSys g) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  const int N = cs.N, M = cs.M, K = cs.K, O = cs.Oa, NQ = cs.nquad, nmax = cs.nmax;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  extern __shared__ __align__(16) double smem[];
  double *Yc = smem;                     // [O]
  double *Z = Yc + O;                    // [O]
  double *zo = Z + O;                    // [nmax]
  double *Zb = zo + nmax;                // [K]
  double *rec = Zb + K + (K & 1) + (size_t)wid * M * kCenRec;  // [M][kCenRec] per warp
  const double detratio = st.detiab[2 * w] * st.detiab[2 * w + 1] / st.psido[w];
  const double *sx = st.x + (size_t)w * 3 * N;
  const double *xqw = st.xq + (size_t)w * 3 * NQ;
  for (int i = 0; i < N; i++) {
    const double *trow = hb.tvtrj + ((size_t)w * N + i) * NQ * M;
    int any = 0;
    for (int k = threadIdx.x; k < NQ * M; k += blockDim.x)
      if (trow[k] != 0.0) any = 1;
    if (!__syncthreads_or(any)) continue;  // the electron has no element (uniform)
    const int s = i < cs.nup ? 0 : 1, n = s == 0 ? cs.nup : cs.ndn, ish = s == 0 ? 0 : cs.nup;
    const int ivirt = cs.md_ivirt[s], iactv = cs.md_iactv[s];
    const double *sl = st.slmi + ((size_t)w * 2 + s) * nmax * nmax + (size_t)n * (i - ish);
    const double *Y = md.ymat + ((size_t)w * 2 + s) * nmax * O;
    const double *aa = md.aa + ((size_t)w * 2 + s) * nmax * O;
    const int *slot = g.slot_orb + s * nmax;
    for (int v = threadIdx.x; v < O; v += blockDim.x) {
      double y = 0;
      if (v >= ivirt)
        for (int irep = iactv; irep < n; irep++) y += Y[(size_t)irep * O + v] * sl[irep];
      Yc[v] = y;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      double a = 0;
      for (int v = ivirt; v < O; v++) a += aa[(size_t)j * O + v] * Yc[v];
      zo[j] = a;
    }
    __syncthreads();
    for (int v = threadIdx.x; v < O; v += blockDim.x) {
      double z = v >= ivirt ? Yc[v] : 0.0;
      for (int j = 0; j < n; j++)
        if (slot[j] == v) z -= zo[j];
      Z[v] = z;
    }
    __syncthreads();
    for (int m = threadIdx.x; m < K; m += blockDim.x) {
      double b = 0;
      for (int v = 0; v < O; v++) b += g.coefT[(size_t)m * O + v] * Z[v];
      Zb[m] = b;
    }
    __syncthreads();
    // the electron's quadrature points, warp per point
    for (int u = wid; u < NQ * M; u += nw) {
      const double trj = trow[u];
      if (trj == 0.0) continue;
      const int q = u / M, ic = u - q * M;
      const double ri_v[3] = {sx[i] - cs.cent[3 * ic], sx[N + i] - cs.cent[3 * ic + 1], sx[2 * N + i] - cs.cent[3 * ic + 2]};
      const double rin = sqrt(ri_v[0] * ri_v[0] + ri_v[1] * ri_v[1] + ri_v[2] * ri_v[2]);
      const double xp[3] = {rin * xqw[q] + cs.cent[3 * ic], rin * xqw[NQ + q] + cs.cent[3 * ic + 1],
                            rin * xqw[2 * NQ + q] + cs.cent[3 * ic + 2]};
      warp_basis_prepass<0>(cs, g, xp, rec, lane);
      __syncwarp();
      double d = 0;
      for (int m = lane; m < K; m += 32) warp_basis_ao<0>(cs, g, rec, m, [&](int, int, double v) { d += v * Zb[m]; });
      d = warp_sum(d);
      if (lane == 0) hb.tvpsp[(((size_t)w * N + i) * NQ + q) * M + ic] += detratio * trj * d;
      __syncwarp();
    }
    __syncthreads();
  }
}

}  // namespace cw
