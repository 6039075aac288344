// move.cuh — single-electron accelerated-Metropolis move, batched over walkers.
//
// One move of electron `iel` for all walkers is six launches:
//   k_propose       metrop6 proposal (vmc/metrop_mov1_slat.f90:131-361)
//   k_jastrow_move  jastrow4e iflag=0 (vmc/jastrow4e.f90:3)
//   k_basis_move    basis_fns for the moved electron (vmc/basis_fns.f90:8)
//   gemm            LCAO contraction (vmc/orbitals_no_qmckl.f90:195)
//   k_decide        ratio + drift at the new point, reverse transition
//                   probability, accept/reject (thread per walker)
//   k_commit        on accept: determinante/detsav (Sherman–Morrison) and
//                   jassav (CTA per walker)
#pragma once
#include "common.cuh"

namespace cw {

__device__ __forceinline__ double thetamx_d(const CSys &cs, double r, double z) {
  return cs.deltat + (2.0 - cs.deltat) / (1.0 + (z * r) * (z * r));
}

// gammai (vmc/gammai.f90:3)
__device__ double gammai_d(double a, double x, double xae, int &iflag) {
  if (x < a + 4) {
    iflag = 1;
    double ap = a, sum = 1 / a, del = sum;
    int iter = (int)(21 + 3 * (x - a));
    for (int n = 1; n <= iter; n++) {
      ap = ap + 1;
      del = del * x / ap;
      sum = sum + del;
    }
    return sum * xae;
  }
  iflag = -1;
  double a0 = 1, a1 = x, b0 = 0, b1 = 1, fac = 1, g = 0;
  int iter = max(20 + (int)llround(a - x), 7);
  for (int n = 1; n <= iter; n++) {
    double an = (double)n, ana = an - a;
    a0 = (a1 + a0 * ana) * fac;
    b0 = (b1 + b0 * ana) * fac;
    double anf = an * fac;
    a1 = x * a0 + anf * a1;
    b1 = x * b0 + anf * b1;
    fac = 1 / a1;
    g = b1 * fac;
  }
  return -(g * xae);
}

// Integral of the Slater-form radial transition density (metrop6 :246-280 / :480-512)
__device__ double t_area_d(double zeta, double co, double rbot, double rtop, double bot) {
  const double d5b2 = 2.5, d2b3 = .666666666666667, g5b2 = 1.329340388179137;
  double rzero = -1.0 / co;
  double zrbot = zeta * rbot, zrtop = zeta * rtop;
  double zebot = sqrt(zrbot * zrbot * zrbot) * exp(-zrbot);
  double zetop = sqrt(zrtop * zrtop * zrtop) * exp(-zrtop);
  int iflagb, iflagt, iflagz;
  double g52bot = gammai_d(d5b2, zrbot, zrbot * zebot, iflagb);
  double g52top = gammai_d(d5b2, zrtop, zrtop * zetop, iflagt);
  if (rzero < rbot || rzero > rtop) {
    double g52dif = (iflagb * iflagt == 1) ? g52top - g52bot : g52top - g52bot + g5b2;
    double g32dif = d2b3 * (g52dif + zetop - zebot);
    return fabs(g32dif + co * g52dif / zeta) / (bot * sqrt(zeta * zeta * zeta));
  }
  double zrzer = zeta * rzero;
  double zezer = sqrt(zrzer * zrzer * zrzer) * exp(-zrzer);
  double g52zer = gammai_d(d5b2, zrzer, zrzer * zezer, iflagz);
  double g52dif1 = (iflagb * iflagz == 1) ? g52zer - g52bot : g52zer - g52bot + g5b2;
  double g32dif1 = d2b3 * (g52dif1 + zezer - zebot);
  double g52dif2 = (iflagt * iflagz == 1) ? g52top - g52zer : g52top - g52zer + g5b2;
  double g32dif2 = d2b3 * (g52dif2 + zetop - zezer);
  return (fabs(g32dif1 + co * g52dif1 / zeta) + fabs(g32dif2 + co * g52dif2 / zeta)) /
         (bot * sqrt(zeta * zeta * zeta));
}

// One candidate of metrop6's radial rejection loop (vmc/metrop_mov1_slat.f90:236-240):
// rtry from the first draw, accepted when top/fmax exceeds the second.
__device__ __forceinline__ bool radial_candidate(DRng &r, double rmin, double deltar, double deltri, double co,
                                                 double zeta, double fmx, double &rtry, double &top) {
  rtry = ((deltar - deltri) * r.uniform() + deltri) * rmin;
  top = sqrt(rtry) * fabs(1.0 + co * rtry) * exp(-zeta * rtry);
  const double ratio = top / fmx;
  return ratio > r.uniform();
}

// Lanes per walker in the proposal and decision kernels: the serial geometry
// is evaluated identically by the G lanes of a walker's group, the dot
// products and the radial candidates are spread over them.
constexpr int kMoveGroup = 8;

// group-wide sum over the kMoveGroup lanes of a walker (only the group's
// lanes take part: other groups of the warp may have left)
__device__ __forceinline__ double group_sum(double v) {
  const unsigned gm = ((1u << kMoveGroup) - 1) << ((threadIdx.x & 31) & ~(kMoveGroup - 1));
#pragma unroll
  for (int o = kMoveGroup / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gm, v, o, kMoveGroup);
  return v;
}

// The radial rejection loop with the reference's draw order, for the walker
// of each group of kMoveGroup lanes: every lane of the group holds the
// walker's stream; in each round lane g of the group tests candidate g of the
// next kMoveGroup (its copy of the stream advanced by 2g draws).  The first
// accepted candidate and the stream state after it are those of the serial
// loop, and every lane of the group ends with them.  Every lane of the warp
// must call it (the rounds continue until every group of the warp is done).
// Returns true for a group that gave up (more than ~10^6 candidates).
__device__ __forceinline__ bool radial_sample_group(DRng &rng, double rmin, double deltar, double deltri, double co,
                                                 double zeta, double fmx, double &rtry, double &top) {
  const int lane = threadIdx.x & 31, g = lane & (kMoveGroup - 1), base = lane - g;
  bool done = false, gave_up = false;
  for (int rounds = 0; __any_sync(0xffffffffu, !done); rounds++) {
    DRng r = rng;
    for (int k = 0; k < 2 * g; k++) r.next();
    double rt, tp;
    const bool ok = !done && radial_candidate(r, rmin, deltar, deltri, co, zeta, fmx, rt, tp);
    const unsigned am = (__ballot_sync(0xffffffffu, ok) >> base) & ((1u << kMoveGroup) - 1);
    const int ks = base + (am ? __ffs(am) - 1 : kMoveGroup - 1);
    const uint64_t n0 = __shfl_sync(0xffffffffu, r.s0, ks), n1 = __shfl_sync(0xffffffffu, r.s1, ks);
    const uint64_t n2 = __shfl_sync(0xffffffffu, r.s2, ks), n3 = __shfl_sync(0xffffffffu, r.s3, ks);
    const double rtk = __shfl_sync(0xffffffffu, rt, ks), tpk = __shfl_sync(0xffffffffu, tp, ks);
    if (!done) {
      rng.s0 = n0; rng.s1 = n1; rng.s2 = n2; rng.s3 = n3;
      if (am) {
        rtry = rtk;
        top = tpk;
        done = true;
      } else if (rounds > (1 << 20) / kMoveGroup) {
        gave_up = true;
        done = true;
      }
    }
  }
  return gave_up;
}

__device__ __forceinline__ void spin_of(const CSys &cs, int iel, int &iab, int &nel, int &ish) {
  if (iel < cs.nup) { iab = 0; nel = cs.nup; ish = 0; }
  else { iab = 1; nel = cs.ndn; ish = cs.nup; }
}

// ---------------------------------------------------------------------------
// Proposal: kMoveGroup lanes per walker.  The drift at the old position
// (compute_determinante_grad iflag_move=1: slmi column . dorb + vj) is a dot
// product over the group; the accelerated-Metropolis geometry is a serial
// chain that the group's lanes evaluate identically; the radial rejection
// loop is cooperative within the group.  The group's lane 0 stores.
// ---------------------------------------------------------------------------
// The kernels of a move are written as bodies over a block index `bid`, so
// the same code runs one system per launch (bid = blockIdx.x) and, in
// ragged.cuh, many systems per launch (bid = the block's index within its
// system's share of the launch).
__device__ __forceinline__ void propose_body(const CSys &cs, const WState &st, const MoveBuf &mb, int iel,
                                             int *acc_count, const int bid) {
  // Every lane runs to the end (the radial sampling is cooperative across the
  // warp); groups past the population mirror the last walker and store nothing.
  // acc_count (optional): the accepted-walker count k_decide appends to,
  // emptied here (the previous move's commit has finished reading it).
  if (acc_count && bid == 0 && threadIdx.x == 0) *acc_count = 0;
  const int gl = threadIdx.x & (kMoveGroup - 1);
  const int wt = (bid * blockDim.x + threadIdx.x) / kMoveGroup;
  const bool live = wt < st.W;
  const int w = live ? wt : st.W - 1;
  const int lane = live ? gl : 1;  // lane 0 of a live group stores
  const int N = cs.N, nmax = cs.nmax;
  int iab, nel, ish;
  spin_of(cs, iel, iab, nel, ish);
  const int iloc = iel - ish;
  const double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax + (size_t)nel * iloc;
  const double *d0p = st.dorbs + (((size_t)w * 3 + 0) * N + iel) * nmax;
  const double *d1p = st.dorbs + (((size_t)w * 3 + 1) * N + iel) * nmax;
  const double *d2p = st.dorbs + (((size_t)w * 3 + 2) * N + iel) * nmax;
  double g0 = 0, g1 = 0, g2 = 0;
  for (int j = gl; j < nel; j += kMoveGroup) {
    const double s = sl[j];
    g0 += s * d0p[j];
    g1 += s * d1p[j];
    g2 += s * d2p[j];
  }
  g0 = group_sum(g0);
  g1 = group_sum(g1);
  g2 = group_sum(g2);

  const double zero = 0, one = 1, two = 2, four = 4, half = 0.5, d3b2 = 1.5, eps = 1.0e-10;
  const double deltar = cs.deltar, deltri = one / deltar, fbias = cs.fbias;
  const double *fjo = st.fjo + (size_t)w * 3 * N;
  const double m0 = mb.md_velo ? mb.md_velo[3 * w] : 0.0, m1 = mb.md_velo ? mb.md_velo[3 * w + 1] : 0.0,
               m2 = mb.md_velo ? mb.md_velo[3 * w + 2] : 0.0;
  double vo[3] = {m0 + g0 + fjo[0 * N + iel], m1 + g1 + fjo[1 * N + iel], m2 + g2 + fjo[2 * N + iel]};
  DRng rng;
  rng.load(st.rng + 4 * (size_t)w);
  MoveScratch m;
  double fxop = one;
  const int nearo = st.nearesto[(size_t)w * N + iel];
  const double znear = cs.znuc[cs.iwctype[nearo]];
  const double zcusp = (cs.nloc == 0) ? znear : zero;
  double rv[3];
  for (int k = 0; k < 3; k++) rv[k] = st.rvmino[((size_t)w * 3 + k) * N + iel];
  const double rmin = sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
  if (lane == 0) st.rmino[(size_t)w * N + iel] = rmin;
  double rbot = rmin * deltri, rtop = rmin * deltar;
  double voldr = zero;
  for (int ic = 0; ic < 3; ic++) voldr += vo[ic] * rv[ic];
  voldr = voldr / rmin;
  double voldp = zero, xaxis[3], yaxis[3], zaxis[3];
  for (int ic = 0; ic < 3; ic++) {
    zaxis[ic] = rv[ic] / rmin;
    xaxis[ic] = vo[ic] - voldr * zaxis[ic];
    voldp += xaxis[ic] * xaxis[ic];
  }
  voldp = sqrt(voldp);
  if (voldp < eps) {
    xaxis[0] = eps * (one - zaxis[0] * zaxis[0]);
    xaxis[1] = eps * (-zaxis[0] * zaxis[1]);
    xaxis[2] = eps * (-zaxis[0] * zaxis[2]);
    voldp = eps * sqrt(one - zaxis[0] * zaxis[0]);
  }
  for (int ic = 0; ic < 3; ic++) xaxis[ic] = xaxis[ic] / voldp;
  voldr = fmax(voldr, -2 * znear);
  yaxis[0] = zaxis[1] * xaxis[2] - zaxis[2] * xaxis[1];
  yaxis[1] = zaxis[2] * xaxis[0] - zaxis[0] * xaxis[2];
  yaxis[2] = zaxis[0] * xaxis[1] - zaxis[1] * xaxis[0];
  voldp = voldp * fbias;
  double root = (zcusp + voldr) * (zcusp + voldr - four / rmin), zeta;
  if (root >= zero) {
    root = sqrt(root);
    zeta = half * (zcusp - voldr - root);
    if (zeta <= zero) zeta = half * (zcusp - voldr + root);
    if (zeta <= zero) zeta = eps;
  } else {
    zeta = (voldr < zero) ? -voldr - eps : one;
  }
  double co = (zeta + voldr) / (one - (zeta + voldr) * rmin);
  root = sqrt((d3b2 * co - zeta) * (d3b2 * co - zeta) + two * zeta * co);
  double rmax1 = (d3b2 * co - zeta + root) / (two * zeta * co);
  if (rmax1 < rbot) rmax1 = rbot;
  if (rmax1 > rtop) rmax1 = rtop;
  double fmx = sqrt(rmax1) * fabs(one + co * rmax1) * exp(-zeta * rmax1);
  if (co < zero) {
    double rmax2 = (d3b2 * co - zeta - root) / (two * zeta * co);
    if (rmax2 < rbot) rmax2 = rbot;
    if (rmax2 > rtop) rmax2 = rtop;
    double fmax2 = sqrt(rmax2) * fabs(one + co * rmax2) * exp(-zeta * rmax2);
    fmx = fmx > fmax2 ? fmx : fmax2;
  }
  double bot = sqrt(rmin) * fabs(one + co * rmin) * exp(-zeta * rmin);
  double rtry, top;
  if (radial_sample_group(rng, rmin, deltar, deltri, co, zeta, fmx, rtry, top) && lane == 0) st.status[w] |= 4;
  fxop = fxop * top / bot;
  double areao = t_area_d(zeta, co, rbot, rtop, bot);
  double raver = half * (rmin + rtry);
  double deltt = thetamx_d(cs, raver, znear);
  double costht = one - deltt * rng.uniform();
  double zprime = rtry * costht;
  double sintht = sqrt(one - costht * costht);
  areao = areao * deltt;
  double term = fmin(voldp * raver * sintht, one);
  fmx = one + term;
  double phitry;
  const double PI = 3.141592653589793115997963468544185161590576171875;
  for (int guard = 0;; guard++) {
    phitry = PI * rng.uniform();
    double cosphi = cos(phitry);
    top = one + term * cosphi;
    if (top > rng.uniform() * fmx) break;
    if (guard > 1000000) {
      if (lane == 0) st.status[w] |= 4;
      break;
    }
  }
  fxop = fxop * top;
  double xprime = rtry * sintht * cos(phitry);
  double yprime = sqrt(fmax(zero, rtry * rtry - xprime * xprime - zprime * zprime));
  if (rng.uniform() < half) yprime = -yprime;
  const double *cn = &cs.cent[3 * nearo];
  double xn[3];
  for (int ic = 0; ic < 3; ic++) {
    const double d = xaxis[ic] * xprime + yaxis[ic] * yprime + zaxis[ic] * zprime;
    xn[ic] = d + cn[ic];
  }
  m.rminno = rtry;
  // geometrical rejection
  double rminn = 99.0e9;
  int nearn = 0;
  for (int j = 0; j < cs.M; j++) {
    double dist = zero;
    for (int ic = 0; ic < 3; ic++) dist += (xn[ic] - cs.cent[3 * j + ic]) * (xn[ic] - cs.cent[3 * j + ic]);
    if (dist < rminn) {
      rminn = dist;
      nearn = j;
    }
  }
  rminn = sqrt(rminn);
  double rminon = zero, dot = zero, rvminn[3], rvminon[3];
  for (int ic = 0; ic < 3; ic++) {
    rvminn[ic] = xn[ic] - cs.cent[3 * nearn + ic];
    rvminon[ic] = st.x[((size_t)w * 3 + ic) * N + iel] - cs.cent[3 * nearn + ic];
    rminon += rvminon[ic] * rvminon[ic];
    dot += rvminn[ic] * rvminon[ic];
  }
  rminon = sqrt(rminon);
  dot = dot / (rminn * rminon);
  const double ravern = half * (rminn + rminon);
  const double delttn = thetamx_d(cs, ravern, cs.znuc[cs.iwctype[nearn]]);
  m.igeo = (rminon > rminn * deltar || dot < one - delttn) ? 1 : 0;
  for (int k = 0; k < 3; k++) {
    m.xnew[k] = xn[k];
    m.rvminn[k] = rvminn[k];
    m.rvminon[k] = rvminon[k];
  }
  m.rminn = rminn;
  m.rminon = rminon;
  m.delttn = delttn;
  m.fxop = fxop;
  m.areao = areao;
  m.rratio = m.rminno / rminon;
  m.nearestn = nearn;
  m.tel = iel;
  if (lane != 0) return;
  mb.ms[w] = m;
  rng.store(st.rng + 4 * (size_t)w);
}
__global__ void __launch_bounds__(128) k_propose(const __grid_constant__ CSys cs, WState st, MoveBuf mb, int iel,
                                                 int *acc_count) {
  propose_body(cs, st, mb, iel, acc_count, blockIdx.x);
}

// ---------------------------------------------------------------------------
// jastrow4e, iflag=0: warp per walker, lanes over the partner electron.
// Per-centre quantities of the moved electron are staged in shared memory.
// ---------------------------------------------------------------------------
// partner electrons per lane in k_jastrow_move: 2 shares each coefficient load
// between two partners but needs ~150 registers; bounded to four blocks per
// SM it spills and measured 39.3 against 39.9 ms per 8192-walker sweep of the
// 120-electron molecule (bitwise the same walk), so one is kept
constexpr int kJmPartners = 1;

template <int NORD>
__device__ __forceinline__ void jastrow_move_body(const CSys &cs, const WState &st, const MoveBuf &mb, int iel,
                                                  const int bid) {
  extern __shared__ __align__(16) double smem[];
  constexpr int NB = een_nb(NORD);        // folded coefficients per centre
  constexpr int PER = 8 + 2 * NB;         // shared doubles per centre (one pad keeps B 16-byte aligned)
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int w = (bid * blockDim.x + threadIdx.x) >> 5;
  const int M = cs.M, N = cs.N;
  double *sh = smem + (size_t)wib * M * PER;
  // per centre ic: rvec(3), r, scaled r, dd1, -kappa dd1 / r, then B[NB], dB[NB]
  double *sh_rv = sh, *sh_r = sh + 3 * M, *sh_s = sh + 4 * M, *sh_d = sh + 5 * M, *sh_g = sh + 6 * M, *sh_B = sh + 8 * M;
  const bool active = (w < st.W);
  int igeo = 1;
  double xi[3] = {0, 0, 0};
  if (active) {
    const MoveScratch &m = mb.ms[w];
    igeo = m.igeo;
    xi[0] = m.xnew[0]; xi[1] = m.xnew[1]; xi[2] = m.xnew[2];
  }
  if (!active || igeo) return;  // whole warp leaves together (same walker)
  if (iel < 0) iel = mb.ms[w].tel;
  const double kap = cs.scalek;
  for (int ic = lane; ic < M; ic += 32) {
    double r2 = 0;
    for (int k = 0; k < 3; k++) {
      const double d = xi[k] - cs.cent[3 * ic + k];
      sh_rv[k * M + ic] = d;
      r2 += d * d;
    }
    const double r = sqrt(r2);
    sh_r[ic] = r;
    double rr, dd1, dd2;
    scale2<double>(cs, r, rr, dd1, dd2);
    sh_s[ic] = rr;
    sh_d[ic] = dd1;
    sh_g[ic] = -kap * dd1 / r;
    mb.enn[((size_t)w * 2 + 0) * M + ic] = rr;
    mb.enn[((size_t)w * 2 + 1) * M + ic] = dd1 / r;
    if (NORD > 1) een_fold<NORD, double>(&cs.c[cs.iwctype[ic] * CW_MAX_TERMS], 1 - kap * rr, sh_B + (size_t)ic * 2 * NB);
  }
  __syncwarp();
  const double *xw = st.x + (size_t)w * 3 * N;
  const double *fso_i = st.fso + ((size_t)w * N + iel) * N;
  const double asym = cs.asymp_r;
  double dfs = 0, dv0 = 0, dv1 = 0, dv2 = 0;
  // each lane takes kJmPartners partners (jj, jj + 32, ...) so that every
  // shared coefficient load serves all of them
  constexpr int P = kJmPartners;
  for (int j0 = lane; j0 < N; j0 += 32 * P) {
    bool ok[P];
    int jj[P];
    double rvee[P][3], rij[P], z[P], du_r[P], fs[P], gi[P][3], gj[P][3];
#pragma unroll
    for (int q = 0; q < P; q++) {
      jj[q] = j0 + 32 * q;
      ok[q] = jj[q] < N && jj[q] != iel;
      // a partner slot past the end or on the moved electron computes on a
      // valid neighbour index and is discarded
      const int jc = ok[q] ? jj[q] : (iel == 0 ? N - 1 : 0);
      const double xj[3] = {xw[jc], xw[N + jc], xw[2 * N + jc]};
      const int i = jc < iel ? iel : jc, j = jc < iel ? jc : iel;
      int isb, ipar;
      double sspinn;
      pair_spin(cs, i, j, isb, ipar, sspinn);
      for (int k = 0; k < 3; k++) rvee[q][k] = xi[k] - xj[k];  // x_iel - x_jj
      rij[q] = sqrt(rvee[q][0] * rvee[q][0] + rvee[q][1] * rvee[q][1] + rvee[q][2] * rvee[q][2]);
      double u, dd1, dd2;
      scale2<double>(cs, rij[q], u, dd1, dd2);
      fs[q] = 0;
      for (int k = 0; k < 3; k++) gi[q][k] = gj[q][k] = 0;
      if (u != asym) {
        double fee, feeu, feeuu;
        ee_term<1, double>(cs, isb, ipar, sspinn, u, fee, feeu, feeuu);
        feeu = feeu * dd1 / rij[q];
        fs[q] += fee;
        for (int k = 0; k < 3; k++) {
          gi[q][k] += feeu * rvee[q][k];
          gj[q][k] -= feeu * rvee[q][k];
        }
      }
      z[q] = 1 - kap * u;
      du_r[q] = -kap * dd1 / rij[q];
    }
    if (NORD > 1) {
      // partners' e-n values from the walker's table (coalesced over lanes),
      // loaded two centres ahead (the table comes from DRAM)
      const double *en_rr = st.enm + (size_t)w * 2 * M * N;
      const double *en_h = en_rr + (size_t)M * N;
      int jt[P];
      double nrr[P], nh[P], nrr2[P], nh2[P];
#pragma unroll
      for (int q = 0; q < P; q++) {
        jt[q] = ok[q] ? jj[q] : (iel == 0 ? N - 1 : 0);
        nrr[q] = en_rr[jt[q]];
        nh[q] = en_h[jt[q]];
        nrr2[q] = M > 1 ? en_rr[N + jt[q]] : 0.0;
        nh2[q] = M > 1 ? en_h[N + jt[q]] : 0.0;
      }
      for (int ic = 0; ic < M; ic++) {
        double rrj[P], hj[P], y[P];
        bool any = false;
        const double rri = sh_s[ic];
#pragma unroll
        for (int q = 0; q < P; q++) {
          rrj[q] = nrr[q];
          hj[q] = nh[q];
          nrr[q] = nrr2[q];
          nh[q] = nh2[q];
          if (ic + 2 < M) {
            nrr2[q] = en_rr[(ic + 2) * N + jt[q]];
            nh2[q] = en_h[(ic + 2) * N + jt[q]];
          }
          any |= ok[q] && !(rri == asym && rrj[q] == asym);
          y[q] = 1 - kap * rrj[q];
        }
        if (!any) continue;
        double fc[P], fu_[P], fi_[P], fj_[P];
        een_apply1_multi<NORD, P>(sh_B + (size_t)ic * 2 * NB, y, z, fc, fu_, fi_, fj_);
        const double gic = sh_g[ic];
        const double rv[3] = {sh_rv[ic], sh_rv[M + ic], sh_rv[2 * M + ic]};
#pragma unroll
        for (int q = 0; q < P; q++) {
          if (rri == asym && rrj[q] == asym) continue;  // this pair-centre term is cut
          // partner to centre: (x_iel - c) - (x_iel - x_jj)
          const double rj_v[3] = {rv[0] - rvee[q][0], rv[1] - rvee[q][1], rv[2] - rvee[q][2]};
          const double fu = fu_[q] * du_r[q];
          const double fi = fi_[q] * gic;
          const double fj = fj_[q] * (-kap) * hj[q];
          fs[q] += fc[q];
          for (int k = 0; k < 3; k++) {
            gi[q][k] += fi * rv[k] + fu * rvee[q][k];
            gj[q][k] += fj * rj_v[k] - fu * rvee[q][k];
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < P; q++) {
      if (!ok[q]) continue;
      const int jq = jj[q];
      mb.fsn[(size_t)w * N + jq] = fs[q];
      for (int k = 0; k < 3; k++) {
        mb.fijn_i[((size_t)w * 3 + k) * N + jq] = gi[q][k];
        mb.fijn_j[((size_t)w * 3 + k) * N + jq] = gj[q][k];
      }
      dfs += fs[q] - fso_i[jq];
      dv0 += gi[q][0] - st.fijo[(((size_t)w * 3 + 0) * N + iel) * N + jq];
      dv1 += gi[q][1] - st.fijo[(((size_t)w * 3 + 1) * N + iel) * N + jq];
      dv2 += gi[q][2] - st.fijo[(((size_t)w * 3 + 2) * N + iel) * N + jq];
    }
  }
  // e-n part of the moved electron
  double fen_s = 0, ge0 = 0, ge1 = 0, ge2 = 0;
  for (int ic = lane; ic < M; ic += 32) {
    const int it = cs.iwctype[ic];
    const double rri = sh_s[ic];
    if (rri == cs.asymp_r) continue;
    const double ri = sh_r[ic];
    const double dd7 = sh_d[ic];
    double fen, feni, fenii;
    en_term<1, double>(cs, it, rri, fen, feni, fenii);
    feni = feni * dd7 / ri;
    fen_s += fen;
    ge0 += feni * sh_rv[0 * M + ic];
    ge1 += feni * sh_rv[1 * M + ic];
    ge2 += feni * sh_rv[2 * M + ic];
  }
  fen_s = warp_sum(fen_s);
  ge0 = warp_sum(ge0);
  ge1 = warp_sum(ge1);
  ge2 = warp_sum(ge2);
  dfs = warp_sum(dfs);
  dv0 = warp_sum(dv0);
  dv1 = warp_sum(dv1);
  dv2 = warp_sum(dv2);
  if (lane == 0) {
    mb.fsn[(size_t)w * N + iel] = fen_s;
    mb.fijn_i[((size_t)w * 3 + 0) * N + iel] = ge0;
    mb.fijn_i[((size_t)w * 3 + 1) * N + iel] = ge1;
    mb.fijn_i[((size_t)w * 3 + 2) * N + iel] = ge2;
    dfs += fen_s - fso_i[iel];
    dv0 += ge0 - st.fijo[(((size_t)w * 3 + 0) * N + iel) * N + iel];
    dv1 += ge1 - st.fijo[(((size_t)w * 3 + 1) * N + iel) * N + iel];
    dv2 += ge2 - st.fijo[(((size_t)w * 3 + 2) * N + iel) * N + iel];
    mb.fsumn[w] = st.fsumo[w] + dfs;
    const double *fjo = st.fjo + (size_t)w * 3 * N;
    mb.vjn[3 * w + 0] = fjo[0 * N + iel] + dv0;
    mb.vjn[3 * w + 1] = fjo[1 * N + iel] + dv1;
    mb.vjn[3 * w + 2] = fjo[2 * N + iel] + dv2;
  }
}
template <int NORD>
__global__ void __launch_bounds__(128, 5) k_jastrow_move(const __grid_constant__ CSys cs, WState st, MoveBuf mb, int iel) {
  jastrow_move_body<NORD>(cs, st, mb, iel, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Mixed-precision jastrow4e: the same warp-per-walker kernel with the pair
// and e-e-n polynomial sums in FP32 (folded coefficients, scaled distances,
// per-pair value and gradients); coordinates differ in FP64 before the cast,
// and the row sums against the stored FP64 tables (dfs, dv) stay FP64.
// ---------------------------------------------------------------------------
// partners per lane of k_jastrow_move_f32: four share each coefficient quad
// load (235 registers unbounded; bounded to three blocks per SM it spills a
// little and measured 29.0 against 30.9 ms per 8192-walker sweep for one
// partner, and 36.0 with two blocks per SM and no spills)
constexpr int kJmF32Partners = 4;

template <int NORD, int P>
__device__ __forceinline__ void jastrow_move_f32_body(const CSys &cs, const WState &st, const MoveBuf &mb, int iel,
                                                      const int bid) {
  extern __shared__ __align__(16) float smemf[];
  constexpr int NB = een_nbp(NORD);        // padded (B, dB) pairs per centre
  constexpr int PER = 8 + 2 * NB;         // shared floats per centre (B 16-byte aligned)
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int w = (bid * blockDim.x + threadIdx.x) >> 5;
  const int M = cs.M, N = cs.N;
  float *sh = smemf + (size_t)wib * M * PER;
  float *sh_rv = sh, *sh_r = sh + 3 * M, *sh_s = sh + 4 * M, *sh_d = sh + 5 * M, *sh_g = sh + 6 * M, *sh_B = sh + 8 * M;
  const bool active = (w < st.W);
  int igeo = 1;
  double xi[3] = {0, 0, 0};
  if (active) {
    const MoveScratch &m = mb.ms[w];
    igeo = m.igeo;
    xi[0] = m.xnew[0]; xi[1] = m.xnew[1]; xi[2] = m.xnew[2];
  }
  if (!active || igeo) return;
  if (iel < 0) iel = mb.ms[w].tel;
  const float kap = (float)cs.scalek;
  const float asym = (float)cs.asymp_r;
  for (int ic = lane; ic < M; ic += 32) {
    float r2 = 0;
    for (int k = 0; k < 3; k++) {
      const float d = (float)(xi[k] - cs.cent[3 * ic + k]);
      sh_rv[k * M + ic] = d;
      r2 += d * d;
    }
    const float r = sqrtf(r2);
    sh_r[ic] = r;
    float rr, dd1, dd2;
    scale2<float>(cs, r, rr, dd1, dd2);
    sh_s[ic] = rr;
    sh_d[ic] = dd1;
    sh_g[ic] = -kap * dd1 / r;
    mb.enn[((size_t)w * 2 + 0) * M + ic] = rr;
    mb.enn[((size_t)w * 2 + 1) * M + ic] = dd1 / r;
    if (NORD > 1) een_fold<NORD, float, true>(&cs.cf[cs.iwctype[ic] * CW_MAX_TERMS], 1 - kap * rr, sh_B + (size_t)ic * 2 * NB);
  }
  __syncwarp();
  const double *xw = st.x + (size_t)w * 3 * N;
  const double *fso_i = st.fso + ((size_t)w * N + iel) * N;
  double dfs = 0, dv0 = 0, dv1 = 0, dv2 = 0;
  // each lane takes P partners (jj, jj + 32, ...): every coefficient quad
  // loaded from shared memory serves all of them
  for (int j0 = lane; j0 < N; j0 += 32 * P) {
    bool ok[P];
    int jj[P];
    double xj[P][3];
    float rvee[P][3], rij[P], z[P], du_r[P], fs[P], gi[P][3], gj[P][3];
#pragma unroll
    for (int q = 0; q < P; q++) {
      jj[q] = j0 + 32 * q;
      ok[q] = jj[q] < N && jj[q] != iel;
      // a slot past the end or on the moved electron computes on a valid
      // neighbour and is discarded
      const int jc = ok[q] ? jj[q] : (iel == 0 ? N - 1 : 0);
      jj[q] = jc == jj[q] ? jj[q] : jc;
      xj[q][0] = xw[jc]; xj[q][1] = xw[N + jc]; xj[q][2] = xw[2 * N + jc];
      const int i = jc < iel ? iel : jc, j = jc < iel ? jc : iel;
      int isb, ipar;
      double sspinn_d;
      pair_spin(cs, i, j, isb, ipar, sspinn_d);
      const float sspinn = (float)sspinn_d;
      for (int k = 0; k < 3; k++) rvee[q][k] = (float)(xi[k] - xj[q][k]);
      rij[q] = sqrtf(rvee[q][0] * rvee[q][0] + rvee[q][1] * rvee[q][1] + rvee[q][2] * rvee[q][2]);
      float u, dd1, dd2;
      scale2<float>(cs, rij[q], u, dd1, dd2);
      fs[q] = 0;
      for (int k = 0; k < 3; k++) gi[q][k] = gj[q][k] = 0;
      if (u != asym) {
        float fee, feeu, feeuu;
        ee_term<1, float>(cs, isb, ipar, sspinn, u, fee, feeu, feeuu);
        feeu = feeu * dd1 / rij[q];
        fs[q] += fee;
        for (int k = 0; k < 3; k++) {
          gi[q][k] += feeu * rvee[q][k];
          gj[q][k] -= feeu * rvee[q][k];
        }
      }
      z[q] = 1 - kap * u;
      du_r[q] = (-kap * dd1) / rij[q];
    }
    if (NORD > 1) {
      // partners' table values two centres ahead
      const float *en_rr = st.enmf + (size_t)w * 2 * M * N;
      const float *en_h = en_rr + (size_t)M * N;
      float nrr[P], nh[P], nrr2[P], nh2[P];
#pragma unroll
      for (int q = 0; q < P; q++) {
        nrr[q] = en_rr[jj[q]];
        nh[q] = en_h[jj[q]];
        nrr2[q] = M > 1 ? en_rr[N + jj[q]] : 0.0f;
        nh2[q] = M > 1 ? en_h[N + jj[q]] : 0.0f;
      }
      for (int ic = 0; ic < M; ic++) {
        float rrj[P], hj[P], y[P];
        bool any = false;
        const float rri = sh_s[ic];
#pragma unroll
        for (int q = 0; q < P; q++) {
          rrj[q] = nrr[q];
          hj[q] = nh[q];
          nrr[q] = nrr2[q];
          nh[q] = nh2[q];
          if (ic + 2 < M) {
            nrr2[q] = en_rr[(size_t)(ic + 2) * N + jj[q]];
            nh2[q] = en_h[(size_t)(ic + 2) * N + jj[q]];
          }
          any |= ok[q] && !(rri == asym && rrj[q] == asym);
          y[q] = 1 - kap * rrj[q];
        }
        if (!any) continue;
        float fc[P], fu_[P], fi_[P], fj_[P];
        een_apply1f_multi<NORD, P>(sh_B + (size_t)ic * 2 * NB, y, z, fc, fu_, fi_, fj_);
        const float gic = sh_g[ic];
        const float rv[3] = {sh_rv[ic], sh_rv[M + ic], sh_rv[2 * M + ic]};
#pragma unroll
        for (int q = 0; q < P; q++) {
          if (rri == asym && rrj[q] == asym) continue;  // this pair-centre term is cut
          // partner-to-centre vector x_j - c = (x_i - c) - (x_i - x_j), from the
          // FP32 vectors already held (no FP64 difference and conversion per term)
          const float rj_v[3] = {rv[0] - rvee[q][0], rv[1] - rvee[q][1], rv[2] - rvee[q][2]};
          const float fu = fu_[q] * du_r[q];
          const float fi = fi_[q] * gic;
          const float fj = fj_[q] * (-kap) * hj[q];
          fs[q] += fc[q];
          for (int k = 0; k < 3; k++) {
            gi[q][k] += fi * rv[k] + fu * rvee[q][k];
            gj[q][k] += fj * rj_v[k] - fu * rvee[q][k];
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < P; q++) {
      if (!ok[q]) continue;
      const int jq = jj[q];
      mb.fsn[(size_t)w * N + jq] = fs[q];
      for (int k = 0; k < 3; k++) {
        mb.fijn_i[((size_t)w * 3 + k) * N + jq] = gi[q][k];
        mb.fijn_j[((size_t)w * 3 + k) * N + jq] = gj[q][k];
      }
      dfs += (double)fs[q] - fso_i[jq];
      dv0 += (double)gi[q][0] - st.fijo[(((size_t)w * 3 + 0) * N + iel) * N + jq];
      dv1 += (double)gi[q][1] - st.fijo[(((size_t)w * 3 + 1) * N + iel) * N + jq];
      dv2 += (double)gi[q][2] - st.fijo[(((size_t)w * 3 + 2) * N + iel) * N + jq];
    }
  }
  // e-n part of the moved electron
  float fen_s = 0, ge0 = 0, ge1 = 0, ge2 = 0;
  for (int ic = lane; ic < M; ic += 32) {
    const int it = cs.iwctype[ic];
    const float rri = sh_s[ic];
    if (rri == asym) continue;
    float fen, feni, fenii;
    en_term<1, float>(cs, it, rri, fen, feni, fenii);
    feni = feni * sh_d[ic] / sh_r[ic];
    fen_s += fen;
    ge0 += feni * sh_rv[0 * M + ic];
    ge1 += feni * sh_rv[1 * M + ic];
    ge2 += feni * sh_rv[2 * M + ic];
  }
  fen_s = warp_sumf(fen_s);
  ge0 = warp_sumf(ge0);
  ge1 = warp_sumf(ge1);
  ge2 = warp_sumf(ge2);
  dfs = warp_sum(dfs);
  dv0 = warp_sum(dv0);
  dv1 = warp_sum(dv1);
  dv2 = warp_sum(dv2);
  if (lane == 0) {
    mb.fsn[(size_t)w * N + iel] = fen_s;
    mb.fijn_i[((size_t)w * 3 + 0) * N + iel] = ge0;
    mb.fijn_i[((size_t)w * 3 + 1) * N + iel] = ge1;
    mb.fijn_i[((size_t)w * 3 + 2) * N + iel] = ge2;
    dfs += (double)fen_s - fso_i[iel];
    dv0 += (double)ge0 - st.fijo[(((size_t)w * 3 + 0) * N + iel) * N + iel];
    dv1 += (double)ge1 - st.fijo[(((size_t)w * 3 + 1) * N + iel) * N + iel];
    dv2 += (double)ge2 - st.fijo[(((size_t)w * 3 + 2) * N + iel) * N + iel];
    mb.fsumn[w] = st.fsumo[w] + dfs;
    const double *fjo = st.fjo + (size_t)w * 3 * N;
    mb.vjn[3 * w + 0] = fjo[0 * N + iel] + dv0;
    mb.vjn[3 * w + 1] = fjo[1 * N + iel] + dv1;
    mb.vjn[3 * w + 2] = fjo[2 * N + iel] + dv2;
  }
}
template <int NORD, int P>
__global__ void __launch_bounds__(128, P == 1 ? 8 : (P == 2 ? 4 : 3)) k_jastrow_move_f32(const __grid_constant__ CSys cs, WState st, MoveBuf mb, int iel) {
  jastrow_move_f32_body<NORD, P>(cs, st, mb, iel, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Basis functions of the moved electron (basis_fns ider=1): warp per walker,
// per-centre prepass then lanes over AOs.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void basis_move_body(const CSys &cs, const WState &st, const MoveBuf &mb, const GSys &g,
                                                const int bid) {
  extern __shared__ __align__(16) double smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int w = (bid * blockDim.x + threadIdx.x) >> 5;
  if (w >= st.W) return;
  const int K = cs.K;
  const MoveScratch &mv = mb.ms[w];
  double *phi = mb.phi + (size_t)w * 4 * K;
  const int kp = mb.kp;
  float *hi = mb.phi_hi ? mb.phi_hi + (size_t)w * 4 * kp : nullptr;
  float *lo = mb.phi_lo ? mb.phi_lo + (size_t)w * 4 * kp : nullptr;
  if (mv.igeo) {
    // the GEMM still reads these rows: keep them finite
    if (hi) {
      for (int t = lane; t < 4 * K; t += 32) {
        hi[(size_t)(t / K) * kp + t % K] = 0.0f;
        lo[(size_t)(t / K) * kp + t % K] = 0.0f;
      }
    } else {
      for (int t = lane; t < 4 * K; t += 32) phi[t] = 0.0;
    }
    return;
  }
  double *rec = smem + (size_t)wib * cs.M * kCenRec;
  const double x[3] = {mv.xnew[0], mv.xnew[1], mv.xnew[2]};
  warp_basis_prepass<1>(cs, g, x, rec, lane);
  __syncwarp();
  if (hi) {
    for (int m = lane; m < K; m += 32)
      warp_basis_ao<1>(cs, g, rec, m, [&](int a, int d, double v) {
        float h, l;
        split_tf32(v, h, l);
        hi[(size_t)d * kp + a] = h;
        lo[(size_t)d * kp + a] = l;
      });
    return;
  }
  for (int m = lane; m < K; m += 32)
    warp_basis_ao<1>(cs, g, rec, m, [&](int a, int d, double v) { phi[(size_t)d * K + a] = v; });
}
__global__ void k_basis_move(const __grid_constant__ CSys cs, WState st, MoveBuf mb, GSys g) {
  basis_move_body(cs, st, mb, g, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Accept / reject: thread per walker.  Ratio and drift at the new point
// (determinante :40-46 + compute_determinante_grad iflag_move=0), the
// reverse transition probability (metrop6 :435-560) and the accept draw.
// Scalar state of accepted moves is committed here; k_commit applies the
// matrix and table updates.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void decide_body(const CSys &cs, const WState &st, const MoveBuf &mb, const GSys &g,
                                            int iel, int *acc_list, int *acc_count, const int bid) {
  // kMoveGroup lanes per walker: the ratio and the drift at the new point are
  // dot products over the group, the rest is evaluated identically by the
  // group's lanes, its lane 0 stores
  const int lane = threadIdx.x & (kMoveGroup - 1);
  const int w = (bid * blockDim.x + threadIdx.x) / kMoveGroup;
  if (w >= st.W) return;  // the whole group (one walker)
  const int N = cs.N, nmax = cs.nmax, Oa = cs.Oa;
  int iab, nel, ish;
  spin_of(cs, iel, iab, nel, ish);
  const int iloc = iel - ish;
  MoveScratch &m = mb.ms[w];
  const double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax + (size_t)nel * iloc;
  const double *orbn = mb.orbn + (size_t)w * 4 * Oa;
  const int *slot = g.slot_orb + iab * nmax;
  const double zero = 0, one = 1, two = 2, four = 4, half = 0.5, eps = 1.0e-10;
  DRng rng;
  rng.load(st.rng + 4 * (size_t)w);
  double p = zero, psidn = 0, psi2n = 0, ratio = 0;
  const double fsumn = mb.fsumn[w];
  if (!m.igeo) {
    for (int j = lane; j < nel; j += kMoveGroup) ratio += sl[j] * orbn[slot[j]];
    ratio = group_sum(ratio);
    const double detn = st.detiab[2 * w + iab] * ratio;
    psidn = mb.md_psidn ? mb.md_psidn[w] : detn * st.detiab[2 * w + (1 - iab)] * cs.cdet;
    if (detn != 0.0) {
      double v0 = 0, v1 = 0, v2 = 0;
      for (int j = lane; j < nel; j += kMoveGroup) {
        const double sc = sl[j] / ratio;
        v0 += sc * orbn[1 * Oa + slot[j]];
        v1 += sc * orbn[2 * Oa + slot[j]];
        v2 += sc * orbn[3 * Oa + slot[j]];
      }
      v0 = group_sum(v0);
      v1 = group_sum(v1);
      v2 = group_sum(v2);
      const double *mv = mb.md_veln ? mb.md_veln + 3 * w : nullptr;
      const double vn[3] = {(mv ? mv[0] : 0.0) + v0 + mb.vjn[3 * w + 0], (mv ? mv[1] : 0.0) + v1 + mb.vjn[3 * w + 1],
                            (mv ? mv[2] : 0.0) + v2 + mb.vjn[3 * w + 2]};
      psi2n = log(fabs(mb.md_psi2g ? mb.md_psi2g[w] : 1.0)) + 2 * (log(fabs(psidn)) + fsumn);
      const double deltar = cs.deltar, deltri = one / deltar;
      const double rminn = m.rminn, rminon = m.rminon;
      const double rbot = rminn * deltri, rtop = rminn * deltar;
      double vnewr = zero;
      for (int ic = 0; ic < 3; ic++) vnewr += vn[ic] * m.rvminn[ic];
      vnewr = vnewr / rminn;
      double vnewp = zero, xaxis[3];
      for (int ic = 0; ic < 3; ic++) {
        xaxis[ic] = vn[ic] - vnewr * m.rvminn[ic] / rminn;
        vnewp += xaxis[ic] * xaxis[ic];
      }
      vnewp = sqrt(vnewp);
      if (vnewp < eps) {
        xaxis[0] = eps * (one - m.rvminn[0] * m.rvminn[0]);
        xaxis[1] = eps * (-m.rvminn[0] * m.rvminn[1]);
        xaxis[2] = eps * (-m.rvminn[0] * m.rvminn[2]);
        vnewp = eps * sqrt(one - m.rvminn[0] * m.rvminn[0] * (two - rminn * rminn));
      }
      for (int ic = 0; ic < 3; ic++) xaxis[ic] = xaxis[ic] / vnewp;
      const double zn = cs.znuc[cs.iwctype[m.nearestn]];
      const double zc = (cs.nloc == 0) ? zn : zero;
      vnewr = fmax(vnewr, -2 * zn);
      vnewp = vnewp * cs.fbias;
      double root = (zc + vnewr) * (zc + vnewr - four / rminn), zeta;
      if (root >= zero) {
        root = sqrt(root);
        zeta = half * (zc - vnewr - root);
        if (zeta <= zero) zeta = half * (zc - vnewr + root);
        if (zeta <= zero) zeta = eps;
      } else {
        zeta = (vnewr < zero) ? -vnewr - eps : one;
      }
      const double co = (zeta + vnewr) / (one - (zeta + vnewr) * rminn);
      const double bot = sqrt(rminn) * fabs(one + co * rminn) * exp(-zeta * rminn);
      const double top = sqrt(rminon) * fabs(one + co * rminon) * exp(-zeta * rminon);
      double fxnp = one * top / bot;
      double arean = t_area_d(zeta, co, rbot, rtop, bot);
      arean = arean * m.delttn;
      double dot = 0;
      for (int ic = 0; ic < 3; ic++) dot += m.rvminn[ic] * m.rvminon[ic];
      dot = dot / (rminn * rminon);
      const double costht = dot;
      const double sintht = sqrt(one - costht * costht);
      const double ravern = half * (rminn + rminon);
      const double term = fmin(vnewp * ravern * sintht, one);
      double cosphi = zero, rnorm = zero;
      for (int ic = 0; ic < 3; ic++) {
        const double term2 = m.rvminon[ic] / rminon - costht * m.rvminn[ic] / rminn;
        rnorm += term2 * term2;
        cosphi += term2 * xaxis[ic];
      }
      cosphi = cosphi / sqrt(rnorm);
      fxnp = fxnp * (one + term * cosphi);
      p = m.rratio * m.rratio * exp(psi2n - st.psi2o[w]) * fabs((fxnp * m.areao) / (m.fxop * arean));
      p = fmin(one, p);
    }
  }
  const int acc = (rng.uniform() < p) ? 1 : 0;
  if (lane != 0) return;
  rng.store(st.rng + 4 * (size_t)w);
  m.acc = acc;
  m.ratio = ratio;
  // accepted walkers listed for the commit (in arrival order: each walker's
  // commit touches its own state only, so the order does not matter)
  if (acc && acc_list) acc_list[atomicAdd(acc_count, 1)] = w;
  if (acc) {
    st.psi2o[w] = psi2n;
    st.psido[w] = psidn;
    st.psijo[w] = fsumn;
    st.fsumo[w] = fsumn;
    st.detiab[2 * w + iab] = st.detiab[2 * w + iab] * ratio;
    st.sums[(size_t)w * 8 + 4] += 1.0;
    st.rmino[(size_t)w * N + iel] = m.rminn;
    st.nearesto[(size_t)w * N + iel] = m.nearestn;
    for (int k = 0; k < 3; k++) {
      st.rvmino[((size_t)w * 3 + k) * N + iel] = m.rvminn[k];
      st.x[((size_t)w * 3 + k) * N + iel] = m.xnew[k];
    }
  }
}
__global__ void __launch_bounds__(128) k_decide(const __grid_constant__ CSys cs, WState st, MoveBuf mb, GSys g, int iel,
                                                int *acc_list, int *acc_count) {
  decide_body(cs, st, mb, g, iel, acc_list, acc_count, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Commit of an accepted move: detsav (Sherman–Morrison, determinante :47-62)
// and jassav.  CTA per walker; rejected walkers return at once.
// ---------------------------------------------------------------------------
// Orbital rows, e-n table row and the Jastrow pair tables of the moved
// electron (the part of detsav / jassav after the inverse).
__device__ __forceinline__ void commit_tables(const CSys &cs, WState &st, const MoveBuf &mb, const GSys &g, int w, int iel) {
  const int tid = threadIdx.x;
  const int N = cs.N, nmax = cs.nmax, Oa = cs.Oa;
  int iab, nel, ish;
  spin_of(cs, iel, iab, nel, ish);
  const double *orbn = mb.orbn + (size_t)w * 4 * Oa;
  const int *slot = g.slot_orb + iab * nmax;
  for (int j = tid; j < nel; j += blockDim.x) {
    const int sj = slot[j];
    st.orbs[((size_t)w * N + iel) * nmax + j] = orbn[sj];
    for (int k = 0; k < 3; k++)
      st.dorbs[(((size_t)w * 3 + k) * N + iel) * nmax + j] = orbn[(1 + k) * Oa + sj];
  }
  // e-n table row of the moved electron
  const int M = cs.M;
  for (int t = tid; t < 2 * M; t += blockDim.x) {
    const int pl = t / M, ic = t % M;
    const double v = mb.enn[((size_t)w * 2 + pl) * M + ic];
    st.enm[(((size_t)w * 2 + pl) * M + ic) * N + iel] = v;
    if (st.enmf) st.enmf[(((size_t)w * 2 + pl) * M + ic) * N + iel] = (float)v;
  }
  // jassav: pair tables and per-electron gradients
  double *fso = st.fso + (size_t)w * N * N;
  for (int jj = tid; jj < N; jj += blockDim.x) {
    const double fsn = mb.fsn[(size_t)w * N + jj];
    fso[(size_t)iel * N + jj] = fsn;
    fso[(size_t)jj * N + iel] = fsn;
    for (int k = 0; k < 3; k++) {
      double *fij = st.fijo + ((size_t)w * 3 + k) * N * N;
      const double gi = mb.fijn_i[((size_t)w * 3 + k) * N + jj];
      if (jj == iel) {
        fij[(size_t)iel * N + iel] = gi;
        st.fjo[((size_t)w * 3 + k) * N + iel] = mb.vjn[3 * w + k];
      } else {
        const double gj = mb.fijn_j[((size_t)w * 3 + k) * N + jj];
        const double old_ji = fij[(size_t)jj * N + iel];
        st.fjo[((size_t)w * 3 + k) * N + jj] = st.fjo[((size_t)w * 3 + k) * N + jj] + gj - old_ji;
        fij[(size_t)iel * N + jj] = gi;
        fij[(size_t)jj * N + iel] = gj;
      }
    }
  }
}

__global__ void k_commit(const __grid_constant__ CSys cs, WState st, MoveBuf mb, GSys g, int iel) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  if (!mb.ms[w].acc) return;
  if (iel < 0) iel = mb.ms[w].tel;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarp = blockDim.x >> 5;
  const int nmax = cs.nmax, Oa = cs.Oa;
  int iab, nel, ish;
  spin_of(cs, iel, iab, nel, ish);
  const int iloc = iel - ish;
  __shared__ double s_orb[256];
  __shared__ double s_col[256];
  const double ratio = mb.ms[w].ratio;
  double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax;
  const double *orbn = mb.orbn + (size_t)w * 4 * Oa;
  const int *slot = g.slot_orb + iab * nmax;
  for (int j = tid; j < nel; j += blockDim.x) {
    s_orb[j] = orbn[slot[j]];
    s_col[j] = sl[(size_t)nel * iloc + j];
  }
  __syncthreads();
  // rows k != iloc: slmi(:,k) -= slmi(:,iloc) * (slmi(:,k)·orb_new)/ratio
  for (int k = wid; k < nel; k += nwarp) {
    if (k == iloc) continue;
    double s = 0;
    for (int j = lane; j < nel; j += 32) s += sl[(size_t)nel * k + j] * s_orb[j];
    s = warp_sum(s) / ratio;
    for (int j = lane; j < nel; j += 32) sl[(size_t)nel * k + j] = sl[(size_t)nel * k + j] - s_col[j] * s;
  }
  for (int j = tid; j < nel; j += blockDim.x) sl[(size_t)nel * iloc + j] = s_col[j] / ratio;
  commit_tables(cs, st, mb, g, w, iel);
}

// The accepted walkers of a move, in walker order: list [W], *count.  One
// block: each thread counts a contiguous run of walkers, a block scan gives
// the runs' offsets.
__global__ void __launch_bounds__(1024) k_accept_list(const MoveScratch *__restrict__ ms, int W, int *list,
                                                      int *count) {
  __shared__ int scan[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int per = (W + nt - 1) / nt, w0 = t * per, w1 = min(W, w0 + per);
  int n = 0;
  for (int w = w0; w < w1; w++) n += ms[w].acc != 0;
  scan[t] = n;
  __syncthreads();
  for (int off = 1; off < nt; off <<= 1) {
    const int v = t >= off ? scan[t - off] : 0;
    __syncthreads();
    scan[t] += v;
    __syncthreads();
  }
  int pos = scan[t] - n;
  for (int w = w0; w < w1; w++)
    if (ms[w].acc) list[pos++] = w;
  if (t == nt - 1) *count = scan[t];
}

// The same commit with the spin's inverse staged in shared memory: the n x n
// block is copied with asynchronous 8-byte copies (cp.async, sm_80+), all in
// flight at once, and while they land the block writes the orbital rows and
// the Jastrow pair tables (independent of the inverse); then the row factors
// (slmi(:,k)·orb_new)/ratio come from shared memory and the updated block is
// written back row by row, coalesced.  Row stride nel+1 (odd) keeps the
// row-per-lane-pair reads free of bank conflicts.  Dynamic shared memory:
// nel*(nel+1) + 3*nel doubles.  Same arithmetic as k_commit.  The blocks loop
// over the list of accepted walkers, so no block is spent on a rejected move.
__device__ __forceinline__ void commit_tile_walker(const CSys &cs, WState &st, const MoveBuf &mb, const GSys &g, int w, int iel) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarp = blockDim.x >> 5;
  const int nmax = cs.nmax, Oa = cs.Oa;
  int iab, nel, ish;
  spin_of(cs, iel, iab, nel, ish);
  const int iloc = iel - ish, ld = nel + 1;
  extern __shared__ __align__(16) double sm[];
  double *s_inv = sm;                        // [nel][ld]
  double *s_orb = sm + (size_t)nel * ld;     // [nel]
  double *s_col = s_orb + nel;               // [nel]
  double *s_fac = s_col + nel;               // [nel]
  const double ratio = mb.ms[w].ratio;
  double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax;
  const double *orbn = mb.orbn + (size_t)w * 4 * Oa;
  const int *slot = g.slot_orb + iab * nmax;
  const unsigned s_base = (unsigned)__cvta_generic_to_shared(s_inv);
  for (int k = wid; k < nel; k += nwarp)
    for (int j = lane; j < nel; j += 32)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s_base + 8u * (unsigned)(k * ld + j)),
                   "l"(sl + (size_t)nel * k + j)
                   : "memory");
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int j = tid; j < nel; j += blockDim.x) s_orb[j] = orbn[slot[j]];
  commit_tables(cs, st, mb, g, w, iel);
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  for (int j = tid; j < nel; j += blockDim.x) s_col[j] = s_inv[iloc * ld + j];
  // two lanes per row, each summing alternate entries; the loop bound is the
  // same for every thread of the block, so whole warps meet the shuffle
  for (int base = 0; base < 2 * nel; base += blockDim.x) {
    const int k2 = base + tid, k = k2 >> 1, h = k2 & 1;
    const bool act = k2 < 2 * nel;
    double s = 0;
    if (act)
      for (int j = h; j < nel; j += 2) s += s_inv[k * ld + j] * s_orb[j];
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    if (act && h == 0) s_fac[k] = s / ratio;
  }
  __syncthreads();
  for (int k = wid; k < nel; k += nwarp) {
    const double f = s_fac[k];
    for (int j = lane; j < nel; j += 32)
      sl[(size_t)nel * k + j] = (k == iloc) ? s_col[j] / ratio : s_inv[k * ld + j] - s_col[j] * f;
  }
}

__global__ void k_commit_tile(const __grid_constant__ CSys cs, WState st, MoveBuf mb, GSys g, int iel_arg, const int *__restrict__ list,
                              const int *__restrict__ count) {
  const int nacc = *count;
  for (int q = blockIdx.x; q < nacc; q += gridDim.x) {
    commit_tile_walker(cs, st, mb, g, list[q], iel_arg < 0 ? mb.ms[list[q]].tel : iel_arg);
    __syncthreads();  // the next walker reuses the shared memory
  }
}

}  // namespace cw
