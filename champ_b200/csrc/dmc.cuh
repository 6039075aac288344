// dmc.cuh — diffusion Monte Carlo step of every walker: dmc_ps
// (dmc/dmc_ps_mov1.f90:4) for pseudopotential wave functions and dmc_ae
// (dmc/dmc_ae_mov1.f90:4) for all-electron ones, with the reweighting of
// dmc/branching.f90 (icut_e=0, icut_br=0, fratio-scaled energies; the
// dmc_eloc_cutoff branch of each).
//
//   k_dmc_propose   drift-diffusion proposal of electron iel (:293-318)
//   (k_jastrow_move, k_basis_move, LCAO GEMM and k_commit are shared with VMC)
//   k_dmc_decide    Green-function acceptance, node crossings, age boost
//                   (:340-435)
//   k_dmc_weights   drift of every electron after hpsi (:516), fratio,
//                   reweight, per-walker sums of the step (:520-673)
//   k_set_quad      the step's quadrature rotation, shared by the population
//   k_walker_copy   walker copies of splitj (dmc/splitj.f90), CTA per copy
#pragma once
#include "common.cuh"

namespace cw {

struct DmcBuf {
  double *vold;     // [cap][3][N] drift of every electron (vold_dmc)
  double *wt;       // [cap]
  double *fratio;   // [cap]
  int *iage;        // [cap]
  double *eprev;    // [cap] eold at the start of the step
  double *acc;      // [cap][DA_NA] per-walker sums of one step
  int *copy_src;    // [cap]
  int *copy_dst;    // [cap]
};

// per-walker sums of one step (reduced on the host in walker order)
enum {
  DA_DFUS2AC = 0, DA_DFUS2UN, DA_DFUS2O, DA_IACCEPT, DA_ACC, DA_TRY, DA_NACC, DA_NODECR,
  DA_WSUM1, DA_ESUM1, DA_PESUM, DA_TPBSUM, DA_TAUSUM, DA_TMOVE, DA_FNORMO, DA_NA = 16
};

struct DmcScalars {
  double tau, etrial, eest, ffi, fprod;
};

__device__ __forceinline__ double gauss_d(DRng &r) {
  // gauss (vmc/gauss.f90:3): one normal deviate, the cosine draw first
  const double twopi = 6.283185307179586231995926937088370323181152343750;
  const double g = cos(twopi * r.uniform());
  return g * sqrt(-2 * log(r.uniform()));
}

// drift of electron e: slmi row · dorbs + vj (compute_determinante_grad
// iflag_move=1)
__device__ __forceinline__ void drift_old(const CSys &cs, const WState &st, int w, int e, double v[3],
                                          const double *md_vel = nullptr) {
  const int N = cs.N, nmax = cs.nmax;
  const int iab = e < cs.nup ? 0 : 1, nel = iab == 0 ? cs.nup : cs.ndn, ish = iab == 0 ? 0 : cs.nup;
  const double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax + (size_t)nel * (e - ish);
  double g0 = 0, g1 = 0, g2 = 0;
  for (int j = 0; j < nel; j++) {
    const double s = sl[j];
    g0 += s * st.dorbs[(((size_t)w * 3 + 0) * N + e) * nmax + j];
    g1 += s * st.dorbs[(((size_t)w * 3 + 1) * N + e) * nmax + j];
    g2 += s * st.dorbs[(((size_t)w * 3 + 2) * N + e) * nmax + j];
  }
  const double *fjo = st.fjo + (size_t)w * 3 * N;
  v[0] = (md_vel ? md_vel[0] : 0.0) + g0 + fjo[e];
  v[1] = (md_vel ? md_vel[1] : 0.0) + g1 + fjo[N + e];
  v[2] = (md_vel ? md_vel[2] : 0.0) + g2 + fjo[2 * N + e];
}

// nearest centre of a point: first minimum of the squared distance
__device__ __forceinline__ int nearest_centre_d(const CSys &cs, const double x[3]) {
  double best = 1.0e100;
  int iw = 0;
  for (int ic = 0; ic < cs.M; ic++) {
    const double d0 = x[0] - cs.cent[3 * ic], d1 = x[1] - cs.cent[3 * ic + 1], d2 = x[2] - cs.cent[3 * ic + 2];
    const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
    if (r2 < best) {
      best = r2;
      iw = ic;
    }
  }
  return iw;
}

// All-electron moves (dmc_ae, dmc/dmc_ae_mov1.f90:227-303 forward,
// :396-474 reverse): the drifted point of an electron at x with drift v in
// the frame of its nearest nucleus (z along the electron, x along the
// angular part of the drift), with the nucleus-dependent adrift, and the
// probability qgaus of sampling the exponential around the nucleus instead
// of the Gaussian around the drifted point.
struct AeFrame {
  int ic;
  double zeta, qgaus, pgaus, xd[3];
};
__device__ __forceinline__ AeFrame ae_frame_d(const CSys &cs, const double x[3], const double v[3], double tau) {
  const double one = 1, two = 2, half = 0.5, eps = 1.0e-10, adrift0 = 0.1;
  AeFrame f;
  f.ic = nearest_centre_d(cs, x);
  const double c[3] = {cs.cent[3 * f.ic], cs.cent[3 * f.ic + 1], cs.cent[3 * f.ic + 2]};
  const double z = cs.znuc[cs.iwctype[f.ic]];
  double rv[3], rmin = 0, vr = 0, v2 = 0;
  for (int k = 0; k < 3; k++) {
    rv[k] = x[k] - c[k];
    rmin += rv[k] * rv[k];
    vr += v[k] * rv[k];
    v2 += v[k] * v[k];
  }
  rmin = sqrt(rmin);
  vr = vr / rmin;
  const double va = sqrt(v2);
  f.zeta = sqrt(one / tau + z * z);
  double zaxis[3], xaxis[3], vp = 0;
  for (int k = 0; k < 3; k++) {
    zaxis[k] = rv[k] / rmin;
    xaxis[k] = v[k] - vr * zaxis[k];
    vp += xaxis[k] * xaxis[k];
  }
  vp = sqrt(vp);
  if (vp < eps) {
    xaxis[0] = eps * (one - zaxis[0] * zaxis[0]);
    xaxis[1] = eps * (-zaxis[0] * zaxis[1]);
    xaxis[2] = eps * (-zaxis[0] * zaxis[2]);
    vp = eps * sqrt(one + eps - zaxis[0] * zaxis[0]);
  }
  for (int k = 0; k < 3; k++) xaxis[k] = xaxis[k] / vp;
  const double hafzr2 = (half * z * rmin) * (half * z * rmin);
  const double adrift = (half * (1 + eps + vr / va)) + adrift0 * hafzr2 / (1 + hafzr2);
  const double vavvt = (sqrt(one + two * adrift * v2 * tau) - one) / (adrift * v2);
  const double rtry = rmin + vavvt * vr;
  if (rtry > 0) {
    f.qgaus = half * erfc(rtry / sqrt(two * tau));
    const double xprime = vavvt * vp * rtry / (half * (rmin + rtry));
    for (int k = 0; k < 3; k++) f.xd[k] = c[k] + xaxis[k] * xprime + zaxis[k] * rtry;
  } else {
    f.qgaus = half * (one + erf(-rtry / sqrt(two * tau)));
    for (int k = 0; k < 3; k++) f.xd[k] = c[k];
  }
  f.pgaus = one - f.qgaus;
  return f;
}

// (sqrt(2 pi tau))^3 / pi of dmc_ae's exponential density (dmc_ae :148)
__device__ __forceinline__ double ae_term(double tau) {
  const double pi = 3.141592653589793115997963468544185161590576171875;
  const double r = sqrt(2.0 * pi * tau);
  return r * r * r / pi;
}

// thread per walker: drift + diffusion of electron iel (dmc_ps's Gaussian
// around the drifted point; dmc_ae's Gaussian / exponential mixture for an
// all-electron wave function)
__global__ void k_dmc_propose(const __grid_constant__ CSys cs, WState st, MoveBuf mb, DmcBuf db, DmcScalars sc, int iel,
                              int *acc_count) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  // acc_count (optional): the accepted-walker count k_dmc_decide appends to
  if (acc_count && w == 0) *acc_count = 0;
  if (w >= st.W) return;
  const int N = cs.N;
  double vo[3];
  drift_old(cs, st, w, iel, vo, mb.md_velo ? mb.md_velo + 3 * w : nullptr);
  for (int k = 0; k < 3; k++) db.vold[((size_t)w * 3 + k) * N + iel] = vo[k];
  const double tau = sc.tau, rttau = sqrt(tau), adrift = 0.5;
  DRng rng;
  rng.load(st.rng + 4 * (size_t)w);
  double dfus2o = 0, fnormo = 1.0;
  MoveScratch &m = mb.ms[w];
  if (cs.nloc == 0) {
    const double xo[3] = {st.x[((size_t)w * 3 + 0) * N + iel], st.x[((size_t)w * 3 + 1) * N + iel],
                          st.x[((size_t)w * 3 + 2) * N + iel]};
    const AeFrame f = ae_frame_d(cs, xo, vo, tau);
    const double c[3] = {cs.cent[3 * f.ic], cs.cent[3 * f.ic + 1], cs.cent[3 * f.ic + 2]};
    double xn[3] = {f.xd[0], f.xd[1], f.xd[2]}, dfusb;
    if (rng.uniform() < f.pgaus) {
      double dfus2b = 0;
      for (int k = 0; k < 3; k++) {
        const double dfus = gauss_d(rng) * rttau;
        dfus2o += dfus * dfus;
        xn[k] = xn[k] + dfus;
        dfus2b += (xn[k] - c[k]) * (xn[k] - c[k]);
      }
      dfusb = sqrt(dfus2b);
    } else {
      const double u1 = rng.uniform(), u2 = rng.uniform(), u3 = rng.uniform();
      dfusb = (-0.5 / f.zeta) * log(u1 * u2 * u3);
      const double costht = 2.0 * (rng.uniform() - 0.5);
      const double sintht = sqrt(1.0 - costht * costht);
      const double phi = 2.0 * 3.141592653589793115997963468544185161590576171875 * rng.uniform();
      for (int k = 0; k < 3; k++) {
        const double dfus = k == 0 ? dfusb * sintht * cos(phi) : k == 1 ? dfusb * sintht * sin(phi) : dfusb * costht;
        dfus2o += (c[k] + dfus - xn[k]) * (c[k] + dfus - xn[k]);
        xn[k] = c[k] + dfus;
      }
    }
    fnormo = f.pgaus + f.qgaus * ae_term(tau) * f.zeta * f.zeta * f.zeta * exp(-2.0 * f.zeta * dfusb + 0.5 * dfus2o / tau);
    for (int k = 0; k < 3; k++) m.xnew[k] = xn[k];
  } else {
    const double v2old = vo[0] * vo[0] + vo[1] * vo[1] + vo[2] * vo[2];
    const double vavvt = (sqrt(1.0 + 2.0 * adrift * v2old * tau) - 1.0) / (adrift * v2old);
    for (int k = 0; k < 3; k++) {
      const double drift = vavvt * vo[k];
      const double dfus = gauss_d(rng) * rttau;
      const double dx = drift + dfus;
      dfus2o += dfus * dfus;
      m.xnew[k] = st.x[((size_t)w * 3 + k) * N + iel] + dx;
    }
  }
  rng.store(st.rng + 4 * (size_t)w);
  m.igeo = 0;
  db.acc[(size_t)w * DA_NA + DA_DFUS2O] = dfus2o;
  db.acc[(size_t)w * DA_NA + DA_FNORMO] = fnormo;
}

// thread per walker: ratio and drift at the new point, reverse diffusion,
// acceptance p = |psi_n/psi_o|^2 G(o<-n)/G(n<-o) with the age boost
__global__ void k_dmc_decide(const __grid_constant__ CSys cs, WState st, MoveBuf mb, GSys g, DmcBuf db, DmcScalars sc, int iel,
                             int *acc_list, int *acc_count) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= st.W) return;
  const int N = cs.N, nmax = cs.nmax, Oa = cs.Oa;
  const int iab = iel < cs.nup ? 0 : 1, nel = iab == 0 ? cs.nup : cs.ndn, ish = iab == 0 ? 0 : cs.nup;
  MoveScratch &m = mb.ms[w];
  const double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax + (size_t)nel * (iel - ish);
  const double *orbn = mb.orbn + (size_t)w * 4 * Oa;
  const int *slot = g.slot_orb + iab * nmax;
  double *acc = db.acc + (size_t)w * DA_NA;
  const double tau = sc.tau, adrift = 0.5;
  double ratio = 0;
  for (int j = 0; j < nel; j++) ratio += sl[j] * orbn[slot[j]];
  const double detn = st.detiab[2 * w + iab] * ratio;
  const double psidn = mb.md_psidn ? mb.md_psidn[w] : detn * st.detiab[2 * w + (1 - iab)] * cs.cdet;
  const double psijn = mb.fsumn[w];
  double vn[3] = {0, 0, 0};
  if (detn != 0.0) {
    double v0 = 0, v1 = 0, v2 = 0;
    for (int j = 0; j < nel; j++) {
      const double s = sl[j] / ratio;
      v0 += s * orbn[1 * Oa + slot[j]];
      v1 += s * orbn[2 * Oa + slot[j]];
      v2 += s * orbn[3 * Oa + slot[j]];
    }
    const double *mv = mb.md_veln ? mb.md_veln + 3 * w : nullptr;
    vn[0] = (mv ? mv[0] : 0.0) + v0 + mb.vjn[3 * w + 0];
    vn[1] = (mv ? mv[1] : 0.0) + v1 + mb.vjn[3 * w + 1];
    vn[2] = (mv ? mv[2] : 0.0) + v2 + mb.vjn[3 * w + 2];
  }
  const double psido = st.psido[w], psijo = st.psijo[w];
  if (psidn * psido <= 0.0) acc[DA_NODECR] += 1;  // icross=1: counted, the move is not refused
  double dfus2n = 0, fnormn = 1.0;
  if (cs.nloc == 0) {
    // dmc_ae's reverse move: the drifted point of the new position and the
    // density of returning to the old one
    const AeFrame f = ae_frame_d(cs, m.xnew, vn, tau);
    double dfus2b = 0;
    for (int k = 0; k < 3; k++) {
      const double xo = st.x[((size_t)w * 3 + k) * N + iel], c = cs.cent[3 * f.ic + k];
      dfus2b += (c - xo) * (c - xo);
      dfus2n += (f.xd[k] - xo) * (f.xd[k] - xo);
    }
    const double dfusb = sqrt(dfus2b);
    fnormn = f.pgaus + f.qgaus * ae_term(tau) * f.zeta * f.zeta * f.zeta * exp(-2.0 * f.zeta * dfusb + 0.5 * dfus2n / tau);
  } else {
    const double v2new = vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2];
    const double vavvt = (sqrt(1.0 + 2.0 * adrift * v2new * tau) - 1.0) / (adrift * v2new);
    for (int k = 0; k < 3; k++) {
      const double xbac = m.xnew[k] + vavvt * vn[k];
      const double dfus = xbac - st.x[((size_t)w * 3 + k) * N + iel];
      dfus2n += dfus * dfus;
    }
  }
  const double dfus2o = acc[DA_DFUS2O];
  double p = (psidn / psido) * (psidn / psido) * exp(2 * (psijn - psijo)) * exp((dfus2o - dfus2n) / (2.0 * tau)) *
             fnormn / acc[DA_FNORMO];
  const int age = db.iage[w];
  if (age > 50) p = p * pow(1.1, (double)(age - 50));
  p = fmin(1.0, p);
  acc[DA_ACC] += p;
  acc[DA_TRY] += 1;
  acc[DA_DFUS2AC] += p * dfus2o;
  acc[DA_DFUS2UN] += dfus2o;
  DRng rng;
  rng.load(st.rng + 4 * (size_t)w);
  const int a = (rng.uniform() < p) ? 1 : 0;
  rng.store(st.rng + 4 * (size_t)w);
  m.acc = a;
  m.ratio = ratio;
  if (a && acc_list) acc_list[atomicAdd(acc_count, 1)] = w;  // for the commit (order free)
  if (a) {
    acc[DA_IACCEPT] = 1;
    acc[DA_NACC] += 1;
    db.iage[w] = 0;
    for (int k = 0; k < 3; k++) st.x[((size_t)w * 3 + k) * N + iel] = m.xnew[k];
    st.psido[w] = psidn;
    st.psijo[w] = psijn;
    st.fsumo[w] = psijn;
    st.detiab[2 * w + iab] = detn;
  }
}

// Warp per walker, after hpsi: drift of every electron, fratio
// (dmc_eloc_cutoff, nloc>0 branch), and for mode 1 the reweighting
// (calculate_reweight) and the walker's sums of the step.
__global__ void k_dmc_weights(const __grid_constant__ CSys cs, WState st, DmcBuf db, DmcScalars sc, int mode, const double *md_vall) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= st.W) return;
  const int N = cs.N;
  const double tau = sc.tau, adrift = 0.5;
  double vav2sum = 0, v2sum = 0;
  for (int e = lane; e < N; e += 32) {
    double v[3];
    drift_old(cs, st, w, e, v, md_vall ? md_vall + ((size_t)w * N + e) * 3 : nullptr);
    for (int k = 0; k < 3; k++) db.vold[((size_t)w * 3 + k) * N + e] = v[k];
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    double vavvt;
    if (cs.nloc == 0) {
      // all-electron branch: adrift of the electron's nearest nucleus, with
      // dmc_ae's adrift0 = 0.1
      const double x[3] = {st.x[((size_t)w * 3 + 0) * N + e], st.x[((size_t)w * 3 + 1) * N + e],
                           st.x[((size_t)w * 3 + 2) * N + e]};
      const int ic = nearest_centre_d(cs, x);
      double rmin = 0, vr = 0;
      for (int k = 0; k < 3; k++) {
        const double rv = x[k] - cs.cent[3 * ic + k];
        rmin += rv * rv;
        vr += v[k] * rv;
      }
      rmin = sqrt(rmin);
      vr = vr / rmin;
      const double va = sqrt(v2), z = cs.znuc[cs.iwctype[ic]];
      const double hafzr2 = (0.5 * z * rmin) * (0.5 * z * rmin);
      const double adriftn = (0.5 * (1 + 1.0e-10 + vr / va)) + 0.1 * hafzr2 / (1 + hafzr2);
      vavvt = (sqrt(1.0 + 2.0 * adriftn * v2 * tau) - 1.0) / (adriftn * v2);
    } else {
      vavvt = (sqrt(1.0 + 2.0 * adrift * v2 * tau * 1.0) - 1.0) / (adrift * v2);
    }
    const double vavvn = vavvt / (tau * 1.0);
    vav2sum += vavvn * vavvn * v2;
    v2sum += v2;
  }
  vav2sum = warp_sum(vav2sum);
  v2sum = warp_sum(v2sum);
  if (lane != 0) return;
  const double fration = sqrt(vav2sum / v2sum);
  if (mode == 0) {
    db.fratio[w] = fration;
    return;
  }
  double *acc = db.acc + (size_t)w * DA_NA;
  const double taunow = tau * acc[DA_DFUS2AC] / acc[DA_DFUS2UN] * 1.0;
  const double enew = st.eold[w];  // hpsi of this step
  const double eold = db.eprev[w];
  const double deo = sc.eest - eold, den = sc.eest - enew;
  const double ewto = sc.eest - deo * db.fratio[w];
  const double ewtn = sc.eest - den * fration;
  double dwt = exp((sc.etrial - 0.5 * (ewto + ewtn)) * taunow);
  dwt = dwt * sc.ffi;
  const double wt = db.wt[w] * dwt;
  db.wt[w] = wt;
  const double wtg = wt * sc.fprod;
  acc[DA_TAUSUM] = wtg * taunow;
  db.fratio[w] = fration;
  if (acc[DA_IACCEPT] == 0) db.iage[w] += 1;
  const double ekino = st.ekino[w];
  acc[DA_WSUM1] = wt;
  acc[DA_ESUM1] = wt * enew;
  acc[DA_PESUM] = wtg * (enew - ekino);
  acc[DA_TPBSUM] = wtg * ekino;
}

// T-move choice of every walker (icasula = -1, nonloc_grid,
// dmc/nonloc_grid.f90:3, over all electrons): warp per walker.  t_norm =
// 1 + tau sum(-t) over the negative matrix elements; when some exist one
// draw p from the walker's stream and the first (electron, point, centre),
// in CHAMP's loop order, whose cumulative -tau t / t_norm exceeds p moves:
// each lane sums a contiguous chunk, a warp scan finds the chunk, its lane
// walks it.  The proposed point is r_en(e, ic) times the rotated quadrature
// direction about the centre.
__global__ void k_tmove_select(const __grid_constant__ CSys cs, WState st, MoveBuf mb, const double *tv, DmcScalars sc) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= st.W) return;
  const int N = cs.N, M = cs.M, NQ = cs.nquad;
  const int L = N * NQ * M;
  const double *t = tv + (size_t)w * L;
  const int per = (L + 31) / 32, a = lane * per, b = min(L, a + per);
  double sneg = 0;
  for (int k = a; k < b; k++) {
    const double v = t[k];
    if (v < 0.0) sneg -= v;
  }
  const double tot = warp_sum(sneg);
  const double tau = sc.tau;
  const double t_norm = 1.0 + tot * tau;
  MoveScratch &m = mb.ms[w];
  if (t_norm == 1.0) {
    if (lane == 0) m.igeo = 1;
    return;
  }
  const double t_normi = 1.0 / t_norm;
  double p = 0;
  if (lane == 0) {
    DRng rng;
    rng.load(st.rng + 4 * (size_t)w);
    p = rng.uniform();
    rng.store(st.rng + 4 * (size_t)w);
  }
  p = __shfl_sync(0xffffffffu, p, 0);
  double cl = 0;
  for (int k = a; k < b; k++) {
    const double v = t[k];
    cl = cl - tau * (v < 0.0 ? v : 0.0) * t_normi;
  }
  double incl = cl;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  const unsigned hit = __ballot_sync(0xffffffffu, incl > p && b > a);
  if (hit == 0) {
    if (lane == 0) m.igeo = 1;
    return;
  }
  const int l0 = __ffs(hit) - 1;
  if (lane != l0) return;
  double t_cum = incl - cl;
  int kk = -1, last_neg = -1;
  for (int k = a; k < b; k++) {
    const double v = t[k];
    if (v < 0.0) last_neg = k;
    t_cum = t_cum - tau * (v < 0.0 ? v : 0.0) * t_normi;
    if (t_cum > p) {
      kk = k;
      break;
    }
  }
  // rounding between the chunk sum and the walk: the chunk's last transition
  if (kk < 0) kk = last_neg;
  if (kk < 0) {
    m.igeo = 1;
    return;
  }
  const int e = kk / (NQ * M), iq = (kk / M) % NQ, ic = kk % M;
  double d[3], r2 = 0;
  for (int k = 0; k < 3; k++) {
    d[k] = st.x[((size_t)w * 3 + k) * N + e] - cs.cent[3 * ic + k];
    r2 += d[k] * d[k];
  }
  const double r = sqrt(r2);
  const double *xq = st.xq + (size_t)w * 3 * NQ;
  for (int k = 0; k < 3; k++) m.xnew[k] = r * xq[k * NQ + iq] + cs.cent[3 * ic + k];
  m.igeo = 0;
  m.tel = e;
}

// T-move of the chosen electron, always accepted (icasula = -1): ratio at
// the point, psi_D, psi_J, commit of the scalars; k_commit applies the
// matrix and table updates.  Thread per walker.
__global__ void k_tmove_accept(const __grid_constant__ CSys cs, WState st, MoveBuf mb, GSys g, DmcBuf db,
                               const double *md_psidn) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= st.W) return;
  MoveScratch &m = mb.ms[w];
  if (m.igeo) {
    m.acc = 0;
    return;
  }
  const int N = cs.N, nmax = cs.nmax, Oa = cs.Oa, iel = m.tel;
  const int iab = iel < cs.nup ? 0 : 1, nel = iab == 0 ? cs.nup : cs.ndn, ish = iab == 0 ? 0 : cs.nup;
  const double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax + (size_t)nel * (iel - ish);
  const double *orbn = mb.orbn + (size_t)w * 4 * Oa;
  const int *slot = g.slot_orb + iab * nmax;
  double ratio = 0;
  for (int j = 0; j < nel; j++) ratio += sl[j] * orbn[slot[j]];
  const double detn = st.detiab[2 * w + iab] * ratio;
  // multideterminant: psi_D of the expansion at the point (k_md_move)
  const double psidn = md_psidn ? md_psidn[w] : detn * st.detiab[2 * w + (1 - iab)] * cs.cdet;
  if (detn == 0.0) {
    st.status[w] |= 1;
    m.acc = 0;
    return;
  }
  m.acc = 1;
  m.ratio = ratio;
  for (int k = 0; k < 3; k++) st.x[((size_t)w * 3 + k) * N + iel] = m.xnew[k];
  st.psido[w] = psidn;
  st.psijo[w] = mb.fsumn[w];
  st.fsumo[w] = mb.fsumn[w];
  st.detiab[2 * w + iab] = detn;
  db.iage[w] = 0;
  db.acc[(size_t)w * DA_NA + DA_TMOVE] = 1;
}

struct QuadRot {
  double x[CW_MAX_QUAD], y[CW_MAX_QUAD], z[CW_MAX_QUAD];
};

__global__ void k_set_quad(const __grid_constant__ CSys cs, WState st, QuadRot q) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= st.W) return;
  const int NQ = cs.nquad;
  double *xq = st.xq + (size_t)w * 3 * NQ;
  for (int i = 0; i < NQ; i++) {
    xq[i] = q.x[i];
    xq[NQ + i] = q.y[i];
    xq[2 * NQ + i] = q.z[i];
  }
}

// Per-walker fields of a splitj copy: every array the next step reads
// (configuration, wave-function tables, drift, fratio) except the random
// stream, which stays with its slot.
struct WalkerRec {
  int nfield;
  double *ptr[24];
  long len[24];  // doubles per walker
};

// CTA per copy: walker copy_src[c] -> slot copy_dst[c].  The host guarantees
// that no source slot is also a destination, so copies run concurrently.
__global__ void k_walker_copy(WalkerRec rec, DmcBuf db, int ncopy) {
  const int c = blockIdx.x;
  if (c >= ncopy) return;
  const int src = db.copy_src[c], dst = db.copy_dst[c];
  for (int f = 0; f < rec.nfield; f++) {
    const long n = rec.len[f];
    const double *p = rec.ptr[f] + (size_t)src * n;
    double *q = rec.ptr[f] + (size_t)dst * n;
    for (long t = threadIdx.x; t < n; t += blockDim.x) q[t] = p[t];
  }
}

}  // namespace cw
