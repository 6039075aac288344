// Jastrow parameter derivatives for the wave-function optimisation sums
// (vmc/deriv_jastrow4.f90, the gvalue part used by optwf_store / sr_o).
//
//   k_jas_raw   d J / d p of every Jastrow coefficient taken on its own, per
//               walker, at the current configuration (CTA per walker)
//   k_jas_o     the linear map from those raw derivatives to the varied
//               parameters of the jasderiv selection (cusp-dependent e-e-n
//               terms folded in), written into the optimisation vector
//
// Raw layout per walker (shared with the CPU oracle):
//   [nctype][norda+1]  a: q = 1 Pade numerator a(1), q = 2 Pade denominator
//                      a(2), q >= 3 the coefficient of r^(q-1)
//   [nspin2b][nordb+1] b: the same for the e-e function (sspinn on the Pade
//                      terms)
//   [nctype][nterms]   c: the e-e-n term values uu(k) ss(l) tt(m)
// The asymptotic constants follow a and b, as in deriv_jastrow4
// (gen/gee subtract their value at asymp_r).
#pragma once
#include "common.cuh"

namespace cw {

__host__ __device__ constexpr int een_nterms(int nord) {
  int i = 0;
  for (int n = 2; n <= nord; n++)
    for (int k = n - 1; k >= 0; k--)
      for (int l = (k == 0 ? n - k - 2 : n - k); l >= 0; l--)
        if (2 * ((n - k - l) / 2) == n - k - l) i++;
  return i;
}

// acc[ll] += uu(k) ss(l) tt(m) for every e-e-n term ll (jastrow4's n/k/l
// enumeration; ss(l) = x^l + y^l, tt(m) = x^m y^m with switch-scaled x, y)
template <int NORD>
__device__ __forceinline__ void een_term_values(const double *uu, const double *xp, const double *yp, double *acc) {
  int ll = 0;
#pragma unroll
  for (int n = 2; n <= NORD; n++)
#pragma unroll
    for (int k = n - 1; k >= 0; k--) {
#pragma unroll
      for (int l = (k == 0 ? n - k - 2 : n - k); l >= 0; l--) {
        const int m = (n - k - l) / 2;
        if (2 * m == n - k - l) {
          acc[ll] += uu[k] * ((xp[l] + yp[l]) * (xp[m] * yp[m]));
          ll++;
        }
      }
    }
}

// Deterministic block reduction of the first nv of NV per-thread values
// (a register array): butterfly within each warp, then thread v adds the
// warps' partials in warp order.
template <int NV>
__device__ __forceinline__ void jas_flush(const double (&acc)[NV], int nv, double *red, double *dst) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; v++) {
    if (v >= nv) break;
    const double s = warp_sum(acc[v]);
    if (lane == 0) red[wid * nv + v] = s;
  }
  __syncthreads();
  for (int v = threadIdx.x; v < nv; v += blockDim.x) {
    double s = 0;
    for (int q = 0; q < nw; q++) s += red[q * nv + v];
    dst[v] = s;
  }
  __syncthreads();
}

constexpr int kJasThreads = 128;

template <int NORD>
__global__ void __launch_bounds__(kJasThreads) k_jas_raw(const __grid_constant__ CSys cs, WState st, double *raw, int nraw) {
  constexpr int NTC = NORD > 1 ? een_nterms(NORD) : 1;
  constexpr int NAM = CW_MAX_NORD + 1;
  __shared__ double red[(kJasThreads / 32) * (NTC > 2 * NAM ? NTC : 2 * NAM)];
  const int w = blockIdx.x;
  if (w >= st.W) return;
  const int N = cs.N, M = cs.M, tid = threadIdx.x;
  const int NA = cs.norda + 1, NB = cs.nordb + 1, NT = cs.nterms;
  const int ob = cs.nctype * NA, oc = ob + cs.nspin2b * NB;
  const double kap = cs.scalek, ar = cs.asymp_r;
  const double *xw = st.x + (size_t)w * 3 * N;
  const double *enr = st.enm + (size_t)w * 2 * M * N;  // scaled e-n distances [M][N]
  double *out = raw + (size_t)w * nraw;
  double arp[NAM];  // asymp_r^p
  arp[0] = 1;
#pragma unroll
  for (int p = 1; p < NAM; p++) arp[p] = arp[p - 1] * ar;

  // a part (deriv_jastrow4.f90:588-640), one centre type at a time
  for (int it = 0; it < cs.nctype; it++) {
    double acc[NAM];
#pragma unroll
    for (int q = 0; q < NAM; q++) acc[q] = 0;
    const double a1 = cs.a4[it * NA], a2 = cs.a4[it * NA + 1];
    const double pa1 = ar / (1 + a2 * ar), pa2 = a1 * ar * ar / ((1 + a2 * ar) * (1 + a2 * ar));
    for (int t = tid; t < N * M; t += blockDim.x) {
      const int ic = t / N;
      if (cs.iwctype[ic] != it) continue;
      const double r = enr[t];
      if (r == ar) continue;
      const double bot0 = 1 + a2 * r;
      acc[0] += r / bot0 - pa1;
      acc[1] += -a1 * r * r / (bot0 * bot0) + pa2;
      double rp = r;
#pragma unroll
      for (int q = 3; q <= NAM; q++) {
        rp *= r;
        if (q <= NA) acc[q - 1] += rp - arp[q - 1];
      }
    }
    jas_flush(acc, NA, red, out + it * NA);
  }

  // b part (deriv_jastrow4.f90:181-234), both spin classes together
  const int npair = N * (N - 1) / 2;
  auto pair_of = [&](int p, int &i, int &j) {
    i = (int)((1.0 + sqrt(8.0 * p + 1.0)) * 0.5);
    while (i * (i - 1) / 2 > p) i--;
    while ((i + 1) * i / 2 <= p) i++;
    j = p - i * (i - 1) / 2;
  };
  {
    double acc[2][NAM];
#pragma unroll
    for (int q = 0; q < NAM; q++) acc[0][q] = acc[1][q] = 0;
    for (int p = tid; p < npair; p += blockDim.x) {
      int i, j, isb, ipar;
      double sspinn;
      pair_of(p, i, j);
      pair_spin(cs, i, j, isb, ipar, sspinn);
      const double d0 = xw[i] - xw[j], d1 = xw[N + i] - xw[N + j], d2 = xw[2 * N + i] - xw[2 * N + j];
      double u, dd1, dd2;
      scale2<double>(cs, sqrt(d0 * d0 + d1 * d1 + d2 * d2), u, dd1, dd2);
      if (u == ar) continue;
      const double b1 = cs.b[isb * NB], b2 = cs.b[isb * NB + 1];
      const double bot0 = 1 + b2 * u;
      double g[NAM];
      g[0] = sspinn * u / bot0 - sspinn * ar / (1 + b2 * ar);
      g[1] = -sspinn * b1 * u * u / (bot0 * bot0) + sspinn * b1 * ar * ar / ((1 + b2 * ar) * (1 + b2 * ar));
      double up = u;
#pragma unroll
      for (int q = 3; q <= NAM; q++) {
        up *= u;
        g[q - 1] = up - arp[q - 1];
      }
#pragma unroll
      for (int q = 0; q < NAM; q++) {
        if (q >= NB) continue;
        if (isb == 0) acc[0][q] += g[q];
        else acc[1][q] += g[q];
      }
    }
    jas_flush(acc[0], NB, red, out + ob);
    if (cs.nspin2b == 2) jas_flush(acc[1], NB, red, out + ob + NB);
  }

  // c part (deriv_jastrow4.f90:250-330), one centre type at a time
  if (NORD > 1) {
    for (int it = 0; it < cs.nctype; it++) {
      double acc[NTC];
#pragma unroll
      for (int q = 0; q < NTC; q++) acc[q] = 0;
      for (int p = tid; p < npair; p += blockDim.x) {
        int i, j;
        pair_of(p, i, j);
        const double d0 = xw[i] - xw[j], d1 = xw[N + i] - xw[N + j], d2 = xw[2 * N + i] - xw[2 * N + j];
        double u, dd1, dd2;
        scale2<double>(cs, sqrt(d0 * d0 + d1 * d1 + d2 * d2), u, dd1, dd2);
        double uu[NORD + 1];
        uu[0] = 1;
        uu[1] = 1 - kap * u;
#pragma unroll
        for (int k = 2; k <= NORD; k++) uu[k] = uu[k - 1] * uu[1];
        for (int ic = 0; ic < M; ic++) {
          if (cs.iwctype[ic] != it) continue;
          const double ri = enr[ic * N + i], rj = enr[ic * N + j];
          if (ri == ar && rj == ar) continue;
          double xp[NORD + 1], yp[NORD + 1];
          xp[0] = yp[0] = 1;
          xp[1] = 1 - kap * ri;
          yp[1] = 1 - kap * rj;
#pragma unroll
          for (int k = 2; k <= NORD; k++) {
            xp[k] = xp[k - 1] * xp[1];
            yp[k] = yp[k - 1] * yp[1];
          }
          een_term_values<NORD>(uu, xp, yp, acc);
        }
      }
      jas_flush(acc, NT, red, out + oc + it * NT);
    }
  }
}

// O[w][k] = sum_r raw[w][r] map[r][k] for the njas varied Jastrow
// parameters, into columns 0..njas-1 of the optimisation vector o (row
// stride np) and rows 0..njas-1 of its transpose ot [np][W]
__global__ void k_jas_o(int W, const double *raw, int nraw, const double *map, int njas, int np, double *o,
                        double *ot) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)W * njas) return;
  const int w = (int)(t / njas), k = (int)(t % njas);
  const double *rw = raw + (size_t)w * nraw;
  double s = 0;
  for (int r = 0; r < nraw; r++) s += rw[r] * map[(size_t)r * njas + k];
  o[(size_t)w * np + k] = s;
  ot[(size_t)k * W + w] = s;
}

}  // namespace cw

namespace cw {
// ---------------------------------------------------------------------------
// Orbital-rotation derivatives for a single determinant (optorb_deriv's
// orbprim, vmc/optorb.f90:5-95, whose multideterminant terms vanish for one
// determinant): for the variation phi_io -> phi_io + a phi_jo,
// d ln psi / d a = sum over the spins whose determinant holds io of
// aa(irep, jo) = sum_i slmi(irep + (i-1) nel) phi_jo(r_i)
// (multideterminant_hpsi, vmc/multideterminant.f90:66-82).
// ---------------------------------------------------------------------------
struct OrbTerm {
  int slot[2];  // slot of io in the up / down determinant (-1: io not there)
  int v;        // index of jo in the list of rotation targets
  int io;       // io itself (active-orbital index, 0-based)
};

// values of the rotation targets at the electrons [e0, e0+ne) of every
// walker, from the value rows of the chunk's LCAO (rows ((w*ne + e)*5 + 0)):
// vals [W][N][nv]
__global__ void k_orb_vals(int W, int N, int e0, int ne, int Oa, const double *__restrict__ orball, int nv,
                           const int *__restrict__ vorb, double *__restrict__ vals) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)W * ne * nv) return;
  const int v = (int)(t % nv);
  const long we = t / nv;
  const int el = (int)(we % ne), w = (int)(we / ne);
  vals[((size_t)w * N + e0 + el) * nv + v] = orball[(size_t)we * 5 * Oa + vorb[v]];
}

// thread per (walker, term): the derivative into the optimisation vector,
// columns [off, off + nterm) of o [W][np] and ot [np][W]
__global__ void k_orb_o(const __grid_constant__ CSys cs, WState st, int nterm, const OrbTerm *__restrict__ terms, int nv,
                        const double *__restrict__ vals, double *o, double *ot, int np, int off) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)st.W * nterm) return;
  const int k = (int)(t % nterm), w = (int)(t / nterm);
  const int N = cs.N, nmax = cs.nmax;
  const OrbTerm tm = terms[k];
  double sum = 0;
  for (int iab = 0; iab < 2; iab++) {
    const int irep = tm.slot[iab];
    if (irep < 0) continue;
    const int nel = iab == 0 ? cs.nup : cs.ndn, ish = iab == 0 ? 0 : cs.nup;
    const double *sl = st.slmi + ((size_t)w * 2 + iab) * nmax * nmax;
    double a = 0;
    for (int i = 0; i < nel; i++) a += sl[irep + (size_t)nel * i] * vals[((size_t)w * N + ish + i) * nv + tm.v];
    sum += a;
  }
  o[(size_t)w * np + off + k] = sum;
  ot[(size_t)(off + k) * st.W + w] = sum;
}
// Expansions: optorb_deriv's excitation part (vmc/optorb.f90:62-84), added
// to k_orb_o's reference part: detratio * sum over spins of
//   sum_i zmat(io,i) orb(i,jo)   (io a virtual orbital, io >= ivirt)
// - sum_i aaz(irep,i) orb(i,jo)  (io held by the reference at slot irep),
// with compute_zmat's (vmc/multideterminant.f90:491-560)
//   zmat(v,irep) = sum_{krep >= iactv} Y(v,krep) slmi(krep,irep)   (v >= ivirt)
//   aaz(j,irep)  = sum_{v >= ivirt} aa(j,v) zmat(v,irep).
// CTA per walker; shared: zmat [O][nmax] and aaz [nmax][nmax] of one spin.
__global__ void __launch_bounds__(128) k_md_orb_o(const __grid_constant__ CSys cs, WState st, MdBuf md, int nterm,
                                                  const OrbTerm *__restrict__ terms, int nv,
                                                  const double *__restrict__ vals, double *o, double *ot, int np,
                                                  int off) {
  const int w = blockIdx.x;
  if (w >= st.W) return;
  const int N = cs.N, O = cs.Oa, nmax = cs.nmax;
  extern __shared__ __align__(16) double smem[];
  double *zm = smem;                       // [O][nmax]: zmat(v, irep) at v * nmax + irep
  double *az = zm + (size_t)O * nmax;      // [nmax][nmax]: aaz(j, irep) at j * nmax + irep
  const double detratio = st.detiab[2 * w] * st.detiab[2 * w + 1] / st.psido[w];
  // each thread keeps the running sums of its terms across the two spins
  constexpr int kMaxPer = 8;
  double dpsi[kMaxPer];
  for (int q = 0; q < kMaxPer; q++) dpsi[q] = 0.0;
  for (int s = 0; s < 2; s++) {
    const int n = s == 0 ? cs.nup : cs.ndn, ish = s == 0 ? 0 : cs.nup;
    if (n == 0) continue;
    const int ivirt = cs.md_ivirt[s], iactv = cs.md_iactv[s];
    const double *Y = md.ymat + ((size_t)w * 2 + s) * nmax * O;   // Y(v, krep) at krep * O + v
    const double *aa = md.aa + ((size_t)w * 2 + s) * nmax * O;    // aa(j, v) at j * O + v
    const double *sl = st.slmi + ((size_t)w * 2 + s) * nmax * nmax;
    __syncthreads();  // the previous spin's tables are no longer read
    for (int q = threadIdx.x; q < (O - ivirt) * n; q += blockDim.x) {
      const int v = ivirt + q / n, irep = q - (q / n) * n;
      double z = 0;
      for (int krep = iactv; krep < n; krep++) z += Y[(size_t)krep * O + v] * sl[krep + (size_t)n * irep];
      zm[(size_t)v * nmax + irep] = z;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
      const int j = q / n, irep = q - (q / n) * n;
      double z = 0;
      for (int v = ivirt; v < O; v++) z += aa[(size_t)j * O + v] * zm[(size_t)v * nmax + irep];
      az[(size_t)j * nmax + irep] = z;
    }
    __syncthreads();
    for (int k = threadIdx.x, q = 0; k < nterm && q < kMaxPer; k += blockDim.x, q++) {
      const OrbTerm tm = terms[k];
      const double *ov = vals + ((size_t)w * N + ish) * nv + tm.v;  // orb(ish + i, jo) at i * nv
      double d = dpsi[q];
      if (tm.io >= ivirt)
        for (int i = 0; i < n; i++) d = d + zm[(size_t)tm.io * nmax + i] * ov[(size_t)i * nv];
      const int irep = tm.slot[s];
      if (irep >= 0)
        for (int i = 0; i < n; i++) d = d - az[(size_t)irep * nmax + i] * ov[(size_t)i * nv];
      dpsi[q] = d;
    }
  }
  for (int k = threadIdx.x, q = 0; k < nterm && q < kMaxPer; k += blockDim.x, q++) {
    const double v = dpsi[q] * detratio + o[(size_t)w * np + off + k];
    o[(size_t)w * np + off + k] = v;
    ot[(size_t)(off + k) * st.W + w] = v;
  }
}
}  // namespace cw
