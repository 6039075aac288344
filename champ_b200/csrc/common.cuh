// common.cuh — device-side building blocks of the walker engine.
//
// System constants travel with every launch as a __grid_constant__ kernel
// parameter (the parameter bank is served by the constant cache, so lanes
// reading the same type parameters in lock-step get a broadcast) — one
// block per context, so contexts of different systems run their kernels
// side by side on one device.  Per-centre records and large tables (radial
// splines, LCAO coefficients) live in the context's global memory and stay
// L2-resident.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define CW_MAX_CENT 512
#define CW_MAX_TYPES 8
#define CW_MAX_RWF 16
#define CW_MAX_TERMS 64
#define CW_MAX_NORD 7
#define CW_MAX_QUAD 86
#define CW_MAX_STATES 8   // CI vectors of a multi-state wave function
#define CW_MAX_ELEC 1024

// ---------------------------------------------------------------------------
// System description passed by value to every kernel (at most the 32764
// bytes a kernel parameter list may hold)
// ---------------------------------------------------------------------------
struct CSys {
  int N, nup, ndn, M, nctype, K, Oa, nmax;
  int norda, nordb, nordc, isc, nspin2b, nocuspb, nterms;
  int nloc, nquad;
  double scalek, asymp_r, asymp_jasb[2];
  double deltar, deltat, fbias, pecent, cdet;
  int mrwf, mpts, mbastyp;
  // per centre, in the context's global memory: coordinates [M][3], atom
  // type [M], first AO [M + 1]
  const double *cent;
  const int *iwctype;
  const int *ao_first;
  // per type
  double znuc[CW_MAX_TYPES];
  int nrbas[CW_MAX_TYPES], igrid[CW_MAX_TYPES], nr[CW_MAX_TYPES], nbastyp[CW_MAX_TYPES];
  double arg[CW_MAX_TYPES], r0[CW_MAX_TYPES];
  double rmaxwf[CW_MAX_TYPES * CW_MAX_RWF];
  double ce[CW_MAX_TYPES * CW_MAX_RWF * 5];
  double ae[CW_MAX_TYPES * CW_MAX_RWF * 2];
  double a4[CW_MAX_TYPES * (CW_MAX_NORD + 1)];
  double b[2 * (CW_MAX_NORD + 1)];
  double c[CW_MAX_TYPES * CW_MAX_TERMS];
  float cf[CW_MAX_TYPES * CW_MAX_TERMS];   // FP32 copy of c (mixed-precision Jastrow)
  // multideterminant expansion (ndet > 1)
  int ndet, md_nuniq[2], md_ivirt[2], md_iactv[2];
  int nstates;  // CI vectors sharing orbitals and Jastrow (1 = one state)
  int iguiding; // > 0: the walk samples the guiding function of the states
  double wg[CW_MAX_STATES];  // guiding weights (weights_g, anormo = 1)
  double asymp_jasa[CW_MAX_TYPES];
  // ECP
  int lpot[CW_MAX_TYPES];
  int necp_term[CW_MAX_TYPES * 4];
  int necp_power[CW_MAX_TYPES * 4 * 16];
  double ecp_exponent[CW_MAX_TYPES * 4 * 16];
  double ecp_coef[CW_MAX_TYPES * 4 * 16];
  double xq0[CW_MAX_QUAD], yq0[CW_MAX_QUAD], zq0[CW_MAX_QUAD], wq[CW_MAX_QUAD];
  // Slm (vmc/slm.f90) as monomials: exponents of x, y, z and the constant
  int slm_a[36], slm_b[36], slm_c[36];
  double slm_k[36];
};

static_assert(sizeof(CSys) <= 31 * 1024, "the system block must fit a kernel parameter list");

// asynchronous 8-byte global -> shared copy (sm_80+): a thread issues all of
// its copies back to back and waits once (cp_async8_wait) before the block
// barrier that publishes them
__device__ __forceinline__ void cp_async8(double *dst_smem, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Global-memory tables of the system.
struct GSys {
  const double *rwf, *d2rwf;      // [nctype][mrwf][mpts]
  const double *gridpow;          // [nctype][mpts+1]  r0*arg^(jx-1), jx = 0..mpts
  const int *iwlbas, *iwrwf;      // [nctype][mbastyp]
  const double *coefT;            // [K][Oa]  (active orbitals)
  const int *slot_orb;            // [2][nmax] active-orbital index of Slater column j, spin s
  const int4 *ao;                 // [K] per AO: centre, radial function (0-based), atom type, Slm index
  // per AO, read with the AO index (lanes of a warp take consecutive AOs, so
  // these loads coalesce where indexing the constant block by type would
  // serialise): radial table offset, grid points of the type, packed Slm
  // exponents (a | b << 8 | c << 16); Slm constant and rmaxwf
  const int4 *aox;                // [K]
  const double2 *aok;             // [K]
  // per centre (x, y), (z, atom type as a double): read where the lanes of a
  // warp take different centres
  const double2 *cen;             // [M][2]
};

// centre ic from the per-centre records (two 16-byte loads)
struct Cen { double x, y, z; int it; };
__device__ __forceinline__ Cen cen_of(const GSys &g, int ic) {
  const double2 a = __ldg(g.cen + 2 * ic), b = __ldg(g.cen + 2 * ic + 1);
  return Cen{a.x, a.y, b.x, (int)b.y};
}

// ---------------------------------------------------------------------------
// Per-walker state (walker-major; component planes so lanes over electrons
// coalesce).
// ---------------------------------------------------------------------------
struct WState {
  int W;
  double *x;          // [W][3][N]
  uint64_t *rng;      // [W][4]
  double *xq;         // [W][3][nquad] rotated quadrature
  double *rmino;      // [W][N]
  int *nearesto;      // [W][N]
  double *rvmino;     // [W][3][N]
  double *psido, *psijo, *psi2o, *eold, *ekino;   // [W]
  double *slmi;       // [W][2][nmax*nmax]   slmi(j + nel*(i)) per spin
  double *detiab;     // [W][2]
  double *orbs;       // [W][N][nmax]   Slater-column orbital values of electron e
  double *dorbs;      // [W][3][N][nmax]
  double *fso;        // [W][N][N] symmetric pair values, diagonal = e-n term
  double *fijo;       // [W][3][N][N] fijo(k,i,j) -> [k][i][j]
  double *fjo;        // [W][3][N]
  double *fsumo;      // [W]
  double *enm;        // [W][2][M][N] e-n table of every electron: scaled distance
                      // rr and dd1/r (rebuilt by hpsi, row of a moved electron
                      // replaced on commit)
  float *enmf;        // [W][2][M][N] FP32 copy of enm (mixed precision only;
                      // the FP32 pair kernel reads it), kept in step with enm
  // estimators [W][8]: wsum esum pesum tpbsum acc ecum1s ecm21s (spare)
  double *sums;
  int *status;        // [W] nonzero: singular matrix / NaN
};

// Scratch of one single-electron move.
struct MoveScratch {
  double xnew[3];
  double rvminn[3];
  double rminn, rminon, rminno, delttn, fxop, areao, rratio;
  int nearestn, igeo;
  double rvminon[3];
  double ratio;       // determinant ratio of the proposed move (k_decide)
  double psidn;       // psi_D at a caller's point (k_hook_ratio)
  int acc;           // accepted? (k_decide)
  int tel;           // electron of a T-move (moves whose launch gives no electron)
};

struct MoveBuf {
  MoveScratch *ms;    // [W]
  double *fsn;        // [W][N]      new pair value of (iel,j); [iel] = e-n term
  double *fijn_i;     // [W][3][N]   grad wrt iel of pair (iel,j)
  double *fijn_j;     // [W][3][N]   grad wrt j of pair (iel,j)
  double *fsumn;      // [W]
  double *vjn;        // [W][3]
  double *phi;        // [W][4][K]  basis at xnew (value, dx, dy, dz)
  double *orbn;       // [W][4][Oa]
  double *enn;        // [W][2][M]  e-n row (rr, dd1/r) of the moved electron at xnew
  float *phi_hi, *phi_lo;  // mixed precision: [W*4][kp] split basis rows (null in FP64)
  int kp;                  // row pitch of phi_hi/phi_lo (K rounded up to 32)
  // multideterminant terms of the move (null for one determinant)
  const double *md_velo;   // [W][3] drift correction at the old position
  const double *md_veln;   // [W][3] drift correction at the proposed position
  const double *md_psidn;  // [W]    psi_D at the proposed position
  const double *md_psi2g;  // [W]    guiding factor psi2g at the proposed position (null: 1)
};

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
// FP64 -> (hi, lo) FP32 pair, hi exactly TF32-representable (round to
// nearest, ties away), lo the FP32 remainder: the operand split of the
// tensor-core LCAO contraction.
__device__ __forceinline__ void split_tf32(double x, float &hi, float &lo) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"((float)x));
  hi = __uint_as_float(h);
  lo = (float)(x - (double)hi);
}

// determinant_psig (vmc/determinant_psig.f90:3) with anormo = 1 from the S
// of every state (psi_i/psi_1 = S_i/S_1, one orbital set and Jastrow):
// psi2g = w_1 + sum_{i>1} w_i (S_i/S_1)^2
__device__ __forceinline__ double md_psig(const CSys &cs, const double *S, int ns) {
  double g = cs.wg[0];
  for (int i = 1; i < ns; i++) {
    const double r = S[i] / S[0];
    g = g + cs.wg[i] * r * r;
  }
  return g;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// xoshiro256** (CHAMP vmc/xoroshiro256starstar.c next / next_uniform_double)
struct DRng {
  uint64_t s0, s1, s2, s3;
  __host__ __device__ __forceinline__ uint64_t next() {
    const uint64_t r1 = s1 * 5;
    const uint64_t result = ((r1 << 7) | (r1 >> 57)) * 9;
    const uint64_t t = s1 << 17;
    s2 ^= s0;
    s3 ^= s1;
    s1 ^= s2;
    s0 ^= s3;
    s2 ^= t;
    s3 = (s3 << 45) | (s3 >> 19);
    return result;
  }
  __host__ __device__ __forceinline__ double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
  __host__ __device__ void load(const uint64_t *p) { s0 = p[0]; s1 = p[1]; s2 = p[2]; s3 = p[3]; }
  __host__ __device__ void store(uint64_t *p) const { p[0] = s0; p[1] = s1; p[2] = s2; p[3] = s3; }
};

// ---------------------------------------------------------------------------
// scale_dist family (vmc/scale_dist.f90:57-353)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T scale0(const CSys &cs, T r) {
  const T k = (T)cs.scalek;
  if (cs.scalek == 0) return r;
  if (cs.isc == 2) return (T(1) - exp(-k * r)) / k;
  if (cs.isc == 3) {
    T rsc = k * r, rsc2 = rsc * rsc, rsc3 = rsc * rsc2;
    return (T(1) - exp(-rsc - T(0.5) * rsc2 - (T(1) / T(3)) * rsc3)) / k;
  }
  if (cs.isc == 4) return r * (T(1) / (T(1) + k * r));
  return r * (T(1) / pow(T(1) + pow(k * r, T(3)), T(1) / T(3)));
}
template <typename T>
__device__ __forceinline__ void scale2(const CSys &cs, T r, T &rr, T &dd1, T &dd2) {
  const T k = (T)cs.scalek;
  if (cs.scalek == 0) { rr = r; dd1 = 1; dd2 = 0; return; }
  if (cs.isc == 2) {
    rr = (T(1) - exp(-k * r)) / k;
    dd1 = T(1) - k * rr;
    dd2 = -k * dd1;
  } else if (cs.isc == 3) {
    T rsc = k * r, rsc2 = rsc * rsc, rsc3 = rsc * rsc2;
    T e = exp(-rsc - T(0.5) * rsc2 - (T(1) / T(3)) * rsc3);
    rr = (T(1) - e) / k;
    dd1 = (T(1) + rsc + rsc2) * e;
    dd2 = -k * rsc2 * (T(3) + T(2) * rsc + rsc2) * e;
  } else if (cs.isc == 4) {
    T deni = T(1) / (T(1) + k * r);
    rr = r * deni;
    dd1 = deni * deni;
    dd2 = -T(2) * k * deni * dd1;
  } else {
    T deni = T(1) / pow(T(1) + pow(k * r, T(3)), T(1) / T(3));
    rr = r * deni;
    dd1 = deni * deni * deni * deni;
    dd2 = -T(4) * (k * r) * (k * r) * k * dd1 * dd1 / deni;
  }
}

// ---------------------------------------------------------------------------
// e-e-n polynomial of jastrow4 / jastrow4e / psinl: the (n,k,l,m) term table
// unrolled at compile time for a given order.
//   MODE 0: value only, 1: value + first derivs, 2: + second derivs
// ---------------------------------------------------------------------------
template <typename T>
struct EenOut { T fc, fu, fuu, fi, fii, fj, fjj, fui, fuj; };

template <int NORD, int MODE, typename T>
__device__ __forceinline__ EenOut<T> een_poly(const T *__restrict__ cc, T u1, T ri1, T rj1) {
  T uu[NORD + 1], rri[NORD + 1], rrj[NORD + 1], ss[NORD + 1], tt[NORD + 1];
  uu[0] = 1; rri[0] = 1; rrj[0] = 1; ss[0] = 2; tt[0] = 1;
#pragma unroll
  for (int p = 1; p <= NORD; p++) {
    uu[p] = (p == 1) ? u1 : uu[1] * uu[p - 1];
    rri[p] = (p == 1) ? ri1 : rri[1] * rri[p - 1];
    rrj[p] = (p == 1) ? rj1 : rrj[1] * rrj[p - 1];
    ss[p] = rri[p] + rrj[p];
    tt[p] = rri[p] * rrj[p];
  }
  EenOut<T> e{0, 0, 0, 0, 0, 0, 0, 0, 0};
  int ll = 0;
#pragma unroll
  for (int n = 2; n <= NORD; n++) {
#pragma unroll
    for (int k = n - 1; k >= 0; k--) {
      const int l_hi = (k == 0) ? n - k - 2 : n - k;
#pragma unroll
      for (int l = l_hi; l >= 0; l--) {
        const int m = (n - k - l) / 2;
        if (2 * m == n - k - l) {
          const T c = cc[ll];
          ll++;
          const T ukm = (k >= 1) ? uu[k - 1] : T(0);
          const T st = ss[l] * tt[m];
          e.fc += c * uu[k] * st;
          if (MODE >= 1) {
            e.fu += c * T(k) * ukm * st;
            const T gi = T(l + m) * ((l + m >= 1) ? rri[l + m - 1] : T(0)) * rrj[m] +
                         T(m) * ((m >= 1) ? rri[m - 1] : T(0)) * rrj[l + m];
            const T gj = T(l + m) * ((l + m >= 1) ? rrj[l + m - 1] : T(0)) * rri[m] +
                         T(m) * ((m >= 1) ? rrj[m - 1] : T(0)) * rri[l + m];
            e.fi += c * uu[k] * gi;
            e.fj += c * uu[k] * gj;
            if (MODE >= 2) {
              e.fuu += c * T(k * (k - 1)) * ((k >= 2) ? uu[k - 2] : T(0)) * st;
              e.fii += c * uu[k] *
                       (T((l + m) * (l + m - 1)) * ((l + m >= 2) ? rri[l + m - 2] : T(0)) * rrj[m] +
                        T(m * (m - 1)) * ((m >= 2) ? rri[m - 2] : T(0)) * rrj[l + m]);
              e.fjj += c * uu[k] *
                       (T((l + m) * (l + m - 1)) * ((l + m >= 2) ? rrj[l + m - 2] : T(0)) * rri[m] +
                        T(m * (m - 1)) * ((m >= 2) ? rrj[m - 2] : T(0)) * rri[l + m]);
              e.fui += c * T(k) * ukm * gi;
              e.fuj += c * T(k) * ukm * gj;
            }
          }
        }
      }
    }
  }
  return e;
}


// ---------------------------------------------------------------------------
// Folded e-e-n polynomial.  With x, y, z the switched scaled distances of
// electron i and j to one centre and of the pair, every e-e-n term is
//   c * z^k * (x^(l+m) y^m + x^m y^(l+m)),
// so for a fixed x the polynomial is  sum_k z^k sum_p B[k][p](x) y^p  with
//   B[k][m]   += c x^(l+m),   B[k][l+m] += c x^m.
// Only (k,p) with 1 <= p <= NORD-1 (k = 0) or 0 <= p <= NORD-k (k >= 1) can
// be non-zero; they are stored packed (18 of 30 entries at order 5).
// een_fold builds B and dB/dx once per (moved electron, centre); een_apply*
// then cost O(nB) per partner instead of O(nterms * NORD).  Same polynomial
// as jastrow4e / psinl, summed in a different order.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int een_pmin(int k) { return k == 0 ? 1 : 0; }
__host__ __device__ constexpr int een_pmax(int nord, int k) { return k == 0 ? nord - 1 : nord - k; }
__host__ __device__ constexpr int een_off(int nord, int k) {
  int o = 0;
  for (int kk = 0; kk < k; kk++) o += een_pmax(nord, kk) - een_pmin(kk) + 1;
  return o;
}
__host__ __device__ constexpr int een_nb(int nord) { return nord <= 1 ? 1 : een_off(nord, nord); }
// FP32 layout: every k group padded to an even number of (B, dB) pairs, so a
// group is read as 16-byte (B, dB, B', dB') quads; pads hold zeros
__host__ __device__ constexpr int een_lenp(int nord, int k) { return (een_pmax(nord, k) - een_pmin(k) + 2) / 2 * 2; }
__host__ __device__ constexpr int een_offp(int nord, int k) {
  int o = 0;
  for (int kk = 0; kk < k; kk++) o += een_lenp(nord, kk);
  return o;
}
__host__ __device__ constexpr int een_nbp(int nord) { return nord <= 1 ? 2 : een_offp(nord, nord); }

// B and dB/dx interleaved: BD[2*t] = B_t, BD[2*t+1] = dB_t (t = packed index,
// or with PAD the padded index of een_offp)
template <int NORD, typename T, bool PAD = false>
__device__ __forceinline__ void een_fold(const T *__restrict__ cc, T x, T *BD) {
  T xp[NORD + 1], dxp[NORD + 1];
  xp[0] = 1;
  dxp[0] = 0;
#pragma unroll
  for (int q = 1; q <= NORD; q++) {
    xp[q] = xp[q - 1] * x;
    dxp[q] = T(q) * xp[q - 1];
  }
  T B[een_nb(NORD)], dB[een_nb(NORD)];
#pragma unroll
  for (int t = 0; t < een_nb(NORD); t++) {
    B[t] = 0;
    dB[t] = 0;
  }
  int ll = 0;
#pragma unroll
  for (int n = 2; n <= NORD; n++) {
#pragma unroll
    for (int k = n - 1; k >= 0; k--) {
      const int l_hi = (k == 0) ? n - k - 2 : n - k;
#pragma unroll
      for (int l = l_hi; l >= 0; l--) {
        const int m = (n - k - l) / 2;
        if (2 * m == n - k - l) {
          const T c = cc[ll];
          ll++;
          const int t1 = een_off(NORD, k) + m - een_pmin(k);
          const int t2 = een_off(NORD, k) + l + m - een_pmin(k);
          B[t1] += c * xp[l + m];
          B[t2] += c * xp[m];
          dB[t1] += c * dxp[l + m];
          dB[t2] += c * dxp[m];
        }
      }
    }
  }
  if (PAD) {
#pragma unroll
    for (int k = 0; k < NORD; k++) {
#pragma unroll
      for (int q = 0; q < een_lenp(NORD, k); q++) {
        const bool real = q <= een_pmax(NORD, k) - een_pmin(k);
        const int t = real ? een_off(NORD, k) + q : 0;
        BD[2 * (een_offp(NORD, k) + q)] = real ? B[t] : T(0);
        BD[2 * (een_offp(NORD, k) + q) + 1] = real ? dB[t] : T(0);
      }
    }
  } else {
#pragma unroll
    for (int t = 0; t < een_nb(NORD); t++) {
      BD[2 * t] = B[t];
      BD[2 * t + 1] = dB[t];
    }
  }
}

// FP32 twin of een_apply1_multi<NORD, 1> (mixed-precision Jastrow): BD in the padded layout
// of een_fold<NORD, float, true>, 16-byte aligned; the y polynomial of each k
// group by Horner's rule with its derivative alongside
template <int NORD>
__device__ __forceinline__ void een_apply1f(const float *__restrict__ BD, float y, float z, float &fc, float &fu,
                                            float &fi, float &fj) {
  const float4 *bd = reinterpret_cast<const float4 *>(BD);
  fc = 0; fu = 0; fi = 0; fj = 0;
  // k descending: the z polynomial by Horner's rule, d/dz alongside
#pragma unroll
  for (int k = NORD - 1; k >= 0; k--) {
    const int pmin = een_pmin(k), pmax = een_pmax(NORD, k), off = een_offp(NORD, k);
    float4 v[een_lenp(NORD, 1) / 2];  // k = 1 is the longest group
#pragma unroll
    for (int q = 0; q < een_lenp(NORD, k); q += 2) v[q / 2] = bd[(off + q) / 2];
    // (B, dB) of power p: quad (p - pmin) / 2, half (p - pmin) % 2
#define EEN_B(p) (((p) - pmin) % 2 ? v[((p) - pmin) / 2].z : v[((p) - pmin) / 2].x)
#define EEN_D(p) (((p) - pmin) % 2 ? v[((p) - pmin) / 2].w : v[((p) - pmin) / 2].y)
    float a = EEN_B(pmax), ax = EEN_D(pmax), ay = 0;
#pragma unroll
    for (int p = pmax - 1; p >= pmin; p--) {
      ay = ay * y + a;
      a = a * y + EEN_B(p);
      ax = ax * y + EEN_D(p);
    }
#undef EEN_B
#undef EEN_D
    if (pmin == 1) {  // k = 0 has no y^0 term
      ay = ay * y + a;
      a *= y;
      ax *= y;
    }
    fu = fu * z + fc;
    fc = fc * z + a;
    fi = fi * z + ax;
    fj = fj * z + ay;
  }
}

// een_apply1f for P partners of one (moved electron, centre) at once: each
// (B, dB, B', dB') quad is loaded once for all of them
template <int NORD, int P>
__device__ __forceinline__ void een_apply1f_multi(const float *__restrict__ BD, const float (&y)[P], const float (&z)[P],
                                                  float (&fc)[P], float (&fu)[P], float (&fi)[P], float (&fj)[P]) {
  const float4 *bd = reinterpret_cast<const float4 *>(BD);
#pragma unroll
  for (int q = 0; q < P; q++) {
    fc[q] = 0; fu[q] = 0; fi[q] = 0; fj[q] = 0;
  }
#pragma unroll
  for (int k = NORD - 1; k >= 0; k--) {
    const int pmin = een_pmin(k), pmax = een_pmax(NORD, k), off = een_offp(NORD, k);
    float4 v[een_lenp(NORD, 1) / 2];
#pragma unroll
    for (int q = 0; q < een_lenp(NORD, k); q += 2) v[q / 2] = bd[(off + q) / 2];
#define EEN_B(p) (((p) - pmin) % 2 ? v[((p) - pmin) / 2].z : v[((p) - pmin) / 2].x)
#define EEN_D(p) (((p) - pmin) % 2 ? v[((p) - pmin) / 2].w : v[((p) - pmin) / 2].y)
    float a[P], ax[P], ay[P];
#pragma unroll
    for (int q = 0; q < P; q++) {
      a[q] = EEN_B(pmax);
      ax[q] = EEN_D(pmax);
      ay[q] = 0;
    }
#pragma unroll
    for (int p = pmax - 1; p >= pmin; p--) {
#pragma unroll
      for (int q = 0; q < P; q++) {
        ay[q] = ay[q] * y[q] + a[q];
        a[q] = a[q] * y[q] + EEN_B(p);
        ax[q] = ax[q] * y[q] + EEN_D(p);
      }
    }
#undef EEN_B
#undef EEN_D
    if (pmin == 1) {
#pragma unroll
      for (int q = 0; q < P; q++) {
        ay[q] = ay[q] * y[q] + a[q];
        a[q] *= y[q];
        ax[q] *= y[q];
      }
    }
#pragma unroll
    for (int q = 0; q < P; q++) {
      fu[q] = fu[q] * z[q] + fc[q];
      fc[q] = fc[q] * z[q] + a[q];
      fi[q] = fi[q] * z[q] + ax[q];
      fj[q] = fj[q] * z[q] + ay[q];
    }
  }
}

// value and first derivatives (d/dz, d/dx, d/dy) of the folded polynomial
// for P partners of one (moved electron, centre) at once: each
// (B, dB) pair is loaded once for all of them.  The y polynomial of every k
// group is evaluated by Horner's rule with its derivative alongside
// (a = a y + B_p, a' = a' y + a), so no power tables are held per partner.
template <int NORD, int P>
__device__ __forceinline__ void een_apply1_multi(const double *__restrict__ BD, const double (&y)[P],
                                                 const double (&z)[P], double (&fc)[P], double (&fu)[P],
                                                 double (&fi)[P], double (&fj)[P]) {
  const double2 *bd = reinterpret_cast<const double2 *>(BD);
#pragma unroll
  for (int q = 0; q < P; q++) {
    fc[q] = 0; fu[q] = 0; fi[q] = 0; fj[q] = 0;
  }
  // k descending: the z polynomial by Horner's rule, d/dz alongside
#pragma unroll
  for (int k = NORD - 1; k >= 0; k--) {
    const int pmin = een_pmin(k), pmax = een_pmax(NORD, k), off = een_off(NORD, k);
    double a[P], ax[P], ay[P];
    {
      const double2 v = bd[off + pmax - pmin];
#pragma unroll
      for (int q = 0; q < P; q++) {
        a[q] = v.x;
        ax[q] = v.y;
        ay[q] = 0;
      }
    }
#pragma unroll
    for (int p = pmax - 1; p >= pmin; p--) {
      const double2 v = bd[off + p - pmin];
#pragma unroll
      for (int q = 0; q < P; q++) {
        ay[q] = ay[q] * y[q] + a[q];
        a[q] = a[q] * y[q] + v.x;
        ax[q] = ax[q] * y[q] + v.y;
      }
    }
    if (pmin == 1) {  // k = 0 has no y^0 term: one more factor of y
#pragma unroll
      for (int q = 0; q < P; q++) {
        ay[q] = ay[q] * y[q] + a[q];
        a[q] *= y[q];
        ax[q] *= y[q];
      }
    }
#pragma unroll
    for (int q = 0; q < P; q++) {
      fu[q] = fu[q] * z[q] + fc[q];
      fc[q] = fc[q] * z[q] + a[q];
      fi[q] = fi[q] * z[q] + ax[q];
      fj[q] = fj[q] * z[q] + ay[q];
    }
  }
}

// value-only fold, packed B (padded to an even count for vector loads)
template <int NORD, typename T>
__device__ __forceinline__ void een_fold0(const T *__restrict__ cc, T x, T *Bout) {
  T xp[NORD + 1];
  xp[0] = 1;
#pragma unroll
  for (int q = 1; q <= NORD; q++) xp[q] = xp[q - 1] * x;
  T B[een_nb(NORD) + 1];
#pragma unroll
  for (int t = 0; t <= een_nb(NORD); t++) B[t] = 0;
  int ll = 0;
#pragma unroll
  for (int n = 2; n <= NORD; n++) {
#pragma unroll
    for (int k = n - 1; k >= 0; k--) {
      const int l_hi = (k == 0) ? n - k - 2 : n - k;
#pragma unroll
      for (int l = l_hi; l >= 0; l--) {
        const int m = (n - k - l) / 2;
        if (2 * m == n - k - l) {
          const T c = cc[ll];
          ll++;
          B[een_off(NORD, k) + m - een_pmin(k)] += c * xp[l + m];
          B[een_off(NORD, k) + l + m - een_pmin(k)] += c * xp[m];
        }
      }
    }
  }
#pragma unroll
  for (int t = 0; t < 2 * ((een_nb(NORD) + 1) / 2); t++) Bout[t] = B[t];
}

// FP32 twin of een_apply0 (mixed path): Bp 8-byte aligned
template <int NORD>
__device__ __forceinline__ float een_apply0f(const float *__restrict__ Bp, float y, float z) {
  constexpr int NB2 = (een_nb(NORD) + 1) / 2;
  float Bv[2 * NB2];
  const float2 *b2 = reinterpret_cast<const float2 *>(Bp);
#pragma unroll
  for (int t = 0; t < NB2; t++) {
    const float2 v = b2[t];
    Bv[2 * t] = v.x;
    Bv[2 * t + 1] = v.y;
  }
  // Horner's rule in y inside each k group and in z over the groups
  float fc = 0;
#pragma unroll
  for (int k = NORD - 1; k >= 0; k--) {
    const int pmin = een_pmin(k), pmax = een_pmax(NORD, k), off = een_off(NORD, k);
    float a = Bv[off + pmax - pmin];
#pragma unroll
    for (int p = pmax - 1; p >= pmin; p--) a = a * y + Bv[off + p - pmin];
    if (pmin == 1) a *= y;  // k = 0 has no y^0 term
    fc = fc * z + a;
  }
  return fc;
}

template <int NORD>
__device__ __forceinline__ double een_apply0(const double *__restrict__ Bp, double y, double z) {
  constexpr int NB2 = (een_nb(NORD) + 1) / 2;
  double Bv[2 * NB2];
  const double2 *b2 = reinterpret_cast<const double2 *>(Bp);
#pragma unroll
  for (int t = 0; t < NB2; t++) {
    const double2 v = b2[t];
    Bv[2 * t] = v.x;
    Bv[2 * t + 1] = v.y;
  }
  // Horner's rule in y inside each k group and in z over the groups
  double fc = 0;
#pragma unroll
  for (int k = NORD - 1; k >= 0; k--) {
    const int pmin = een_pmin(k), pmax = een_pmax(NORD, k), off = een_off(NORD, k);
    double a = Bv[off + pmax - pmin];
#pragma unroll
    for (int p = pmax - 1; p >= pmin; p--) a = a * y + Bv[off + p - pmin];
    if (pmin == 1) a *= y;  // k = 0 has no y^0 term
    fc = fc * z + a;
  }
  return fc;
}

// e-e-n term of one pair and centre with first and second derivatives (the
// full-Jastrow case of jastrow4.f90): per term only P = x^(l+m) y^m +
// x^m y^(l+m) and its x/y derivatives, scaled by the z factors of its k.
template <int NORD, typename T>
__device__ __forceinline__ EenOut<T> een_pair2(const T *__restrict__ cc, T z, T x, T y) {
  // only the power tables of x, y and z stay live; derivative factors are
  // compile-time constants of each unrolled term
  T xp[NORD + 1], yp[NORD + 1], zk[NORD];
  xp[0] = 1; yp[0] = 1; zk[0] = 1;
#pragma unroll
  for (int q = 1; q <= NORD; q++) {
    xp[q] = xp[q - 1] * x;
    yp[q] = yp[q - 1] * y;
  }
#pragma unroll
  for (int k = 1; k < NORD; k++) zk[k] = zk[k - 1] * z;
  EenOut<T> e{0, 0, 0, 0, 0, 0, 0, 0, 0};
  int ll = 0;
#pragma unroll
  for (int n = 2; n <= NORD; n++) {
#pragma unroll
    for (int k = n - 1; k >= 0; k--) {
      const int l_hi = (k == 0) ? n - k - 2 : n - k;
#pragma unroll
      for (int l = l_hi; l >= 0; l--) {
        const int m = (n - k - l) / 2;
        if (2 * m == n - k - l) {
          const T c = cc[ll];
          ll++;
          const int a = l + m, b = m;
          const T xa1 = a >= 1 ? T(a) * xp[a >= 1 ? a - 1 : 0] : T(0);
          const T xb1 = b >= 1 ? T(b) * xp[b >= 1 ? b - 1 : 0] : T(0);
          const T ya1 = a >= 1 ? T(a) * yp[a >= 1 ? a - 1 : 0] : T(0);
          const T yb1 = b >= 1 ? T(b) * yp[b >= 1 ? b - 1 : 0] : T(0);
          const T xa2 = a >= 2 ? T(a * (a - 1)) * xp[a >= 2 ? a - 2 : 0] : T(0);
          const T xb2 = b >= 2 ? T(b * (b - 1)) * xp[b >= 2 ? b - 2 : 0] : T(0);
          const T ya2 = a >= 2 ? T(a * (a - 1)) * yp[a >= 2 ? a - 2 : 0] : T(0);
          const T yb2 = b >= 2 ? T(b * (b - 1)) * yp[b >= 2 ? b - 2 : 0] : T(0);
          const T P = xp[a] * yp[b] + xp[b] * yp[a];
          const T Px = xa1 * yp[b] + xb1 * yp[a];
          const T Py = xp[a] * yb1 + xp[b] * ya1;
          const T Pxx = xa2 * yp[b] + xb2 * yp[a];
          const T Pyy = xp[a] * yb2 + xp[b] * ya2;
          const T cz = c * zk[k];
          const T cdz = k >= 1 ? c * T(k) * zk[k >= 1 ? k - 1 : 0] : T(0);
          const T cd2z = k >= 2 ? c * T(k * (k - 1)) * zk[k >= 2 ? k - 2 : 0] : T(0);
          e.fc += cz * P;
          e.fu += cdz * P;
          e.fuu += cd2z * P;
          e.fi += cz * Px;
          e.fii += cz * Pxx;
          e.fui += cdz * Px;
          e.fj += cz * Py;
          e.fjj += cz * Pyy;
          e.fuj += cdz * Py;
        }
      }
    }
  }
  return e;
}

// three of the four values of a 16-byte (float) / 32-byte (double) aligned
// quadruple, in vector loads
template <typename T>
__device__ __forceinline__ void ld3(const T *p, T &a, T &b, T &c);
template <>
__device__ __forceinline__ void ld3<float>(const float *p, float &a, float &b, float &c) {
  const float4 v = *reinterpret_cast<const float4 *>(p);
  a = v.x; b = v.y; c = v.z;
}
template <>
__device__ __forceinline__ void ld3<double>(const double *p, double &a, double &b, double &c) {
  const double2 v = *reinterpret_cast<const double2 *>(p);
  a = v.x; b = v.y;
  c = p[2];
}

// Fold with first and second x-derivatives: BD4[4*t .. 4*t+2] = B, dB, d2B
// (BD4[4*t+3] pads the quadruple for the vector loads of een_apply2)
template <int NORD, typename T>
__device__ __forceinline__ void een_fold2(const T *__restrict__ cc, T x, T *BD4) {
  T xp[NORD + 1];
  xp[0] = 1;
#pragma unroll
  for (int q = 1; q <= NORD; q++) xp[q] = xp[q - 1] * x;
  // one output entry at a time (gather form: every term's contributions to
  // entry t, in term order), so only three accumulators are live
#pragma unroll
  for (int t = 0; t < een_nb(NORD); t++) {
    T B = 0, dB = 0, d2B = 0;
    int ll = 0;
#pragma unroll
    for (int n = 2; n <= NORD; n++) {
#pragma unroll
      for (int k = n - 1; k >= 0; k--) {
        const int l_hi = (k == 0) ? n - k - 2 : n - k;
#pragma unroll
        for (int l = l_hi; l >= 0; l--) {
          const int m = (n - k - l) / 2;
          if (2 * m == n - k - l) {
            const int a = l + m, b = m;
            const int t1 = een_off(NORD, k) + b - een_pmin(k);   // y^m   gets c x^(l+m)
            const int t2 = een_off(NORD, k) + a - een_pmin(k);   // y^(l+m) gets c x^m
            if (t1 == t || t2 == t) {
              const T c = cc[ll];
              if (t1 == t) {
                B += c * xp[a];
                if (a >= 1) dB += c * T(a) * xp[a >= 1 ? a - 1 : 0];
                if (a >= 2) d2B += c * T(a * (a - 1)) * xp[a >= 2 ? a - 2 : 0];
              }
              if (t2 == t) {
                B += c * xp[b];
                if (b >= 1) dB += c * T(b) * xp[b >= 1 ? b - 1 : 0];
                if (b >= 2) d2B += c * T(b * (b - 1)) * xp[b >= 2 ? b - 2 : 0];
              }
            }
            ll++;
          }
        }
      }
    }
    BD4[4 * t] = B;
    BD4[4 * t + 1] = dB;
    BD4[4 * t + 2] = d2B;
    BD4[4 * t + 3] = T(0);
  }
}

// all nine value/derivative sums of the e-e-n term (jastrow4.f90 fc, fu,
// fuu, fi, fii, fj, fjj, fui, fuj) from the folded row coefficients.  The y
// polynomial of every k group by Horner's rule with its first derivative and
// half its second derivative carried alongside (h = h y + a', a' = a' y + a,
// a = a y + B_p); the z polynomial over the groups the same way (k
// descending); fuu and fjj doubled once at the end.
template <int NORD, typename T = double>
__device__ __forceinline__ EenOut<T> een_apply2(const T *__restrict__ BD4, T y, T z) {
  EenOut<T> e{0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = NORD - 1; k >= 0; k--) {
    const int pmin = een_pmin(k), pmax = een_pmax(NORD, k), off = een_off(NORD, k);
    T a, ax, axx, ay = 0, ayy = 0;  // ayy: half the second derivative
    ld3<T>(BD4 + 4 * (off + pmax - pmin), a, ax, axx);
#pragma unroll
    for (int p = pmax - 1; p >= pmin; p--) {
      T b0, b1, b2;
      ld3<T>(BD4 + 4 * (off + p - pmin), b0, b1, b2);
      ayy = ayy * y + ay;
      ay = ay * y + a;
      a = a * y + b0;
      ax = ax * y + b1;
      axx = axx * y + b2;
    }
    if (pmin == 1) {  // k = 0 has no y^0 term
      ayy = ayy * y + ay;
      ay = ay * y + a;
      a *= y;
      ax *= y;
      axx *= y;
    }
    e.fuu = e.fuu * z + e.fu;
    e.fu = e.fu * z + e.fc;
    e.fc = e.fc * z + a;
    e.fui = e.fui * z + e.fi;
    e.fi = e.fi * z + ax;
    e.fii = e.fii * z + axx;
    e.fuj = e.fuj * z + e.fj;
    e.fj = e.fj * z + ay;
    e.fjj = e.fjj * z + ayy;
  }
  e.fuu *= T(2);
  e.fjj *= T(2);
  return e;
}

// e-e-n coefficients of atom type it in the compute precision
template <typename T>
__device__ __forceinline__ const T *een_coef(const CSys &cs, int it);
template <>
__device__ __forceinline__ const double *een_coef<double>(const CSys &cs, int it) { return &cs.c[it * CW_MAX_TERMS]; }
template <>
__device__ __forceinline__ const float *een_coef<float>(const CSys &cs, int it) { return &cs.cf[it * CW_MAX_TERMS]; }

// Padé + polynomial e-e term (jastrow4.f90 ee part) at scaled u:
// returns fee, d fee/du, d2 fee/du2 (MODE>=2)
template <int MODE, typename T>
__device__ __forceinline__ void ee_term(const CSys &cs, int isb, int ipar, T sspinn, T u, T &fee, T &feeu, T &feeuu) {
  const int nb = cs.nordb + 1;
  T b0 = (T)cs.b[isb * nb + 0], b1 = (T)cs.b[isb * nb + 1];
  T top = sspinn * b0 * u, topu = sspinn * b0;
  T bot = T(1) + b1 * u, botu = b1, bot2 = bot * bot;
  fee = top / bot - (T)cs.asymp_jasb[ipar];
  feeu = topu / bot - botu * top / bot2;
  if (MODE >= 2) feeuu = (-(T(2) * botu * topu) / bot + T(2) * botu * botu * top / bot2) / bot;
  T up = u;  // u^(iord-1)
  T upm = 1; // u^(iord-2)
  for (int iord = 2; iord <= cs.nordb; iord++) {
    T bc = (T)cs.b[isb * nb + iord];
    T uord = up * u;
    fee += bc * uord;
    feeu += bc * T(iord) * up;
    if (MODE >= 2) feeuu += bc * T(iord * (iord - 1)) * upm;
    upm = up;
    up = uord;
  }
}

// Padé + polynomial e-n term (jastrow4.f90 en part) at scaled r
template <int MODE, typename T>
__device__ __forceinline__ void en_term(const CSys &cs, int it, T r, T &fen, T &feni, T &fenii) {
  const int na = cs.norda + 1;
  T a0 = (T)cs.a4[it * na + 0], a1 = (T)cs.a4[it * na + 1];
  T top = a0 * r, topi = a0;
  T bot = T(1) + a1 * r, boti = a1, bot2 = bot * bot;
  fen = top / bot - (T)cs.asymp_jasa[it];
  feni = topi / bot - boti * top / bot2;
  if (MODE >= 2) fenii = (-(T(2) * boti * topi) / bot + T(2) * boti * boti * top / bot2) / bot;
  T rp = r, rpm = 1;
  for (int iord = 2; iord <= cs.norda; iord++) {
    T ac = (T)cs.a4[it * na + iord];
    T rord = rp * r;
    fen += ac * rord;
    feni += ac * T(iord) * rp;
    if (MODE >= 2) fenii += ac * T(iord * (iord - 1)) * rpm;
    rpm = rp;
    rp = rord;
  }
}

// Slm (vmc/slm.f90): monomial exponents and constants of index l (1-based).
__device__ __forceinline__ void slm_def(int l, int &a, int &b, int &c, double &k) {
  const double CS_ = 0.28209479177387814, CP_ = 0.48860251190291992, CD1 = 0.630783130505040,
               CD2 = 1.092548430592079, CF_ = 0.74635266518023078, CF2 = 1.66889529453113635,
               CF3 = 2.89061144264055405, CG_ = 0.8462843753216345, CG2 = 2.2390579955406924,
               CG3 = 2.890611442640554, CG4 = 5.006685883593409;
  switch (l) {
    case 1: a = 0; b = 0; c = 0; k = CS_; break;
    case 2: a = 1; b = 0; c = 0; k = CP_; break;
    case 3: a = 0; b = 1; c = 0; k = CP_; break;
    case 4: a = 0; b = 0; c = 1; k = CP_; break;
    case 5: a = 2; b = 0; c = 0; k = CD1; break;
    case 6: a = 1; b = 1; c = 0; k = CD2; break;
    case 7: a = 1; b = 0; c = 1; k = CD2; break;
    case 8: a = 0; b = 2; c = 0; k = CD1; break;
    case 9: a = 0; b = 1; c = 1; k = CD2; break;
    case 10: a = 0; b = 0; c = 2; k = CD1; break;
    case 11: a = 3; b = 0; c = 0; k = CF_; break;
    case 12: a = 2; b = 1; c = 0; k = CF2; break;
    case 13: a = 2; b = 0; c = 1; k = CF2; break;
    case 14: a = 1; b = 2; c = 0; k = CF2; break;
    case 15: a = 1; b = 1; c = 1; k = CF3; break;
    case 16: a = 1; b = 0; c = 2; k = CF2; break;
    case 17: a = 0; b = 3; c = 0; k = CF_; break;
    case 18: a = 0; b = 2; c = 1; k = CF2; break;
    case 19: a = 0; b = 1; c = 2; k = CF2; break;
    case 20: a = 0; b = 0; c = 3; k = CF_; break;
    case 21: a = 4; b = 0; c = 0; k = CG_; break;
    case 22: a = 3; b = 1; c = 0; k = CG2; break;
    case 23: a = 3; b = 0; c = 1; k = CG2; break;
    case 24: a = 2; b = 2; c = 0; k = CG3; break;
    case 25: a = 2; b = 1; c = 1; k = CG4; break;
    case 26: a = 2; b = 0; c = 2; k = CG3; break;
    case 27: a = 1; b = 3; c = 0; k = CG2; break;
    case 28: a = 1; b = 2; c = 1; k = CG4; break;
    case 29: a = 1; b = 1; c = 2; k = CG4; break;
    case 30: a = 1; b = 0; c = 3; k = CG2; break;
    case 31: a = 0; b = 4; c = 0; k = CG_; break;
    case 32: a = 0; b = 3; c = 1; k = CG2; break;
    case 33: a = 0; b = 2; c = 2; k = CG3; break;
    case 34: a = 0; b = 1; c = 3; k = CG2; break;
    default: a = 0; b = 0; c = 4; k = CG_; break;
  }
}
__device__ __forceinline__ double ipw(double x, int n) {
  double r = 1;
  for (int i = 0; i < n; i++) r *= x;
  return r;
}
__device__ __forceinline__ void slm_eval(int l, double x, double y, double z, double &v, double *dv, double &lap) {
  int a, b, c;
  double k;
  slm_def(l, a, b, c, k);
  double px = ipw(x, a), py = ipw(y, b), pz = ipw(z, c);
  v = k * px * py * pz;
  dv[0] = a ? k * a * ipw(x, a - 1) * py * pz : 0.0;
  dv[1] = b ? k * b * px * ipw(y, b - 1) * pz : 0.0;
  dv[2] = c ? k * c * px * py * ipw(z, c - 1) : 0.0;
  lap = 0;
  if (a >= 2) lap += k * a * (a - 1) * ipw(x, a - 2) * py * pz;
  if (b >= 2) lap += k * b * (b - 1) * px * ipw(y, b - 2) * pz;
  if (c >= 2) lap += k * c * (c - 1) * px * py * ipw(z, c - 2);
}

// basis_fns + phi_combine for one centre: writes the AOs of centre ic at
// displacement xc (= x - cent).  out(m, d) receives value (d=0), gradient
// (d=1..3, ider>=1) and Laplacian (d=4, ider>=2).
template <typename Store>
__device__ __forceinline__ void basis_centre(const CSys &cs, const GSys &g, int ic, const double *xc, int ider, Store out) {
  // basis_fns + splfit (vmc/splfit.f90:3-94) for every radial function of
  // the centre.  The grid interval (jx, ref0, ref1) depends only on r and
  // the atom type, so it is located once per centre; r0*arg^(jx-1) comes
  // from a per-type table instead of pow().  Radial functions are then
  // evaluated one at a time and combined with every AO that uses them
  // (iwrwf), so no per-thread array of spline values is needed.
  const int it = cs.iwctype[ic];
  const double r = sqrt(xc[0] * xc[0] + xc[1] * xc[1] + xc[2] * xc[2]);
  const double ri = 1.0 / r;
  const int nrb = cs.nrbas[it];
  const int nbt = cs.nbastyp[it];
  const int m0 = cs.ao_first[ic];
  const double xcri[3] = {xc[0] * ri, xc[1] * ri, xc[2] * ri};
  const int *iwl = g.iwlbas + it * cs.mbastyp;
  const int *iwr = g.iwrwf + it * cs.mbastyp;
  // grid location (splfit :33-55)
  const int ig = cs.igrid[it];
  const double arg = cs.arg[it], r0 = cs.r0[it];
  const double *gp = g.gridpow + (size_t)it * (cs.mpts + 1);
  double xr, ref0 = 0, ref1 = 0, delh = 1;
  int jx;
  if (ig == 1) {
    xr = (r - r0) / arg + 1;
    jx = (int)xr;
    ref0 = r0 + arg * (jx - 1);
    ref1 = ref0 + arg;
    delh = arg;
  } else if (ig == 2) {
    xr = (log(r) - log(r0)) / log(arg) + 1;
    jx = (int)xr;
    if (jx >= 1 && jx <= cs.mpts) {
      ref0 = __ldg(gp + jx);
      ref1 = ref0 * arg;
      delh = ref1 - ref0;
    }
  } else {
    xr = (log((r + r0) / r0)) / log(arg) + 1.0;
    jx = (int)xr;
    if (jx >= 1 && jx <= cs.mpts) {
      ref0 = __ldg(gp + jx) - r0;
      ref1 = (ref0 + r0) * arg - r0;
      delh = ref1 - ref0;
    }
  }
  const int spline = (jx >= 1 && jx < cs.nr[it]);
  const double sixth = 1.0 / 6.0;
  const double delhi = 1.0 / delh;
  const double bb = (r - ref0) * delhi;
  const double aa = (ref1 - r) * delhi;
  const double cc = aa * (aa * aa - 1.0) * delh * delh * sixth;
  const double dd = bb * (bb * bb - 1.0) * delh * delh * sixth;
  const double t1 = (3.0 * aa * aa - 1.0) * delh * sixth, t2 = (3.0 * bb * bb - 1.0) * delh * sixth;
  for (int irb = 0; irb < nrb; irb++) {
    double w[4];
    if (r <= cs.rmaxwf[it * CW_MAX_RWF + irb]) {
      if (spline) {
        const size_t tb = (size_t)(irb + cs.mrwf * it) * cs.mpts;
        const double y0 = __ldg(g.rwf + tb + jx - 1), y1 = __ldg(g.rwf + tb + jx);
        const double d0 = __ldg(g.d2rwf + tb + jx - 1), d1 = __ldg(g.d2rwf + tb + jx);
        w[0] = aa * y0 + bb * y1 + cc * d0 + dd * d1;
        w[1] = (y1 - y0) * delhi + (-t1 * d0 + t2 * d1);
        w[2] = aa * d0 + bb * d1;
        w[3] = (-d0 + d1) * delhi;
      } else if (jx < 1) {
        const double *ce = &cs.ce[(it * CW_MAX_RWF + irb) * 5];
        const double rpow[5] = {1.0, r, r * r, r * r * r, r * r * r * r};
        double v = ce[0];
        for (int ii = 2; ii <= 5; ii++) v += ce[ii - 1] * rpow[ii - 1];
        w[0] = v;
        double p1 = 0, p2 = 0, p3 = 0;
        for (int ii = 2; ii <= 5; ii++) {
          const double c = ce[ii - 1];
          p1 += (ii - 1) * c * rpow[ii - 2];
          if (ii >= 3) p2 += (ii - 1) * (ii - 2) * c * rpow[ii - 3];
          if (ii >= 4) p3 += (ii - 1) * (ii - 2) * (ii - 3) * c * rpow[ii - 4];
        }
        w[1] = p1; w[2] = p2; w[3] = p3;
      } else {
        const double *ae = &cs.ae[(it * CW_MAX_RWF + irb) * 2];
        w[0] = ae[0] * exp(-ae[1] * r);
        w[1] = -ae[1] * w[0];
        w[2] = -ae[1] * w[1];
        w[3] = -ae[1] * w[2];
      }
    } else {
      w[0] = w[1] = w[2] = w[3] = 0.0;
    }
    for (int ib = 0; ib < nbt; ib++) {
      if (__ldg(iwr + ib) - 1 != irb) continue;
      const int l = __ldg(iwl + ib);
      double y, dy[3], lap;
      slm_eval(l, xc[0], xc[1], xc[2], y, dy, lap);
      out(m0 + ib, 0, y * w[0]);
      if (ider >= 1) {
        double dum = 0;
        for (int jj = 0; jj < 3; jj++) {
          out(m0 + ib, 1 + jj, y * xcri[jj] * w[1] + dy[jj] * w[0]);
          dum += dy[jj] * xcri[jj];
        }
        if (ider >= 2) {
          double d2 = y * w[2] + y * 2.0 * ri * w[1] + lap * w[0];
          d2 += 2.0 * dum * w[1];
          out(m0 + ib, 4, d2);
        }
      }
    }
  }
}


// ---------------------------------------------------------------------------
// Warp-cooperative basis evaluation of one point for all K AOs.
// Lanes first stage per-centre data (displacement, powers, spline interval
// and weights) in shared memory, then run over AOs: every lane follows the
// same code (table-driven Slm monomials), and consecutive lanes write
// consecutive AOs.  Same arithmetic as basis_centre/splfit.
// ---------------------------------------------------------------------------
constexpr int kCenRec = 28;  // doubles per centre record

template <int IDER>
__device__ __forceinline__ void warp_basis_prepass(const CSys &cs, const GSys &g, const double *x, double *rec, int lane) {
  for (int ic = lane; ic < cs.M; ic += 32) {
    double *q = rec + (size_t)ic * kCenRec;
    const Cen cc = cen_of(g, ic);
    const int it = cc.it;
    const double xc0 = x[0] - cc.x, xc1 = x[1] - cc.y, xc2 = x[2] - cc.z;
    const double r = sqrt(xc0 * xc0 + xc1 * xc1 + xc2 * xc2);
    const double ri = 1.0 / r;
    const int ig = cs.igrid[it];
    const double arg = cs.arg[it], r0 = cs.r0[it];
    const double *gp = g.gridpow + (size_t)it * (cs.mpts + 1);
    double xr, ref0 = 0, ref1 = 0, delh = 1;
    int jx;
    if (ig == 1) {
      xr = (r - r0) / arg + 1;
      jx = (int)xr;
      ref0 = r0 + arg * (jx - 1);
      ref1 = ref0 + arg;
      delh = arg;
    } else if (ig == 2) {
      xr = (log(r) - log(r0)) / log(arg) + 1;
      jx = (int)xr;
      if (jx >= 1 && jx <= cs.mpts) {
        ref0 = __ldg(gp + jx);
        ref1 = ref0 * arg;
        delh = ref1 - ref0;
      }
    } else {
      xr = (log((r + r0) / r0)) / log(arg) + 1.0;
      jx = (int)xr;
      if (jx >= 1 && jx <= cs.mpts) {
        ref0 = __ldg(gp + jx) - r0;
        ref1 = (ref0 + r0) * arg - r0;
        delh = ref1 - ref0;
      }
    }
    const double sixth = 1.0 / 6.0, delhi = 1.0 / delh;
    const double bb = (r - ref0) * delhi, aa = (ref1 - r) * delhi;
    q[0] = xc0; q[1] = xc1; q[2] = xc2; q[3] = r; q[4] = ri;
    q[5] = (double)jx;
    q[6] = aa; q[7] = bb;
    q[8] = aa * (aa * aa - 1.0) * delh * delh * sixth;
    q[9] = bb * (bb * bb - 1.0) * delh * delh * sixth;
    q[10] = (3.0 * aa * aa - 1.0) * delh * sixth;
    q[11] = (3.0 * bb * bb - 1.0) * delh * sixth;
    q[12] = delhi;
    double px = 1, py = 1, pz = 1;
#pragma unroll
    for (int p = 0; p < 5; p++) {
      q[13 + p] = px; q[18 + p] = py; q[23 + p] = pz;
      px *= xc0; py *= xc1; pz *= xc2;
    }
  }
}

// value (d=0), gradient (d=1..3, IDER>=1), Laplacian (d=4, IDER>=2) of AO m
template <int IDER, typename Store>
__device__ __forceinline__ void warp_basis_ao(const CSys &cs, const GSys &g, const double *rec, int m, Store out) {
  const int4 a4 = __ldg(g.ao + m);
  const int4 ax = __ldg(g.aox + m);
  const double2 ak = __ldg(g.aok + m);
  const int ic = a4.x, irb = a4.y, it = a4.z;
  const double *q = rec + (size_t)ic * kCenRec;
  const double r = q[3], ri = q[4];
  const int jx = (int)q[5];
  double w0 = 0, w1 = 0, w2 = 0;
  if (r <= ak.y) {
    if (jx >= 1 && jx < ax.y) {
      const size_t tb = (size_t)ax.x;
      const double y0 = __ldg(g.rwf + tb + jx - 1), y1 = __ldg(g.rwf + tb + jx);
      const double d0 = __ldg(g.d2rwf + tb + jx - 1), d1 = __ldg(g.d2rwf + tb + jx);
      w0 = q[6] * y0 + q[7] * y1 + q[8] * d0 + q[9] * d1;
      w1 = (y1 - y0) * q[12] + (-q[10] * d0 + q[11] * d1);
      w2 = q[6] * d0 + q[7] * d1;
    } else if (jx < 1) {
      const double *ce = &cs.ce[(it * CW_MAX_RWF + irb) * 5];
      const double rpow[5] = {1.0, r, r * r, r * r * r, r * r * r * r};
      w0 = ce[0];
      for (int ii = 2; ii <= 5; ii++) w0 += ce[ii - 1] * rpow[ii - 1];
      for (int ii = 2; ii <= 5; ii++) {
        const double c = ce[ii - 1];
        w1 += (ii - 1) * c * rpow[ii - 2];
        if (ii >= 3) w2 += (ii - 1) * (ii - 2) * c * rpow[ii - 3];
      }
    } else {
      const double *ae = &cs.ae[(it * CW_MAX_RWF + irb) * 2];
      w0 = ae[0] * exp(-ae[1] * r);
      w1 = -ae[1] * w0;
      w2 = -ae[1] * w1;
    }
  }
  const int ea = ax.z & 255, eb = (ax.z >> 8) & 255, ec = ax.z >> 16;
  const double k = ak.x;
  const double *X = q + 13, *Y = q + 18, *Z = q + 23;
  const double y = k * X[ea] * Y[eb] * Z[ec];
  out(m, 0, y * w0);
  if (IDER >= 1) {
    const double dy0 = ea ? k * ea * X[ea - 1] * Y[eb] * Z[ec] : 0.0;
    const double dy1 = eb ? k * eb * X[ea] * Y[eb - 1] * Z[ec] : 0.0;
    const double dy2 = ec ? k * ec * X[ea] * Y[eb] * Z[ec - 1] : 0.0;
    const double xr0 = q[0] * ri, xr1 = q[1] * ri, xr2 = q[2] * ri;
    out(m, 1, y * xr0 * w1 + dy0 * w0);
    out(m, 2, y * xr1 * w1 + dy1 * w0);
    out(m, 3, y * xr2 * w1 + dy2 * w0);
    if (IDER >= 2) {
      double lap = 0;
      if (ea >= 2) lap += k * ea * (ea - 1) * X[ea - 2] * Y[eb] * Z[ec];
      if (eb >= 2) lap += k * eb * (eb - 1) * X[ea] * Y[eb - 2] * Z[ec];
      if (ec >= 2) lap += k * ec * (ec - 1) * X[ea] * Y[eb] * Z[ec - 2];
      const double dum = dy0 * xr0 + dy1 * xr1 + dy2 * xr2;
      double d2 = y * w2 + y * 2.0 * ri * w1 + lap * w0;
      d2 += 2.0 * dum * w1;
      out(m, 4, d2);
    }
  }
}

// gauss_pot (vmc/readps_gauss.f90:57): channel l is CHAMP's 1-based index
__device__ __forceinline__ double gauss_pot_d(const CSys &cs, double r, int l, int ict) {
  double v = 0, rsq = r * r;
  const int base = (ict * 4 + (l - 1)) * 16;
  const int nt = cs.necp_term[ict * 4 + (l - 1)];
  for (int i = 0; i < nt; i++) {
    int pw = cs.necp_power[base + i];
    double p = (pw != 2) ? pow(r, (double)(pw - 2)) : 1.0;
    double ex = cs.ecp_exponent[base + i];
    double e = (ex * rsq > 7.0e2) ? 0.0 : cs.ecp_coef[base + i] * exp(-ex * rsq);
    v += p * e;
  }
  return v;
}

__device__ __forceinline__ double yl0_d(int l, double costh) {
  if (l == 1) return 1.0;
  if (l == 2) return 3.0 * costh;
  if (l == 3) return 2.5 * (3 * costh * costh - 1);
  return 3.5 * (5 * costh * costh * costh - 3 * costh);
}

// pair spin classification of jastrow4 (isb, ipar, sspinn) for i > j
__device__ __forceinline__ void pair_spin(const CSys &cs, int i, int j, int &isb, int &ipar, double &sspinn) {
  sspinn = 1;
  isb = 0;
  ipar = 0;
  if (i < cs.nup || j >= cs.nup) {
    if (cs.nspin2b == 2) isb = 1;
    else if (cs.nocuspb == 0) sspinn = 0.5;
    ipar = 1;
  }
}
