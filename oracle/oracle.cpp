// oracle.cpp — CPU FP64 restatement of CHAMP's VMC hot path.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).  Arrays keep CHAMP's Fortran
// column-major layout with 0-based indices; the index helpers below spell out
// the Fortran subscript each one stands for.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

namespace {

using std::vector;

// ---------------------------------------------------------------------------
// xoshiro256** — restates vmc/xoroshiro256starstar.c:22-65 (next, jump) and
// :125 (next_uniform_double).
// ---------------------------------------------------------------------------
struct Rng {
  uint64_t s[4];
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t result = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
  void jump() {
    static const uint64_t J[] = {0x180ec6d33cfd0abaULL, 0xd5a61266f0c9392cULL,
                                 0xa9582618e03fc9aaULL, 0x39abdc4529b1661cULL};
    uint64_t s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int i = 0; i < 4; i++)
      for (int b = 0; b < 64; b++) {
        if (J[i] & (1ULL << b)) {
          s0 ^= s[0]; s1 ^= s[1]; s2 ^= s[2]; s3 ^= s[3];
        }
        next();
      }
    s[0] = s0; s[1] = s1; s[2] = s2; s[3] = s3;
  }
};

const double PI = 4.0 * std::atan(1.0);  // module constants, m_constant.f90:52

// ---------------------------------------------------------------------------
// System: copies of the module arrays plus the derived Jastrow asymptotes.
// ---------------------------------------------------------------------------
struct Sys {
  int N, nup, ndn, M, nctype;
  vector<int> iwctype;
  vector<double> cent, znuc;
  double pecent;
  int mrwf, mpts;
  vector<int> nrbas, igrid, nr;
  vector<double> arg, r0, rwf, d2rwf, ce, ae, rmaxwf;
  int mbastyp;
  vector<int> nbastyp, iwlbas, iwrwf;
  int K, O, ndet;
  vector<double> coef, cdet;   // cdet: sign-adjusted by multideterminants_define
  int nstates = 1;             // CI vectors sharing orbitals and Jastrow (csfs nstates)
  int iguiding = 0;            // > 0: sample the guiding function (mstates_ctrl)
  vector<double> weights_g;    // [nstates] (mstates3; anormo = 1)
  vector<double> cdet_st;      // [nstates][ndet], sign-adjusted like cdet; row 0 = cdet
  vector<double> detsign;      // [ndet] +-1: orbital-order sign folded into cdet
  vector<int> iworbd;  // iworbd(j) for kref=1, 1-based orbital
  vector<int> iworbd_all;      // [ndet][N] 1-based, reordered as multideterminants_define does
  // compact multideterminant tables per spin (multideterminants_define,
  // vmc/set_input_data.f90:46), all indices 0-based, kref = determinant 0
  struct MdSpin {
    int ivirt = 0, iactv = 0;          // first virtual orbital, first active slot
    int nuniq = 0, nsingle = 0, ndouble = 0;
    vector<int> numrep;                // [nuniq]
    vector<int> irepcol, ireporb;      // [nuniq][MEXCIT] replaced slot / new orbital
    vector<int> kdet2, kaux2;          // full determinants not kref-equivalent and their unique index
  } md[2];
  int norda, nordb, nordc, isc, nspin2b, nocuspb, nterms;
  double scalek;
  vector<double> a4, b, c;
  double asymp_r;
  vector<double> asymp_jasa;  // [nctype]
  double asymp_jasb[2];
  int nloc;
  vector<int> lpot, necp_term, necp_power;
  vector<double> ecp_exponent, ecp_coef;
  int nquad;
  vector<double> xq0, yq0, zq0, wq;
  double deltar, deltat, fbias;
  // index helpers
  double RWF(int ir, int irb, int it) const { return rwf[ir + mpts * (irb + mrwf * it)]; }
  double D2RWF(int ir, int irb, int it) const { return d2rwf[ir + mpts * (irb + mrwf * it)]; }
  double CE(int ii, int irb, int it) const { return ce[ii + CW_NCOEF * (irb + mrwf * it)]; }
  double AE(int ii, int irb, int it) const { return ae[ii + 2 * (irb + mrwf * it)]; }
  double COEF(int m, int iorb) const { return coef[m + K * iorb]; }
  double A4(int ip, int it) const { return a4[ip + (norda + 1) * it]; }   // a4(ip+1,it)
  double B(int ip, int isb) const { return b[ip + (nordb + 1) * isb]; }    // b(ip+1,isb)
  double C(int ll, int it) const { return c[ll + nterms * it]; }           // c(ll+1,it)
};

int nterms4(int nord) {
  // nterms4 (vmc/jastrow4.f90): same enumeration as the e-e-n loops.
  int i = 0;
  for (int n = 2; n <= nord; n++)
    for (int k = n - 1; k >= 0; k--) {
      int l_hi = (k == 0) ? n - k - 2 : n - k;
      for (int l = l_hi; l >= 0; l--) {
        int m = (n - k - l) / 2;
        if (2 * m == n - k - l) i++;
      }
    }
  return i;
}

constexpr int MEXCIT = 10;  // vmc_mod MEXCIT (module/m_vmc.f90:99)

// multideterminants_define (vmc/set_input_data.f90:46-414) with kref = 1:
// per spin, the excitation of every determinant relative to kref (replaced
// reference slots irepcol in slot order, new orbitals ireporb in the
// determinant's order), the permutation sign folded into cdet, the unique
// spin-determinants (first occurrence of each excitation) ordered singles,
// doubles, then the rest, and the (determinant, unique index) lists of the
// determinants whose spin part differs from kref.  The reference reorders
// the unique list by pairwise swaps; a stable partition is used here, which
// changes only the summation order of the Y-matrix accumulation.
bool multideterminants_define(Sys &s) {
  const int N = s.N, nd = s.ndet;
  vector<int> numrep((size_t)nd * 2, 0), irc((size_t)nd * 2 * N, 0), iro((size_t)nd * 2 * N, 0);
  vector<int> itot(nd, 0);
  auto IW = [&](int k, int i) -> int & { return s.iworbd_all[(size_t)k * N + i]; };
  for (int k = 1; k < nd; k++) {
    for (int iab = 0; iab < 2; iab++) {
      const int nel = iab == 0 ? s.nup : s.ndn, ish = iab == 0 ? 0 : s.nup;
      int &nr = numrep[k * 2 + iab];
      nr = 0;
      for (int iref = 0; iref < nel; iref++) {
        const int iwref = IW(0, iref + ish);
        bool in = false;
        for (int i = 0; i < nel; i++)
          if (IW(k, i + ish) == iwref) in = true;
        if (!in) irc[((size_t)k * 2 + iab) * N + nr++] = iref;
      }
      int isub = 0;
      for (int i = 0; i < nel; i++) {
        const int iw = IW(k, i + ish);
        bool in = false;
        for (int iref = 0; iref < nel; iref++)
          if (iw == IW(0, iref + ish)) in = true;
        if (!in) iro[((size_t)k * 2 + iab) * N + isub++] = iw - 1;
      }
      if (isub != nr) return false;
      vector<int> sw(nel);
      for (int i = 0; i < nel; i++) sw[i] = IW(0, i + ish);
      for (int r = 0; r < nr; r++) sw[irc[((size_t)k * 2 + iab) * N + r]] = iro[((size_t)k * 2 + iab) * N + r] + 1;
      int iphase = 0;
      for (int i = 0; i < nel; i++) {
        if (IW(k, i + ish) != sw[i]) {
          for (int l = i + 1; l < nel; l++) {
            if (sw[l] == IW(k, i + ish)) {
              std::swap(sw[i], sw[l]);
              iphase++;
            }
          }
        }
      }
      itot[k] += iphase;
    }
    if (itot[k] % 2) {
      s.detsign[k] = -1.0;
      s.cdet[k] = -s.cdet[k];
      for (int st = 0; st < s.nstates; st++) s.cdet_st[(size_t)st * nd + k] = -s.cdet_st[(size_t)st * nd + k];
    }
  }
  for (int k = 1; k < nd; k++) {
    for (int i = 0; i < N; i++) IW(k, i) = IW(0, i);
    for (int iab = 0; iab < 2; iab++) {
      const int ish = iab == 0 ? 0 : s.nup;
      for (int r = 0; r < numrep[k * 2 + iab]; r++)
        IW(k, irc[((size_t)k * 2 + iab) * N + r] + ish) = iro[((size_t)k * 2 + iab) * N + r] + 1;
    }
  }
  for (int iab = 0; iab < 2; iab++) {
    Sys::MdSpin &m = s.md[iab];
    const int nel = iab == 0 ? s.nup : s.ndn;
    m = Sys::MdSpin();
    m.iactv = nel;
    m.ivirt = s.nup;  // ivirt(1)=nup+1 and ivirt(2)=ndn+1 in CHAMP's 1-based numbering
    if (iab == 1) m.ivirt = s.ndn;
    for (int k = 1; k < nd; k++)
      for (int r = 0; r < numrep[k * 2 + iab]; r++) {
        m.iactv = std::min(m.iactv, irc[((size_t)k * 2 + iab) * N + r]);
        m.ivirt = std::min(m.ivirt, iro[((size_t)k * 2 + iab) * N + r]);
      }
    auto same = [&](int a, int b) {
      if (numrep[a * 2 + iab] != numrep[b * 2 + iab]) return false;
      for (int r = 0; r < numrep[a * 2 + iab]; r++) {
        if (irc[((size_t)a * 2 + iab) * N + r] != irc[((size_t)b * 2 + iab) * N + r]) return false;
        if (iro[((size_t)a * 2 + iab) * N + r] != iro[((size_t)b * 2 + iab) * N + r]) return false;
      }
      return true;
    };
    // iwundet: kref if no excitation, else the first determinant with the same excitation
    vector<int> iwun(nd, 0);
    for (int i = 1; i < nd; i++) {
      if (numrep[i * 2 + iab] == 0) { iwun[i] = 0; continue; }
      int j = 0;
      while (j != i && !same(j, i)) j++;
      iwun[i] = j;
    }
    vector<int> uniq;
    for (int k = 1; k < nd; k++)
      if (iwun[k] == k) uniq.push_back(k);
    vector<int> order;
    for (int pass = 0; pass < 3; pass++)
      for (int k : uniq) {
        const int nr = numrep[k * 2 + iab];
        if ((pass == 0 && nr == 1) || (pass == 1 && nr == 2) || (pass == 2 && nr > 2)) order.push_back(k);
      }
    m.nuniq = (int)order.size();
    m.numrep.assign(m.nuniq, 0);
    m.irepcol.assign((size_t)m.nuniq * MEXCIT, 0);
    m.ireporb.assign((size_t)m.nuniq * MEXCIT, 0);
    vector<int> kidx(nd, -1);
    for (int kk = 0; kk < m.nuniq; kk++) {
      const int k = order[kk];
      kidx[k] = kk;
      const int nr = numrep[k * 2 + iab];
      if (nr > MEXCIT) return false;
      m.numrep[kk] = nr;
      if (nr == 1) m.nsingle++;
      else if (nr == 2) m.ndouble++;
      for (int r = 0; r < nr; r++) {
        m.irepcol[(size_t)kk * MEXCIT + r] = irc[((size_t)k * 2 + iab) * N + r];
        m.ireporb[(size_t)kk * MEXCIT + r] = iro[((size_t)k * 2 + iab) * N + r];
      }
    }
    for (int k = 1; k < nd; k++) {
      const int kun = iwun[k];
      if (kun != 0) {
        m.kdet2.push_back(k);
        m.kaux2.push_back(kidx[kun]);
      }
    }
  }
  return true;
}

// set_scale_dist (vmc/scale_dist.f90:3-55)
void set_scale_dist(Sys &s) {
  s.asymp_r = 1.0 / s.scalek;
  s.asymp_jasa.assign(s.nctype, 0.0);
  for (int it = 0; it < s.nctype; it++) {
    double v = s.A4(0, it) * s.asymp_r / (1 + s.A4(1, it) * s.asymp_r);
    for (int iord = 2; iord <= s.norda; iord++) v += s.A4(iord, it) * std::pow(s.asymp_r, iord);
    s.asymp_jasa[it] = v;
  }
  for (int i = 0; i < 2; i++) {
    double sspinn;
    int isp;
    if (i == 0) {
      sspinn = 1;
      isp = 0;
    } else {
      sspinn = (s.nspin2b == 1 && s.nocuspb == 0) ? 0.5 : 1.0;
      isp = s.nspin2b - 1;
    }
    double v = sspinn * s.B(0, isp) * s.asymp_r / (1 + s.B(1, isp) * s.asymp_r);
    for (int iord = 2; iord <= s.nordb; iord++) v += s.B(iord, isp) * std::pow(s.asymp_r, iord);
    s.asymp_jasb[i] = v;
  }
}

// ---------------------------------------------------------------------------
// scale_dist family (vmc/scale_dist.f90:57-353), isc = 2..5
// ---------------------------------------------------------------------------
inline void scale_dist0(const Sys &s, double r, double &rr) {
  double k = s.scalek;
  if (k == 0) { rr = r; return; }
  if (s.isc == 2) rr = (1 - std::exp(-k * r)) / k;
  else if (s.isc == 3) {
    double rsc = k * r, rsc2 = rsc * rsc, rsc3 = rsc * rsc2;
    rr = (1 - std::exp(-rsc - 0.5 * rsc2 - (1.0 / 3.0) * rsc3)) / k;
  } else if (s.isc == 4) rr = r * (1 / (1 + k * r));
  else rr = r * (1 / std::pow(1 + std::pow(k * r, 3), 1.0 / 3.0));
}
inline void scale_dist1(const Sys &s, double r, double &rr, double &dd1) {
  double k = s.scalek;
  if (k == 0) { rr = r; dd1 = 1; return; }
  if (s.isc == 2) {
    rr = (1 - std::exp(-k * r)) / k;
    dd1 = 1 - k * rr;
  } else if (s.isc == 3) {
    double rsc = k * r, rsc2 = rsc * rsc, rsc3 = rsc * rsc2;
    double e = std::exp(-rsc - 0.5 * rsc2 - (1.0 / 3.0) * rsc3);
    rr = (1 - e) / k;
    dd1 = (1 + rsc + rsc2) * e;
  } else if (s.isc == 4) {
    double deni = 1 / (1 + k * r);
    rr = r * deni;
    dd1 = deni * deni;
  } else {
    double deni = 1 / std::pow(1 + std::pow(k * r, 3), 1.0 / 3.0);
    rr = r * deni;
    dd1 = std::pow(deni, 4);
  }
}
inline void scale_dist2(const Sys &s, double r, double &rr, double &dd1, double &dd2) {
  double k = s.scalek;
  if (k == 0) { rr = r; dd1 = 1; dd2 = 0; return; }
  if (s.isc == 2) {
    rr = (1 - std::exp(-k * r)) / k;
    dd1 = 1 - k * rr;
    dd2 = -k * dd1;
  } else if (s.isc == 3) {
    double rsc = k * r, rsc2 = rsc * rsc, rsc3 = rsc * rsc2;
    double e = std::exp(-rsc - 0.5 * rsc2 - (1.0 / 3.0) * rsc3);
    rr = (1 - e) / k;
    dd1 = (1 + rsc + rsc2) * e;
    dd2 = -k * rsc2 * (3 + 2 * rsc + rsc2) * e;
  } else if (s.isc == 4) {
    double deni = 1 / (1 + k * r);
    rr = r * deni;
    dd1 = deni * deni;
    dd2 = -2 * k * deni * dd1;
  } else {
    double deni = 1 / std::pow(1 + std::pow(k * r, 3), 1.0 / 3.0);
    rr = r * deni;
    dd1 = std::pow(deni, 4);
    dd2 = -4 * (k * r) * (k * r) * k * dd1 * dd1 / deni;
  }
}

// ---------------------------------------------------------------------------
// Slm (vmc/slm.f90:7): Cartesian monomials x^a y^b z^c times a constant.
// ---------------------------------------------------------------------------
const double CS = 0.28209479177387814, CP = 0.48860251190291992, CD1 = 0.630783130505040,
             CD2 = 1.092548430592079, CF = 0.74635266518023078, CF2 = 1.66889529453113635,
             CF3 = 2.89061144264055405, CG = 0.8462843753216345, CG2 = 2.2390579955406924,
             CG3 = 2.890611442640554, CG4 = 5.006685883593409;
struct SlmDef { int a, b, c; double k; };
const SlmDef SLM[35] = {
    {0, 0, 0, CS},  {1, 0, 0, CP},  {0, 1, 0, CP},  {0, 0, 1, CP},                     // 1-4
    {2, 0, 0, CD1}, {1, 1, 0, CD2}, {1, 0, 1, CD2}, {0, 2, 0, CD1}, {0, 1, 1, CD2},
    {0, 0, 2, CD1},                                                                    // 5-10
    {3, 0, 0, CF},  {2, 1, 0, CF2}, {2, 0, 1, CF2}, {1, 2, 0, CF2}, {1, 1, 1, CF3},
    {1, 0, 2, CF2}, {0, 3, 0, CF},  {0, 2, 1, CF2}, {0, 1, 2, CF2}, {0, 0, 3, CF},    // 11-20
    {4, 0, 0, CG},  {3, 1, 0, CG2}, {3, 0, 1, CG2}, {2, 2, 0, CG3}, {2, 1, 1, CG4},
    {2, 0, 2, CG3}, {1, 3, 0, CG2}, {1, 2, 1, CG4}, {1, 1, 2, CG4}, {1, 0, 3, CG2},
    {0, 4, 0, CG},  {0, 3, 1, CG2}, {0, 2, 2, CG3}, {0, 1, 3, CG2}, {0, 0, 4, CG}};  // 21-35

inline double ipow(double x, int n) {
  double r = 1;
  for (int i = 0; i < n; i++) r *= x;
  return r;
}
// l is CHAMP's 1-based Slm index
void slm(int l, const double *rv, double &y, double *dy, double &lap) {
  const SlmDef &d = SLM[l - 1];
  double x = rv[0], yy = rv[1], z = rv[2];
  double px = ipow(x, d.a), py = ipow(yy, d.b), pz = ipow(z, d.c);
  y = d.k * px * py * pz;
  dy[0] = d.a ? d.k * d.a * ipow(x, d.a - 1) * py * pz : 0.0;
  dy[1] = d.b ? d.k * d.b * px * ipow(yy, d.b - 1) * pz : 0.0;
  dy[2] = d.c ? d.k * d.c * px * py * ipow(z, d.c - 1) : 0.0;
  lap = 0;
  if (d.a >= 2) lap += d.k * d.a * (d.a - 1) * ipow(x, d.a - 2) * py * pz;
  if (d.b >= 2) lap += d.k * d.b * (d.b - 1) * px * ipow(yy, d.b - 2) * pz;
  if (d.c >= 2) lap += d.k * d.c * (d.c - 1) * px * py * ipow(z, d.c - 2);
}

// ---------------------------------------------------------------------------
// splfit (vmc/splfit.f90:3-94): radial function irb of type it at r.
// ---------------------------------------------------------------------------
void splfit(const Sys &s, double r, int irb, int it, double *wfv, int ider) {
  int ig = s.igrid[it];
  double arg = s.arg[it], r0 = s.r0[it];
  double xr, ref0 = 0, ref1 = 0, delh = 0;
  int jx;
  if (ig == 1) {
    xr = (r - r0) / arg + 1;
    jx = (int)xr;
    ref0 = r0 + arg * (jx - 1);
    ref1 = ref0 + arg;
    delh = arg;
  } else if (ig == 2) {
    double dlrad0 = std::log(r0), dlogag = std::log(arg);
    xr = (std::log(r) - dlrad0) / dlogag + 1;
    jx = (int)xr;
    ref0 = r0 * std::pow(arg, jx - 1);
    ref1 = ref0 * arg;
    delh = ref1 - ref0;
  } else {
    double dlogag = std::log(arg);
    xr = (std::log((r + r0) / r0)) / dlogag + 1.0;
    jx = (int)xr;
    ref0 = r0 * std::pow(arg, jx - 1) - r0;
    ref1 = (ref0 + r0) * arg - r0;
    delh = ref1 - ref0;
  }
  if (jx < 1) {
    wfv[0] = s.CE(0, irb, it);
    for (int ii = 2; ii <= CW_NCOEF; ii++) wfv[0] += s.CE(ii - 1, irb, it) * ipow(r, ii - 1);
    if (ider >= 1) {
      wfv[1] = wfv[2] = wfv[3] = 0;
      for (int ii = 2; ii <= CW_NCOEF; ii++) {
        double cc = s.CE(ii - 1, irb, it);
        wfv[1] += (ii - 1) * cc * ipow(r, ii - 2);
        if (ii >= 3) wfv[2] += (ii - 1) * (ii - 2) * cc * ipow(r, ii - 3);
        if (ii >= 4) wfv[3] += (ii - 1) * (ii - 2) * (ii - 3) * cc * ipow(r, ii - 4);
      }
    }
  } else if (jx >= s.nr[it]) {
    wfv[0] = s.AE(0, irb, it) * std::exp(-s.AE(1, irb, it) * r);
    if (ider >= 1) {
      wfv[1] = -s.AE(1, irb, it) * wfv[0];
      wfv[2] = -s.AE(1, irb, it) * wfv[1];
      wfv[3] = -s.AE(1, irb, it) * wfv[2];
    }
  } else {
    // Fortran jx is 1-based: rwf(jx) -> index jx-1
    double y0 = s.RWF(jx - 1, irb, it), y1 = s.RWF(jx, irb, it);
    double d0 = s.D2RWF(jx - 1, irb, it), d1 = s.D2RWF(jx, irb, it);
    const double sixth = 1.0 / 6.0;
    double delhi = 1.0 / delh;
    double bb = (r - ref0) * delhi;
    double aa = (ref1 - r) * delhi;
    double cc = aa * (aa * aa - 1.0) * delh * delh * sixth;
    double dd = bb * (bb * bb - 1.0) * delh * delh * sixth;
    wfv[0] = aa * y0 + bb * y1 + cc * d0 + dd * d1;
    if (ider >= 1) {
      wfv[1] = (y1 - y0) * delhi + (-(3.0 * aa * aa - 1.0) * d0 + (3.0 * bb * bb - 1.0) * d1) * delh * sixth;
      wfv[2] = aa * d0 + bb * d1;
      wfv[3] = (-d0 + d1) * delhi;
    }
  }
}

// ---------------------------------------------------------------------------
// basis_fns (vmc/basis_fns.f90:8-214) + phi_combine (:217-296) for the
// electrons/points k in [k1,k2): fills phin(m,k), dphin(m,k,3), d2phin(m,k)
// with leading dimension ncoord.
// ---------------------------------------------------------------------------
void basis_fns(const Sys &s, int k1, int k2, int ncoord, const double *rvec_en, const double *r_en,
               int ider, double *phin, double *dphin, double *d2phin) {
  const int K = s.K;
  int lilm = 0;
  double wfv[64][4];
  for (int ic = 0; ic < s.M; ic++) {
    int it = s.iwctype[ic];
    int nrb = s.nrbas[it], nbt = s.nbastyp[it];
    int num_slms = 0;
    for (int ib = 0; ib < nbt; ib++) num_slms = std::max(num_slms, s.iwlbas[ib + s.mbastyp * it]);
    vector<double> yv(num_slms), dyv(3 * num_slms), lapv(num_slms);
    for (int k = k1; k < k2; k++) {
      double xc[3] = {rvec_en[0 + 3 * (k + ncoord * ic)], rvec_en[1 + 3 * (k + ncoord * ic)],
                      rvec_en[2 + 3 * (k + ncoord * ic)]};
      double r = r_en[k + ncoord * ic];
      double r2 = r * r, ri = 1.0 / r, ri2 = ri * ri;
      (void)ri2;
      for (int irb = 0; irb < nrb; irb++) {
        if (r <= s.rmaxwf[irb + s.mrwf * it])
          splfit(s, r, irb, it, wfv[irb], ider);
        else
          wfv[irb][0] = wfv[irb][1] = wfv[irb][2] = wfv[irb][3] = 0.0;
      }
      (void)r2;
      for (int i = 0; i < num_slms; i++) slm(i + 1, xc, yv[i], &dyv[3 * i], lapv[i]);
      for (int ib = 0; ib < nbt; ib++) {
        int l = s.iwlbas[ib + s.mbastyp * it];
        int irb = s.iwrwf[ib + s.mbastyp * it] - 1;
        const double *w = wfv[irb];
        double y = yv[l - 1];
        const double *dy = &dyv[3 * (l - 1)];
        double ddy_lap = lapv[l - 1];
        int m = lilm + ib;
        phin[m + K * k] = y * w[0];
        if (ider == 1) {
          double xcri[3] = {xc[0] * ri, xc[1] * ri, xc[2] * ri};
          for (int jj = 0; jj < 3; jj++) dphin[m + K * (k + ncoord * jj)] = y * xcri[jj] * w[1] + dy[jj] * w[0];
        } else if (ider >= 2) {
          double xcri[3] = {xc[0] * ri, xc[1] * ri, xc[2] * ri};
          double d2phi = y * w[2] + y * 2.0 * ri * w[1] + ddy_lap * w[0];
          double dum = 0;
          for (int jj = 0; jj < 3; jj++) {
            dphin[m + K * (k + ncoord * jj)] = y * xcri[jj] * w[1] + dy[jj] * w[0];
            dum += dy[jj] * xcri[jj];
          }
          d2phi += 2.0 * dum * w[1];
          d2phin[m + K * k] = d2phi;
        }
      }
    }
    lilm += nbt;
  }
}

// ---------------------------------------------------------------------------
// Walker state: the CHAMP module variables one rank holds.
// ---------------------------------------------------------------------------
struct Walker {
  const Sys *s;
  int N, M, K, O;
  // config (module config)
  vector<double> xold, xnew, vold, vnew;
  double psido, psijo, psi2o, eold, ekino;
  vector<double> rmino, rminn, rminno, rminon, rvmino, rvminn, rvminno, rvminon, delttn;
  vector<int> nearesto, nearestn;
  // distances (distance_mod, distances_sav)
  vector<double> r_en, rvec_en, r_ee, rvec_ee;
  vector<double> r_en_sav, rvec_en_sav, r_ee_sav, rvec_ee_sav;
  // jastrow_update
  vector<double> fso, fijo, d2ijo, fjo, fsn, fijn, d2ijn, fjn;
  double fsumo, d2o, fsumn, d2n;
  vector<double> vj, vjn;  // velocity_jastrow (== fjo/fjn)
  // phifun
  vector<double> phin, dphin, d2phin;
  // orbval / multislatern
  vector<double> orb, dorb, ddorb, orbn, dorbn, ddorbn;
  // slater
  vector<double> slmi[2], slmin, fp[2], fpp[2], ddx, d2dx2, dorb_tmp;
  double detiab[2], detn;
  // multideterminant state (multimat, multislater, ycompact and their "n" twins)
  vector<double> aa[2], aan;          // [n][O] column-major aa(irep,jrep) = [irep + n*jrep]
  vector<double> wfmat[2], wfmatn;    // [nuniq][MEXCIT^2]
  vector<double> ddet[2], ddetn;      // [nuniq] excitation ratios
  vector<double> detall[2], detalln;  // [ndet] detiab(k,iab)
  vector<double> ymat[2], ymatn;      // [O][n] ymat(jrep,irep) = [jrep + O*irep]
  vector<double> bmat;                // [N][O] b(iorb,i) = [iorb + O*i] (kinetic + nonlocal)
  vector<double> bkin;                // [N][O]
  double psidn_md = 0;                // psid at the proposed position (multideterminant)
  // quadrature (qua), rotated per step
  vector<double> xq, yq, zq;
  // ecp
  vector<double> vps;  // vps(i,ic,l) [i + N*(ic + M*l)]
  vector<double> tvpsp;  // t_vpsp(ic,iq,i) [(i*nquad + iq)*M + ic] of the last hpsi (T-moves)
  // multideterminant T-moves: the quadrature points of the last nonloc
  // (iel, ic, iq) and b_t(iorb, point) = orbital value x term_radial_jas
  vector<int> tq_iel, tq_ic, tq_iq;
  vector<double> tq_trj, btq;  // [npt], [npt][O]
  // estimators (estsum, forcewt, est*)
  double esum, wsum, pesum, tpbsum, acc, esum1;
  // several states: energies and psi_D of the last hpsi, block sums per state
  vector<double> e_st, ekin_st, psid_st, wsum_st, esum_st, pesum_st, tpbsum_st;
  // guiding function: psi_D of every state at the current and at the proposed
  // configuration, and psi2g = sum_i w_i (psi_i/psi_1)^2 at the current one
  vector<double> psid_cur, psidn_st;
  double psi2g_o = 1.0;
  // CI-coefficient derivatives of the last hpsi (optci_deloc's ci_o, taken
  // with respect to the input coefficients) and the SR sums of the sweeps
  vector<double> ci_o, sr_o, sr_eo, sr_oo;
  double sr_w = 0;
  bool opt_ci = false;
  double ecum, ecm2, wcum, pecum, tpbcum, pecm2, tpbcm2, ecum1, ecm21, ecum1s, ecm21s;
  Rng rng;
  bool singular = false;

  explicit Walker(const Sys *sys) : s(sys) {
    N = s->N; M = s->M; K = s->K; O = s->O;
    xold.assign(3 * N, 0); xnew = vold = vnew = xold;
    rmino.assign(N, 0); rminn = rminno = rminon = delttn = rmino;
    rvmino.assign(3 * N, 0); rvminn = rvminno = rvminon = rvmino;
    nearesto.assign(N, 0); nearestn = nearesto;
    r_en.assign(N * M, 0); rvec_en.assign(3 * N * M, 0);
    int np = N * (N - 1) / 2;
    r_ee.assign(std::max(np, 1), 0); rvec_ee.assign(3 * std::max(np, 1), 0);
    r_en_sav.assign(M, 0); rvec_en_sav.assign(3 * M, 0); r_ee_sav.assign(N, 0); rvec_ee_sav.assign(3 * N, 0);
    fso.assign(N * N, 0); fijo.assign(3 * N * N, 0); d2ijo.assign(N * N, 0); fjo.assign(3 * N, 0);
    fsn = fso; fijn = fijo; d2ijn = d2ijo; fjn = fjo;
    fsumo = d2o = fsumn = d2n = 0;
    vj.assign(3 * N, 0); vjn = vj;
    int ncoord = std::max(N, 2 * N * std::max(s->nquad, 1));
    phin.assign((size_t)K * ncoord, 0); dphin.assign((size_t)K * ncoord * 3, 0); d2phin.assign((size_t)K * ncoord, 0);
    orb.assign(N * O, 0); dorb.assign(O * N * 3, 0); ddorb.assign(O * N, 0);
    orbn.assign(O, 0); dorbn.assign(O * 3, 0); ddorbn.assign(O, 0);
    int n1 = s->nup, n2 = s->ndn;
    slmi[0].assign(std::max(n1 * n1, 1), 0); slmi[1].assign(std::max(n2 * n2, 1), 0);
    slmin.assign(std::max(std::max(n1 * n1, n2 * n2), 1), 0);
    fp[0].assign(3 * std::max(n1 * n1, 1), 0); fp[1].assign(3 * std::max(n2 * n2, 1), 0);
    fpp[0].assign(std::max(n1 * n1, 1), 0); fpp[1].assign(std::max(n2 * n2, 1), 0);
    ddx.assign(3 * N, 0); d2dx2.assign(N, 0); dorb_tmp.assign(3 * O, 0);
    detiab[0] = detiab[1] = detn = 0;
    if (s->ndet > 1) {
      int nmx = std::max(std::max(n1, n2), 1);
      for (int iab = 0; iab < 2; iab++) {
        int nel = std::max(iab == 0 ? n1 : n2, 1);
        aa[iab].assign((size_t)nel * O, 0);
        wfmat[iab].assign((size_t)std::max(s->md[iab].nuniq, 1) * MEXCIT * MEXCIT, 0);
        ddet[iab].assign(std::max(s->md[iab].nuniq, 1), 0);
        detall[iab].assign(s->ndet, 0);
        ymat[iab].assign((size_t)O * nel, 0);
      }
      aan.assign((size_t)nmx * O, 0);
      wfmatn.assign((size_t)std::max(std::max(s->md[0].nuniq, s->md[1].nuniq), 1) * MEXCIT * MEXCIT, 0);
      ddetn.assign(std::max(std::max(s->md[0].nuniq, s->md[1].nuniq), 1), 0);
      detalln.assign(s->ndet, 0);
      ymatn.assign((size_t)O * nmx, 0);
    }
    bmat.assign((size_t)N * O, 0);
    bkin.assign((size_t)N * O, 0);
    xq = s->xq0; yq = s->yq0; zq = s->zq0;
    vps.assign((size_t)N * M * CW_MPS_L, 0);
    tvpsp.assign((size_t)N * std::max(s->nquad, 1) * M, 0.0);
    zero_estimators();
  }
  void zero_estimators() {
    esum = wsum = pesum = tpbsum = acc = esum1 = 0;
    for (auto *v : {&wsum_st, &esum_st, &pesum_st, &tpbsum_st}) v->assign(s->nstates, 0.0);
    for (auto *v : {&e_st, &ekin_st, &psid_st}) v->resize(s->nstates, 0.0);
    ecum = ecm2 = wcum = pecum = tpbcum = pecm2 = tpbcm2 = ecum1 = ecm21 = ecum1s = ecm21s = 0;
  }

  // ---- distances (vmc/distances.f90:3-109) ----
  void distances(int iel, const double *x) {  // iel: -1 == all (CHAMP iel=0)
    int i1, i2;
    if (iel < 0) {
      i1 = 0; i2 = N - 1;
    } else {
      i1 = i2 = iel;
      for (int ic = 0; ic < M; ic++) {
        r_en_sav[ic] = r_en[iel + N * ic];
        for (int m = 0; m < 3; m++) rvec_en_sav[m + 3 * ic] = rvec_en[m + 3 * (iel + N * ic)];
      }
      for (int jj = 0; jj < iel; jj++) {
        int ij = iel * (iel - 1) / 2 + jj;
        r_ee_sav[jj] = r_ee[ij];
        for (int m = 0; m < 3; m++) rvec_ee_sav[m + 3 * jj] = rvec_ee[m + 3 * ij];
      }
      for (int jj = iel + 1; jj < N; jj++) {
        int ij = jj * (jj - 1) / 2 + iel;
        r_ee_sav[jj] = r_ee[ij];
        for (int m = 0; m < 3; m++) rvec_ee_sav[m + 3 * jj] = rvec_ee[m + 3 * ij];
      }
    }
    for (int i = i1; i <= i2; i++)
      for (int ic = 0; ic < M; ic++) {
        double r = 0;
        for (int m = 0; m < 3; m++) {
          double d = x[m + 3 * i] - s->cent[m + 3 * ic];
          rvec_en[m + 3 * (i + N * ic)] = d;
        }
        for (int m = 0; m < 3; m++) r += rvec_en[m + 3 * (i + N * ic)] * rvec_en[m + 3 * (i + N * ic)];
        r_en[i + N * ic] = std::sqrt(r);
      }
    auto pair = [&](int i, int j, int ij) {  // rvec_ee(ij) = x(i) - x(j)
      double r = 0;
      for (int m = 0; m < 3; m++) rvec_ee[m + 3 * ij] = x[m + 3 * i] - x[m + 3 * j];
      for (int m = 0; m < 3; m++) r += rvec_ee[m + 3 * ij] * rvec_ee[m + 3 * ij];
      r_ee[ij] = std::sqrt(r);
    };
    if (iel < 0) {
      for (int i = 1; i < N; i++)
        for (int j = 0; j < i; j++) pair(i, j, i * (i - 1) / 2 + j);
    } else {
      for (int i = 0; i < iel; i++) pair(iel, i, iel * (iel - 1) / 2 + i);
      for (int i = iel + 1; i < N; i++) pair(i, iel, i * (i - 1) / 2 + iel);
    }
  }
  // distancese_restore (vmc/distances.f90:164)
  void distancese_restore(int iel) {
    for (int ic = 0; ic < M; ic++) {
      r_en[iel + N * ic] = r_en_sav[ic];
      for (int m = 0; m < 3; m++) rvec_en[m + 3 * (iel + N * ic)] = rvec_en_sav[m + 3 * ic];
    }
    for (int jj = 0; jj < N; jj++) {
      if (jj == iel) continue;
      int i = jj < iel ? iel : jj, j = jj < iel ? jj : iel;
      int ij = i * (i - 1) / 2 + j;
      r_ee[ij] = r_ee_sav[jj];
      for (int m = 0; m < 3; m++) rvec_ee[m + 3 * ij] = rvec_ee_sav[m + 3 * jj];
    }
  }

  // ---- e-e-n polynomial shared by jastrow_factor4 / jastrow4e ----
  // Accumulates fc, fu, fuu, fi, fii, fj, fjj, fui, fuj (vmc/jastrow4.f90 n/k/l loop).
  struct Een { double fc, fu, fuu, fi, fii, fj, fjj, fui, fuj; };
  Een een_terms(const double *uu, const double *ss, const double *tt, const double *rri,
                const double *rrj, int it, bool second) const {
    // arrays are offset so index -3 .. nordj is valid: pass pointers to index 0
    Een e{0, 0, 0, 0, 0, 0, 0, 0, 0};
    int ll = 0;
    for (int n = 2; n <= s->nordc; n++)
      for (int k = n - 1; k >= 0; k--) {
        int l_hi = (k == 0) ? n - k - 2 : n - k;
        for (int l = l_hi; l >= 0; l--) {
          int m = (n - k - l) / 2;
          if (2 * m == n - k - l) {
            double cc = s->C(ll, it);
            ll++;
            e.fc += cc * uu[k] * ss[l] * tt[m];
            e.fu += cc * k * uu[k - 1] * ss[l] * tt[m];
            e.fi += cc * uu[k] * ((l + m) * rri[l + m - 1] * rrj[m] + m * rri[m - 1] * rrj[l + m]);
            e.fj += cc * uu[k] * ((l + m) * rrj[l + m - 1] * rri[m] + m * rrj[m - 1] * rri[l + m]);
            if (second) {
              e.fuu += cc * k * (k - 1) * uu[k - 2] * ss[l] * tt[m];
              e.fii += cc * uu[k] * ((l + m) * (l + m - 1) * rri[l + m - 2] * rrj[m] + m * (m - 1) * rri[m - 2] * rrj[l + m]);
              e.fjj += cc * uu[k] * ((l + m) * (l + m - 1) * rrj[l + m - 2] * rri[m] + m * (m - 1) * rrj[m - 2] * rri[l + m]);
              e.fui += cc * k * uu[k - 1] * ((l + m) * rri[l + m - 1] * rrj[m] + m * rri[m - 1] * rrj[l + m]);
              e.fuj += cc * k * uu[k - 1] * ((l + m) * rrj[l + m - 1] * rri[m] + m * rrj[m - 1] * rri[l + m]);
            }
          }
        }
      }
    return e;
  }

  static inline int FI(int i, int j, int N) { return i + N * j; }
  static inline int FIJ(int k, int i, int j, int N) { return k + 3 * (i + N * j); }

  // ---- raw Jastrow parameter derivatives (vmc/deriv_jastrow4.f90 gvalue) ----
  // d J / d p for every Jastrow coefficient taken on its own, before CHAMP's
  // selection of varied parameters and its cusp-dependent c terms (a linear
  // map applied on the host):
  //   a part [nctype][norda+1]: q = 1 Pade numerator a(1), q = 2 Pade
  //     denominator a(2), q >= 3 the r^(q-1) coefficient (:588-630);
  //   b part [nspin2b][nordb+1]: the same for the e-e function, with the
  //     sspinn factor on the Pade terms (:181-234);
  //   c part [nctype][nterms]: the e-e-n term values pc = uu(k) ss(l) tt(m)
  //     summed over pairs and centres of the type (:320-330).
  // Pairs whose scaled distance is asymptotic skip the b part; pair-centre
  // combinations with both e-n distances asymptotic skip the c part; e-n
  // distances at the asymptote skip the a part (:150, :266, :553).
  void jas_raw(double *out) const {
    const int NA = s->norda + 1, NB = s->nordb + 1, NT = s->nterms;
    const int ob = s->nctype * NA, oc = ob + s->nspin2b * NB;
    std::fill(out, out + oc + s->nctype * NT, 0.0);
    const double ar = s->asymp_r;
    const int nordj = std::max(std::max(s->norda, s->nordb), s->nordc);
    vector<double> UU(nordj + 4, 0), SS(nordj + 4, 0), TT(nordj + 4, 0), RI(nordj + 4, 0), RJ(nordj + 4, 0);
    double *uu = &UU[3], *ss = &SS[3], *tt = &TT[3], *rri = &RI[3], *rrj = &RJ[3];
    uu[0] = 1; ss[0] = 2; tt[0] = 1; rri[0] = 1; rrj[0] = 1;
    for (int i = 1; i < N; i++)
      for (int j = 0; j < i; j++) {
        const int ij = i * (i - 1) / 2 + j;
        double sspinn = 1;
        int isb = 0;
        if (i < s->nup || j >= s->nup) {
          if (s->nspin2b == 2) isb = 1;
          else if (s->nocuspb == 0) sspinn = 0.5;
        }
        double dd1;
        scale_dist1(*s, r_ee[ij], uu[1], dd1);
        if (uu[1] != ar) {
          const double b1 = s->B(0, isb), b2 = s->B(1, isb);
          double *g = out + ob + isb * NB;
          g[0] += sspinn * uu[1] / (1 + b2 * uu[1]) - sspinn * ar / (1 + b2 * ar);
          if (NB > 1) {
            const double bot0 = 1 + b2 * uu[1];
            g[1] += -sspinn * b1 * uu[1] * uu[1] / (bot0 * bot0) +
                    sspinn * b1 * ar * ar / ((1 + b2 * ar) * (1 + b2 * ar));
          }
          for (int q = 3; q <= NB; q++) g[q - 1] += std::pow(uu[1], q - 1) - std::pow(ar, q - 1);
        }
        if (s->nordc <= 1) continue;
        const double z = 1 - s->scalek * uu[1];
        for (int iord = 1; iord <= s->nordc; iord++) uu[iord] = iord == 1 ? z : z * uu[iord - 1];
        for (int ic = 0; ic < M; ic++) {
          const int it = s->iwctype[ic];
          double dd7, dd8;
          scale_dist1(*s, r_en[i + N * ic], rri[1], dd7);
          scale_dist1(*s, r_en[j + N * ic], rrj[1], dd8);
          if (rri[1] == ar && rrj[1] == ar) continue;
          rri[1] = 1 - s->scalek * rri[1];
          rrj[1] = 1 - s->scalek * rrj[1];
          for (int iord = 1; iord <= s->nordc; iord++) {
            rri[iord] = rri[1] * rri[iord - 1];
            rrj[iord] = rrj[1] * rrj[iord - 1];
            ss[iord] = rri[iord] + rrj[iord];
            tt[iord] = rri[iord] * rrj[iord];
          }
          double *g = out + oc + it * NT;
          int ll = 0;
          for (int n = 2; n <= s->nordc; n++)
            for (int k = n - 1; k >= 0; k--) {
              const int l_hi = (k == 0) ? n - k - 2 : n - k;
              for (int l = l_hi; l >= 0; l--) {
                const int m = (n - k - l) / 2;
                if (2 * m == n - k - l) g[ll++] += uu[k] * ss[l] * tt[m];
              }
            }
        }
      }
    for (int i = 0; i < N; i++)
      for (int ic = 0; ic < M; ic++) {
        const int it = s->iwctype[ic];
        double r, dd7;
        scale_dist1(*s, r_en[i + N * ic], r, dd7);
        if (r == ar) continue;
        const double a1 = s->A4(0, it), a2 = s->A4(1, it);
        double *g = out + it * NA;
        g[0] += r / (1 + a2 * r) - ar / (1 + a2 * ar);
        if (NA > 1) {
          const double bot0 = 1 + a2 * r;
          g[1] += -a1 * r * r / (bot0 * bot0) + a1 * ar * ar / ((1 + a2 * ar) * (1 + a2 * ar));
        }
        for (int q = 3; q <= NA; q++) g[q - 1] += std::pow(r, q - 1) - std::pow(ar, q - 1);
      }
  }

  // ---- jastrow_factor4 (vmc/jastrow4.f90:3): full J with Laplacian ----
  void jastrow_factor4() {
    const int nordj = std::max(std::max(s->norda, s->nordb), s->nordc);
    vector<double> UU(nordj + 4, 0), SS(nordj + 4, 0), TT(nordj + 4, 0), RI(nordj + 4, 0), RJ(nordj + 4, 0);
    double *uu = &UU[3], *ss = &SS[3], *tt = &TT[3], *rri = &RI[3], *rrj = &RJ[3];
    fsumo = 0; d2o = 0;
    std::fill(fjo.begin(), fjo.end(), 0.0);
    uu[0] = 1; ss[0] = 2; tt[0] = 1; rri[0] = 1; rrj[0] = 1;
    if (N >= 2) {
      int ij = 0;
      for (int i = 1; i < N; i++)
        for (int j = 0; j < i; j++, ij++) {
          fso[FI(i, j, N)] = 0;
          d2ijo[FI(i, j, N)] = 0;
          for (int k = 0; k < 3; k++) fijo[FIJ(k, i, j, N)] = fijo[FIJ(k, j, i, N)] = 0;
          double sspinn = 1;
          int isb = 0, ipar = 0;
          if (i < s->nup || j >= s->nup) {
            if (s->nspin2b == 2) isb = 1;
            else if (s->nocuspb == 0) sspinn = 0.5;
            ipar = 1;
          }
          double rij = r_ee[ij], dd1, dd2;
          scale_dist2(*s, rij, uu[1], dd1, dd2);
          if (uu[1] != s->asymp_r) {
            double top = sspinn * s->B(0, isb) * uu[1], topu = sspinn * s->B(0, isb), topuu = 0;
            double bot = 1 + s->B(1, isb) * uu[1], botu = s->B(1, isb), botuu = 0, bot2 = bot * bot;
            double fee = top / bot - s->asymp_jasb[ipar];
            double feeu = topu / bot - botu * top / bot2;
            double feeuu = topuu - (botuu * top + 2 * botu * topu) / bot + 2 * botu * botu * top / bot2;
            feeuu = feeuu / bot;
            for (int iord = 2; iord <= s->nordb; iord++) {
              uu[iord] = uu[1] * uu[iord - 1];
              fee += s->B(iord, isb) * uu[iord];
              feeu += s->B(iord, isb) * iord * uu[iord - 1];
              feeuu += s->B(iord, isb) * iord * (iord - 1) * uu[iord - 2];
            }
            feeuu = feeuu * dd1 * dd1 + feeu * dd2;
            feeu = feeu * dd1 / rij;
            fso[FI(i, j, N)] += fee;
            for (int k = 0; k < 3; k++) {
              fijo[FIJ(k, i, j, N)] += feeu * rvec_ee[k + 3 * ij];
              fijo[FIJ(k, j, i, N)] -= feeu * rvec_ee[k + 3 * ij];
            }
            d2ijo[FI(i, j, N)] += 2 * (feeuu + 2 * feeu);
          }
          if (s->nordc > 1) {
            // switch_scale2 on uu(1)
            uu[1] = 1 - s->scalek * uu[1];
            dd1 = -s->scalek * dd1;
            dd2 = -s->scalek * dd2;
            for (int iord = 2; iord <= s->nordc; iord++) uu[iord] = uu[1] * uu[iord - 1];
            for (int ic = 0; ic < M; ic++) {
              int it = s->iwctype[ic];
              double ri = r_en[i + N * ic], rj = r_en[j + N * ic];
              double dd7, dd8, dd9, dd10;
              scale_dist2(*s, ri, rri[1], dd7, dd9);
              scale_dist2(*s, rj, rrj[1], dd8, dd10);
              if (rri[1] == s->asymp_r && rrj[1] == s->asymp_r) continue;
              rri[1] = 1 - s->scalek * rri[1]; dd7 = -s->scalek * dd7; dd9 = -s->scalek * dd9;
              rrj[1] = 1 - s->scalek * rrj[1]; dd8 = -s->scalek * dd8; dd10 = -s->scalek * dd10;
              double sgs = ri + rj, tgs = ri - rj;
              double u2pst = rij * rij + sgs * tgs, u2mst = rij * rij - sgs * tgs;
              for (int iord = 1; iord <= s->nordc; iord++) {
                rri[iord] = rri[1] * rri[iord - 1];
                rrj[iord] = rrj[1] * rrj[iord - 1];
                ss[iord] = rri[iord] + rrj[iord];
                tt[iord] = rri[iord] * rrj[iord];
              }
              Een e = een_terms(uu, ss, tt, rri, rrj, it, true);
              double fuu = e.fuu * dd1 * dd1 + e.fu * dd2;
              double fu = e.fu * dd1 / rij;
              double fui = e.fui * dd1 * dd7, fuj = e.fuj * dd1 * dd8;
              double fii = e.fii * dd7 * dd7 + e.fi * dd9, fjj = e.fjj * dd8 * dd8 + e.fj * dd10;
              double fi = e.fi * dd7 / ri, fj = e.fj * dd8 / rj;
              fso[FI(i, j, N)] += e.fc;
              for (int k = 0; k < 3; k++) {
                fijo[FIJ(k, i, j, N)] += fi * rvec_en[k + 3 * (i + N * ic)] + fu * rvec_ee[k + 3 * ij];
                fijo[FIJ(k, j, i, N)] += fj * rvec_en[k + 3 * (j + N * ic)] - fu * rvec_ee[k + 3 * ij];
              }
              d2ijo[FI(i, j, N)] += 2 * (fuu + 2 * fu) + fui * u2pst / (ri * rij) + fuj * u2mst / (rj * rij) +
                                    fii + 2 * fi + fjj + 2 * fj;
            }
          }
          fsumo += fso[FI(i, j, N)];
          for (int k = 0; k < 3; k++) {
            fjo[k + 3 * i] += fijo[FIJ(k, i, j, N)];
            fjo[k + 3 * j] += fijo[FIJ(k, j, i, N)];
          }
          d2o += d2ijo[FI(i, j, N)];
        }
    }
    for (int i = 0; i < N; i++) {
      fso[FI(i, i, N)] = 0;
      for (int k = 0; k < 3; k++) fijo[FIJ(k, i, i, N)] = 0;
      d2ijo[FI(i, i, N)] = 0;
      for (int ic = 0; ic < M; ic++) {
        int it = s->iwctype[ic];
        double ri = r_en[i + N * ic], dd7, dd9;
        scale_dist2(*s, ri, rri[1], dd7, dd9);
        if (rri[1] == s->asymp_r) continue;
        double top = s->A4(0, it) * rri[1], topi = s->A4(0, it), topii = 0;
        double bot = 1 + s->A4(1, it) * rri[1], boti = s->A4(1, it), botii = 0, bot2 = bot * bot;
        double fen = top / bot - s->asymp_jasa[it];
        double feni = topi / bot - boti * top / bot2;
        double fenii = topii - (botii * top + 2 * boti * topi) / bot + 2 * boti * boti * top / bot2;
        fenii = fenii / bot;
        for (int iord = 2; iord <= s->norda; iord++) {
          rri[iord] = std::pow(rri[1], iord);
          fen += s->A4(iord, it) * rri[iord];
          feni += s->A4(iord, it) * iord * rri[iord - 1];
          fenii += s->A4(iord, it) * iord * (iord - 1) * rri[iord - 2];
        }
        fenii = fenii * dd7 * dd7 + feni * dd9;
        feni = feni * dd7 / ri;
        fso[FI(i, i, N)] += fen;
        for (int k = 0; k < 3; k++) fijo[FIJ(k, i, i, N)] += feni * rvec_en[k + 3 * (i + N * ic)];
        d2ijo[FI(i, i, N)] += fenii + 2 * feni;
      }
      fsumo += fso[FI(i, i, N)];
      for (int k = 0; k < 3; k++) fjo[k + 3 * i] += fijo[FIJ(k, i, i, N)];
      d2o += d2ijo[FI(i, i, N)];
    }
  }

  // ---- jastrow4e (vmc/jastrow4e.f90:3), iflag 0 (no Laplacian) or 1 ----
  void jastrow4e(int iel, int iflag) {
    const int nordj = std::max(std::max(s->norda, s->nordb), s->nordc);
    vector<double> UU(nordj + 4, 0), SS(nordj + 4, 0), TT(nordj + 4, 0), RI(nordj + 4, 0), RJ(nordj + 4, 0);
    double *uu = &UU[3], *ss = &SS[3], *tt = &TT[3], *rri = &RI[3], *rrj = &RJ[3];
    uu[0] = 1; ss[0] = 2; tt[0] = 1; rri[0] = 1; rrj[0] = 1;
    const bool second = iflag > 0;
    if (N >= 2) {
      fjn = fjo;
      fsumn = fsumo;
      d2n = d2o;
      for (int jj = 0; jj < N; jj++) {
        if (jj == iel) continue;
        int i = jj < iel ? iel : jj, j = jj < iel ? jj : iel;
        int ij = i * (i - 1) / 2 + j;
        for (int k = 0; k < 3; k++) fijn[FIJ(k, i, j, N)] = fijn[FIJ(k, j, i, N)] = 0;
        fsn[FI(i, j, N)] = 0;
        d2ijn[FI(i, j, N)] = 0;
        double sspinn = 1;
        int ipar = 0, isb = 0;
        if (i < s->nup || j >= s->nup) {
          if (s->nspin2b == 2) isb = 1;
          else if (s->nocuspb == 0) sspinn = 0.5;
          ipar = 1;
        }
        double rij = r_ee[ij], dd1, dd2 = 0;
        if (!second) scale_dist1(*s, rij, uu[1], dd1);
        else scale_dist2(*s, rij, uu[1], dd1, dd2);
        if (uu[1] != s->asymp_r) {
          double top = sspinn * s->B(0, isb) * uu[1], topu = sspinn * s->B(0, isb);
          double bot = 1 + s->B(1, isb) * uu[1], botu = s->B(1, isb), bot2 = bot * bot;
          double fee = top / bot - s->asymp_jasb[ipar];
          double feeu = topu / bot - botu * top / bot2;
          for (int iord = 2; iord <= s->nordb; iord++) {
            uu[iord] = uu[1] * uu[iord - 1];
            fee += s->B(iord, isb) * uu[iord];
            feeu += s->B(iord, isb) * iord * uu[iord - 1];
          }
          double feeuu = 0;
          if (second) {
            double topuu = 0, botuu = 0;
            feeuu = topuu - (botuu * top + 2 * botu * topu) / bot + 2 * botu * botu * top / bot2;
            feeuu = feeuu / bot;
            for (int iord = 2; iord <= s->nordb; iord++) feeuu += s->B(iord, isb) * iord * (iord - 1) * uu[iord - 2];
            feeuu = feeuu * dd1 * dd1 + feeu * dd2;
          }
          feeu = feeu * dd1 / rij;
          fsn[FI(i, j, N)] += fee;
          for (int k = 0; k < 3; k++) {
            fijn[FIJ(k, i, j, N)] += feeu * rvec_ee[k + 3 * ij];
            fijn[FIJ(k, j, i, N)] -= feeu * rvec_ee[k + 3 * ij];
          }
          if (second) d2ijn[FI(i, j, N)] += 2 * (feeuu + 2 * feeu);
        }
        if (s->nordc > 1) {
          uu[1] = 1 - s->scalek * uu[1];
          dd1 = -s->scalek * dd1;
          if (second) dd2 = -s->scalek * dd2;
          for (int iord = 2; iord <= s->nordc; iord++) uu[iord] = uu[1] * uu[iord - 1];
          for (int ic = 0; ic < M; ic++) {
            int it = s->iwctype[ic];
            double ri = r_en[i + N * ic], rj = r_en[j + N * ic];
            double dd7, dd8, dd9 = 0, dd10 = 0;
            if (!second) {
              scale_dist1(*s, ri, rri[1], dd7);
              scale_dist1(*s, rj, rrj[1], dd8);
            } else {
              scale_dist2(*s, ri, rri[1], dd7, dd9);
              scale_dist2(*s, rj, rrj[1], dd8, dd10);
            }
            if (rri[1] == s->asymp_r && rrj[1] == s->asymp_r) continue;
            rri[1] = 1 - s->scalek * rri[1]; dd7 = -s->scalek * dd7;
            rrj[1] = 1 - s->scalek * rrj[1]; dd8 = -s->scalek * dd8;
            if (second) { dd9 = -s->scalek * dd9; dd10 = -s->scalek * dd10; }
            for (int iord = 1; iord <= s->nordc; iord++) {
              rri[iord] = rri[1] * rri[iord - 1];
              rrj[iord] = rrj[1] * rrj[iord - 1];
              ss[iord] = rri[iord] + rrj[iord];
              tt[iord] = rri[iord] * rrj[iord];
            }
            Een e = een_terms(uu, ss, tt, rri, rrj, it, second);
            double fuu = 0, fui = 0, fuj = 0, fii = 0, fjj = 0, u2pst = 0, u2mst = 0;
            if (second) {
              double sgs = ri + rj, tgs = ri - rj;
              u2pst = rij * rij + sgs * tgs;
              u2mst = rij * rij - sgs * tgs;
              fuu = e.fuu * dd1 * dd1 + e.fu * dd2;
              fui = e.fui * dd1 * dd7;
              fuj = e.fuj * dd1 * dd8;
              fii = e.fii * dd7 * dd7 + e.fi * dd9;
              fjj = e.fjj * dd8 * dd8 + e.fj * dd10;
            }
            double fu = e.fu * dd1 / rij, fi = e.fi * dd7 / ri, fj = e.fj * dd8 / rj;
            fsn[FI(i, j, N)] += e.fc;
            for (int k = 0; k < 3; k++) {
              fijn[FIJ(k, i, j, N)] += fi * rvec_en[k + 3 * (i + N * ic)] + fu * rvec_ee[k + 3 * ij];
              fijn[FIJ(k, j, i, N)] += fj * rvec_en[k + 3 * (j + N * ic)] - fu * rvec_ee[k + 3 * ij];
            }
            if (second)
              d2ijn[FI(i, j, N)] += 2 * (fuu + 2 * fu) + fui * u2pst / (ri * rij) + fuj * u2mst / (rj * rij) + fii +
                                    2 * fi + fjj + 2 * fj;
          }
        }
        fsumn = fsumn + fsn[FI(i, j, N)] - fso[FI(i, j, N)];
        for (int k = 0; k < 3; k++) {
          fjn[k + 3 * i] = fjn[k + 3 * i] + fijn[FIJ(k, i, j, N)] - fijo[FIJ(k, i, j, N)];
          fjn[k + 3 * j] = fjn[k + 3 * j] + fijn[FIJ(k, j, i, N)] - fijo[FIJ(k, j, i, N)];
        }
        d2n = d2n + d2ijn[FI(i, j, N)] - d2ijo[FI(i, j, N)];
      }
    }
    // e-n part (label 65)
    for (int k = 0; k < 3; k++) fijn[FIJ(k, iel, iel, N)] = 0;
    fsn[FI(iel, iel, N)] = 0;
    d2ijn[FI(iel, iel, N)] = 0;
    for (int ic = 0; ic < M; ic++) {
      int it = s->iwctype[ic];
      double ri = r_en[iel + N * ic], dd7, dd9 = 0;
      if (!second) scale_dist1(*s, ri, rri[1], dd7);
      else scale_dist2(*s, ri, rri[1], dd7, dd9);
      if (rri[1] == s->asymp_r) continue;
      double top = s->A4(0, it) * rri[1], topi = s->A4(0, it);
      double bot = s->A4(1, it) * rri[1], boti = s->A4(1, it);
      bot = 1 + bot;
      double bot2 = bot * bot;
      double fen = top / bot - s->asymp_jasa[it];
      double feni = topi / bot - boti * top / bot2;
      for (int iord = 2; iord <= s->norda; iord++) {
        rri[iord] = std::pow(rri[1], iord);
        fen += s->A4(iord, it) * rri[iord];
        feni += s->A4(iord, it) * iord * rri[iord - 1];
      }
      double fenii = 0;
      if (second) {
        double topii = 0, botii = 0;
        fenii = topii - (botii * top + 2 * boti * topi) / bot + 2 * boti * boti * top / bot2;
        fenii = fenii / bot;
        for (int iord = 2; iord <= s->norda; iord++) fenii += s->A4(iord, it) * iord * (iord - 1) * rri[iord - 2];
        fenii = fenii * dd7 * dd7 + feni * dd9;
      }
      feni = feni * dd7 / ri;
      fsn[FI(iel, iel, N)] += fen;
      for (int k = 0; k < 3; k++) fijn[FIJ(k, iel, iel, N)] += feni * rvec_en[k + 3 * (iel + N * ic)];
      if (second) d2ijn[FI(iel, iel, N)] += fenii + 2 * feni;
    }
    fsumn = fsumn + fsn[FI(iel, iel, N)] - fso[FI(iel, iel, N)];
    for (int k = 0; k < 3; k++)
      fjn[k + 3 * iel] = fjn[k + 3 * iel] + fijn[FIJ(k, iel, iel, N)] - fijo[FIJ(k, iel, iel, N)];
    d2n = d2n + d2ijn[FI(iel, iel, N)] - d2ijo[FI(iel, iel, N)];
  }

  // jastrowe (vmc/jastrowe.f90:3): v = fjn, psij = fsumn
  void jastrowe(int iel, int iflag) {
    jastrow4e(iel, iflag);
    vjn = fjn;
  }
  // jassav (vmc/jassav.f90:3)
  void jassav(int iel, int iflag) {
    fsumo = fsumn;
    fjo = fjn;
    for (int j = 0; j <= iel; j++) fso[FI(iel, j, N)] = fsn[FI(iel, j, N)];
    for (int j = iel + 1; j < N; j++) fso[FI(j, iel, N)] = fsn[FI(j, iel, N)];
    for (int j = 0; j < N; j++)
      for (int k = 0; k < 3; k++) {
        fijo[FIJ(k, iel, j, N)] = fijn[FIJ(k, iel, j, N)];
        fijo[FIJ(k, j, iel, N)] = fijn[FIJ(k, j, iel, N)];
      }
    if (iflag > 0) {
      d2o = d2n;
      for (int j = 0; j <= iel; j++) d2ijo[FI(iel, j, N)] = d2ijn[FI(iel, j, N)];
      for (int j = iel + 1; j < N; j++) d2ijo[FI(j, iel, N)] = d2ijn[FI(j, iel, N)];
    }
    vj = vjn;
  }

  // ---- orbitals (vmc/orbitals_no_qmckl.f90:19): all electrons, ider=2 ----
  void orbitals_all() {
    basis_fns(*s, 0, N, N, rvec_en.data(), r_en.data(), 2, phin.data(), dphin.data(), d2phin.data());
    for (int i = 0; i < N; i++)
      for (int iorb = 0; iorb < O; iorb++) {
        double a = 0, d1 = 0, d2 = 0, d3 = 0, dd = 0;
        for (int m = 0; m < K; m++) {
          double cm = s->COEF(m, iorb);
          a += cm * phin[m + K * i];
          d1 += cm * dphin[m + K * (i + N * 0)];
          d2 += cm * dphin[m + K * (i + N * 1)];
          d3 += cm * dphin[m + K * (i + N * 2)];
          dd += cm * d2phin[m + K * i];
        }
        orb[i + N * iorb] = a;
        dorb[iorb + O * (i + N * 0)] = d1;
        dorb[iorb + O * (i + N * 1)] = d2;
        dorb[iorb + O * (i + N * 2)] = d3;
        ddorb[iorb + O * i] = dd;
      }
  }
  // orbitalse (vmc/orbitals_no_qmckl.f90:195): one electron, ider=1 or 2
  void orbitalse(int iel, int iflag) {
    int ider = iflag > 0 ? 2 : 1;
    basis_fns(*s, iel, iel + 1, N, rvec_en.data(), r_en.data(), ider, phin.data(), dphin.data(), d2phin.data());
    for (int iorb = 0; iorb < O; iorb++) {
      double a = 0, d1 = 0, d2 = 0, d3 = 0, dd = 0;
      for (int m = 0; m < K; m++) {
        double cm = s->COEF(m, iorb);
        a += cm * phin[m + K * iel];
        d1 += cm * dphin[m + K * (iel + N * 0)];
        d2 += cm * dphin[m + K * (iel + N * 1)];
        d3 += cm * dphin[m + K * (iel + N * 2)];
        if (ider == 2) dd += cm * d2phin[m + K * iel];
      }
      orbn[iorb] = a;
      dorbn[iorb + O * 0] = d1;
      dorbn[iorb + O * 1] = d2;
      dorbn[iorb + O * 2] = d3;
      if (ider == 2) ddorbn[iorb] = dd;
    }
  }

  int nel_of(int iab) const { return iab == 0 ? s->nup : s->ndn; }
  int occ(int jslot) const { return s->iworbd[jslot] - 1; }  // iworbd(j,kref), 0-based orbital

  // ---- determinant (vmc/determinant.f90:9) + matinv ----
  bool determinant() {
    orbitals_all();
    for (int iab = 0; iab < 2; iab++) {
      int ish = iab == 0 ? 0 : s->nup, nel = nel_of(iab);
      detiab[iab] = 1.0;
      vector<double> &sl = slmi[iab];
      for (int j = 0; j < nel; j++) {
        int jorb = occ(j + ish);
        int jk = nel * j;
        for (int e = 0; e < nel; e++) {
          sl[jk + e] = orb[(ish + e) + N * jorb];
          // fp(k, j, iab) with stride nel*3 over electrons: fp(k, j + nel*e)
          for (int k = 0; k < 3; k++) fp[iab][k + 3 * (j + nel * e)] = dorb[jorb + O * ((ish + e) + N * k)];
          fpp[iab][j + nel * e] = ddorb[jorb + O * (ish + e)];
        }
      }
      if (nel > 0) {
        if (or_matinv(sl.data(), nel, &detiab[iab]) != 0) return false;
      }
      for (int i = 0; i < nel; i++) {
        int ik = nel * i;
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        for (int j = 0; j < nel; j++) {
          a0 += sl[j + ik] * fp[iab][0 + 3 * (j + ik)];
          a1 += sl[j + ik] * fp[iab][1 + 3 * (j + ik)];
          a2 += sl[j + ik] * fp[iab][2 + 3 * (j + ik)];
          a3 += sl[j + ik] * fpp[iab][j + ik];
        }
        ddx[0 + 3 * (i + ish)] = a0;
        ddx[1 + 3 * (i + ish)] = a1;
        ddx[2 + 3 * (i + ish)] = a2;
        d2dx2[i + ish] = a3;
      }
    }
    return true;
  }

  // ---- determinante (vmc/determinante.f90:3): ratio + eager SM update ----
  void determinante(int iel, int iflag) {
    orbitalse(iel, iflag);
    int iab = iel < s->nup ? 0 : 1, nel = nel_of(iab), ish = iab == 0 ? 0 : s->nup;
    int ikel = nel * (iel - ish);
    const vector<double> &sl = slmi[iab];
    double ratio = 0;
    for (int j = 0; j < nel; j++) ratio += sl[j + ikel] * orbn[occ(j + ish)];
    detn = detiab[iab] * ratio;
    if (ratio == 0.0) return;
    for (int i = 0; i < nel; i++) {
      if (i + ish == iel) continue;
      int ik = nel * i;
      double sum = 0;
      for (int j = 0; j < nel; j++) sum += sl[j + ik] * orbn[occ(j + ish)];
      sum = sum / ratio;
      for (int j = 0; j < nel; j++) slmin[j + ik] = sl[j + ik] - sl[j + ikel] * sum;
    }
    for (int j = 0; j < nel; j++) slmin[j + ikel] = sl[j + ikel] / ratio;
  }
  // detsav (vmc/detsav.f90:3), single determinant
  void detsav(int iel) {
    int iab = iel < s->nup ? 0 : 1, nel = nel_of(iab);
    for (int j = 0; j < nel * nel; j++) slmi[iab][j] = slmin[j];
    if (s->ndet > 1) {
      // detsav (vmc/detsav.f90:41-82): ymat, aa (virtual columns), wfmat, detiab
      const Sys::MdSpin &m = s->md[iab];
      for (int j = m.ivirt; j < O; j++)
        for (int i = 0; i < nel; i++) {
          ymat[iab][j + (size_t)O * i] = ymatn[j + (size_t)O * i];
          aa[iab][i + (size_t)nel * j] = aan[i + (size_t)nel * j];
        }
      for (int kk = 0; kk < m.nuniq; kk++) {
        const int nr = m.numrep[kk];
        for (int t = 0; t < nr * nr; t++)
          wfmat[iab][(size_t)kk * MEXCIT * MEXCIT + t] = wfmatn[(size_t)kk * MEXCIT * MEXCIT + t];
        ddet[iab][kk] = ddetn[kk];
      }
      for (int k = 0; k < s->ndet; k++) detall[iab][k] = detalln[k];
    }
    detiab[iab] = detn;
    for (int iorb = 0; iorb < O; iorb++) {
      orb[iel + N * iorb] = orbn[iorb];
      for (int k = 0; k < 3; k++) dorb[iorb + O * (iel + N * k)] = dorbn[iorb + O * k];
    }
  }

  // ---- multideterminant pieces ----
  // Excitation determinants of the unique spin-determinants of spin iab
  // from aa: ratio dd(kk) and the inverse of the excitation matrix in wf
  // (multideterminante.f90:69-124, multideterminant.f90:119-215).
  bool md_tables(int iab, const double *aav, double *wf, double *dd) const {
    const Sys::MdSpin &m = s->md[iab];
    const int nel = nel_of(iab);
    for (int kk = 0; kk < m.nuniq; kk++) {
      const int nr = m.numrep[kk];
      const int *rc = &m.irepcol[(size_t)kk * MEXCIT], *ro = &m.ireporb[(size_t)kk * MEXCIT];
      double *w = wf + (size_t)kk * MEXCIT * MEXCIT;
      if (nr == 1) {
        dd[kk] = aav[rc[0] + (size_t)nel * ro[0]];
        w[0] = 1.0 / dd[kk];
      } else if (nr == 2) {
        w[0] = aav[rc[0] + (size_t)nel * ro[0]];
        w[1] = aav[rc[1] + (size_t)nel * ro[0]];
        w[2] = aav[rc[0] + (size_t)nel * ro[1]];
        w[3] = aav[rc[1] + (size_t)nel * ro[1]];
        dd[kk] = w[0] * w[3] - w[2] * w[1];
        const double deti = 1.0 / dd[kk], aux = w[0];
        w[0] = w[3] * deti;
        w[1] = -w[1] * deti;
        w[2] = -w[2] * deti;
        w[3] = aux * deti;
      } else {
        for (int jr = 0; jr < nr; jr++)
          for (int ir = 0; ir < nr; ir++) w[ir + nr * jr] = aav[rc[ir] + (size_t)nel * ro[jr]];
        if (or_matinv(w, nr, &dd[kk]) != 0) return false;
      }
    }
    return true;
  }
  // detiab(k,iab) of every determinant from the reference value and the ratios
  void md_unroll(int iab, double dref, const double *dd, double *dall) const {
    const Sys::MdSpin &m = s->md[iab];
    for (int k = 0; k < s->ndet; k++) dall[k] = dref;
    for (size_t t = 0; t < m.kdet2.size(); t++) dall[m.kdet2[t]] = dall[m.kdet2[t]] * dd[m.kaux2[t]];
  }
  // compute_ymat (vmc/multideterminant.f90:258)
  void compute_ymat(int iab, const double *du, const double *dd_, const double *wf, double *y,
                    const double *cd = nullptr) const {
    if (!cd) cd = s->cdet.data();
    const Sys::MdSpin &m = s->md[iab];
    const int nel = nel_of(iab);
    const double detrefi = 1.0 / (du[0] * dd_[0]);
    std::fill(y, y + (size_t)O * nel, 0.0);
    vector<double> ceq(std::max(m.nuniq, 1), 0.0);
    for (size_t t = 0; t < m.kdet2.size(); t++) {
      const int k = m.kdet2[t], kw = m.kaux2[t];
      const double detall_k = detrefi * du[k] * dd_[k] * cd[k];
      ceq[kw] = ceq[kw] + detall_k;
    }
    for (int kk = 0; kk < m.nuniq; kk++) {
      const int nr = m.numrep[kk];
      const int *rc = &m.irepcol[(size_t)kk * MEXCIT], *ro = &m.ireporb[(size_t)kk * MEXCIT];
      const double *w = wf + (size_t)kk * MEXCIT * MEXCIT;
      for (int ir = 0; ir < nr; ir++)
        for (int jr = 0; jr < nr; jr++) y[ro[jr] + (size_t)O * rc[ir]] += ceq[kk] * w[jr + nr * ir];
    }
  }
  // multideterminante_grad (vmc/multideterminante.f90:149): velocity from Y
  void md_grad(int iel, const double *b, int ldb, double detratio, const double *sl, const double *aav,
               const double *y, double *vel) const {
    vel[0] = vel[1] = vel[2] = 0;
    if (s->ndet == 1) return;
    const int iab = iel < s->nup ? 0 : 1, nel = nel_of(iab), ish = iab == 0 ? 0 : s->nup, jel = iel - ish;
    const Sys::MdSpin &m = s->md[iab];
    vector<double> gmat((size_t)nel * O * 3, 0.0);
    for (int kk = 0; kk < 3; kk++)
      for (int jrep = m.ivirt; jrep < O; jrep++) {
        double dum = 0.0;
        for (int j = 0; j < nel; j++) dum += b[occ(j + ish) + (size_t)ldb * kk] * aav[j + (size_t)nel * jrep];
        dum = b[jrep + (size_t)ldb * kk] - dum;
        for (int irep = m.iactv; irep < nel; irep++)
          gmat[irep + (size_t)nel * (jrep + (size_t)O * kk)] = dum * sl[irep + (size_t)nel * jel];
      }
    for (int kk = 0; kk < 3; kk++) {
      double dum = 0;
      for (int jrep = m.ivirt; jrep < O; jrep++)
        for (int irep = m.iactv; irep < nel; irep++)
          dum += y[jrep + (size_t)O * irep] * gmat[irep + (size_t)nel * (jrep + (size_t)O * kk)];
      vel[kk] = dum * detratio;
    }
  }
  // multideterminante (vmc/multideterminante.f90:3): tables at the proposed
  // position from the updated inverse slmin and the new orbital row
  bool multideterminante(int iel) {
    const int iab = iel < s->nup ? 0 : 1, nel = nel_of(iab), ish = iab == 0 ? 0 : s->nup;
    const Sys::MdSpin &m = s->md[iab];
    for (int jrep = m.ivirt; jrep < O; jrep++)
      for (int irep = 0; irep < nel; irep++) {
        double dum = 0.0;
        for (int i = 0; i < nel; i++) {
          const double o = (i + ish == iel) ? orbn[jrep] : orb[(i + ish) + (size_t)N * jrep];
          dum += slmin[irep + (size_t)nel * i] * o;
        }
        aan[irep + (size_t)nel * jrep] = dum;
      }
    if (!md_tables(iab, aan.data(), wfmatn.data(), ddetn.data())) return false;
    md_unroll(iab, detn, ddetn.data(), detalln.data());
    if (iab == 0) compute_ymat(0, detalln.data(), detall[1].data(), wfmatn.data(), ymatn.data());
    else compute_ymat(1, detall[0].data(), detalln.data(), wfmatn.data(), ymatn.data());
    return true;
  }
  // update_ymat (vmc/multideterminant.f90:562): after the last electron of a
  // spin has been offered its move, the other spin's Y sees the new dets
  void update_ymat(int iel) {
    if (s->ndet == 1) return;
    if ((iel != s->nup - 1 && iel != N - 1) || s->ndn == 0) return;
    const int iab = (iel == s->nup - 1) ? 1 : 0;
    compute_ymat(iab, detall[0].data(), detall[1].data(), wfmat[iab].data(), ymat[iab].data());
  }
  // multideterminant_tmove (dmc/multideterminant_tmove.f90:3, icasula < 0):
  // every quadrature point's T-move element gains the excitations' part,
  // detratio * sum_{jrep >= ivirt, irep >= iactv} ymat(jrep,irep) gmat(irep,jrep)
  // with gmat(irep,jrep) = (b_t(jrep) - sum_j b_t(occ_j) aa(j,jrep)) slmi(irep,jel).
  // psi_D is linear in the moved electron's orbital row, so the element
  // becomes psi_D(x_q)/psi_D(x) * term_radial_jas exactly.
  void md_tmove(double psid) {
    if (s->ndet == 1) return;
    const double detratio = detiab[0] * detiab[1] / psid;
    for (size_t q = 0; q < tq_iel.size(); q++) {
      const int iel = tq_iel[q];
      const int iab = iel < s->nup ? 0 : 1, nel = nel_of(iab), ish = iab == 0 ? 0 : s->nup, jel = iel - ish;
      const Sys::MdSpin &m = s->md[iab];
      const double *bt = btq.data() + (size_t)O * q;
      double sum = 0;
      for (int jrep = m.ivirt; jrep < O; jrep++) {
        double dum = 0;
        for (int j = 0; j < nel; j++) dum = dum + bt[occ(j + ish)] * aa[iab][j + (size_t)nel * jrep];
        dum = bt[jrep] - dum;
        for (int irep = m.iactv; irep < nel; irep++)
          sum = sum + ymat[iab][jrep + (size_t)O * irep] * (dum * slmi[iab][irep + (size_t)nel * jel]);
      }
      tvpsp[((size_t)iel * s->nquad + tq_iq[q]) * M + tq_ic[q]] += sum * detratio;
    }
  }
  // determinante_ref_grad (vmc/determinante.f90:285) with the given slmi column
  void ref_grad(int iel, const double *sl, const double *dorbv /* dorb(norb,3) */, int ldo, double *v) {
    int iab = iel < s->nup ? 0 : 1, nel = nel_of(iab), ish = iab == 0 ? 0 : s->nup;
    int ik = (iel - ish) * nel;
    v[0] = v[1] = v[2] = 0;
    for (int j = 0; j < nel; j++) {
      int o = occ(j + ish);
      v[0] += sl[j + ik] * dorbv[o + ldo * 0];
      v[1] += sl[j + ik] * dorbv[o + ldo * 1];
      v[2] += sl[j + ik] * dorbv[o + ldo * 2];
    }
  }
  // compute_determinante_grad (vmc/determinante.f90:69), single det, iflag_move 1 or 0
  // determinant_psig (vmc/determinant_psig.f90:3) with anormo = 1
  double psig_of(const double *ps) const {
    double g = s->weights_g[0];
    for (int i = 1; i < s->nstates; i++) {
      const double r = ps[i] / ps[0];
      g = g + s->weights_g[i] * r * r;
    }
    return g;
  }
  // compute_determinante_grad with iguiding > 0 (vmc/determinante.f90:150-171,
  // :196-229): sum_i w_i (psi_i/psi_1)^2 (vd_i + vref + vj) / psi2g with each
  // state's multideterminant velocity from its own Y
  void grad_guiding(int iel, int iflag_move, double *vd) {
    const int iab = iel < s->nup ? 0 : 1, ns = s->nstates;
    const double *ps = iflag_move == 1 ? psid_cur.data() : psidn_st.data();
    vector<double> ys((size_t)O * std::max(nel_of(iab), 1));
    double vref[3], vjv[3];
    const double *b;
    const double *sl;
    const double *aav;
    if (iflag_move == 1) {
      double *dt = dorb_tmp.data();
      for (int k = 0; k < 3; k++)
        for (int iorb = 0; iorb < O; iorb++) dt[iorb + O * k] = dorb[iorb + O * (iel + N * k)];
      ref_grad(iel, slmi[iab].data(), dt, O, vref);
      b = dt;
      sl = slmi[iab].data();
      aav = aa[iab].data();
      for (int k = 0; k < 3; k++) vjv[k] = vj[k + 3 * iel];
    } else {
      ref_grad(iel, slmin.data(), dorbn.data(), O, vref);
      b = dorbn.data();
      sl = slmin.data();
      aav = aan.data();
      for (int k = 0; k < 3; k++) vjv[k] = vjn[k + 3 * iel];
    }
    const double dpair = iflag_move == 1 ? detiab[0] * detiab[1] : (iab == 0 ? detn * detiab[1] : detiab[0] * detn);
    const double psi2gi = 1.0 / psig_of(ps);
    vd[0] = vd[1] = vd[2] = 0.0;
    for (int i = 0; i < ns; i++) {
      const double *cd = s->cdet_st.data() + (size_t)i * s->ndet;
      if (iflag_move == 1)
        compute_ymat(iab, detall[0].data(), detall[1].data(), wfmat[iab].data(), ys.data(), cd);
      else if (iab == 0)
        compute_ymat(0, detalln.data(), detall[1].data(), wfmatn.data(), ys.data(), cd);
      else
        compute_ymat(1, detall[0].data(), detalln.data(), wfmatn.data(), ys.data(), cd);
      double vs[3];
      md_grad(iel, b, O, dpair / ps[i], sl, aav, ys.data(), vs);
      const double ratio = ps[i] / ps[0];
      for (int k = 0; k < 3; k++) vd[k] = vd[k] + s->weights_g[i] * ratio * ratio * (vs[k] + vref[k] + vjv[k]);
    }
    for (int k = 0; k < 3; k++) vd[k] = vd[k] * psi2gi;
  }
  void grad(int iel, int iflag_move, double *vd) {
    if (s->iguiding > 0) {
      grad_guiding(iel, iflag_move, vd);
      return;
    }
    const int iab = iel < s->nup ? 0 : 1;
    double vel[3] = {0, 0, 0};
    if (iflag_move == 1) {
      double *dt = dorb_tmp.data();
      for (int k = 0; k < 3; k++)
        for (int iorb = 0; iorb < O; iorb++) dt[iorb + O * k] = dorb[iorb + O * (iel + N * k)];
      double vref[3];
      ref_grad(iel, slmi[iab].data(), dt, O, vref);
      if (s->ndet > 1) {
        const double detratio = detiab[0] * detiab[1] / psido;
        md_grad(iel, dt, O, detratio, slmi[iab].data(), aa[iab].data(), ymat[iab].data(), vel);
      }
      for (int k = 0; k < 3; k++) vd[k] = vel[k] + vref[k] + vj[k + 3 * iel];
    } else {
      double vref[3];
      ref_grad(iel, slmin.data(), dorbn.data(), O, vref);
      if (s->ndet > 1) {
        const double detratio = (iab == 0 ? detn * detiab[1] : detiab[0] * detn) / psidn_md;
        md_grad(iel, dorbn.data(), O, detratio, slmin.data(), aan.data(), ymatn.data(), vel);
      }
      for (int k = 0; k < 3; k++) vd[k] = vel[k] + vref[k] + vjn[k + 3 * iel];
    }
  }

  // ---- psie (vmc/hpsie.f90:3), single det; returns psid ----
  double psie(int iel, const double *x, double &psij, int iflag) {
    distances(iel, x);
    jastrowe(iel, iflag);
    psij = fsumn;
    determinante(iel, iflag);
    if (detn == 0.0) return 0.0;
    int iab = iel < s->nup ? 0 : 1;
    if (s->ndet == 1) return detn * detiab[1 - iab] * s->cdet[0];
    if (!multideterminante(iel)) {
      singular = true;
      return 0.0;
    }
    // determinante_psit (vmc/determinante_psit.f90:4)
    double determ = 0.0;
    for (int k = 0; k < s->ndet; k++) determ += detalln[k] * detall[1 - iab][k] * s->cdet[k];
    psidn_md = determ;
    if (s->iguiding > 0) {
      psidn_st.resize(s->nstates);
      for (int i = 0; i < s->nstates; i++) {
        const double *cd = s->cdet_st.data() + (size_t)i * s->ndet;
        double d = 0.0;
        for (int k = 0; k < s->ndet; k++) d += detalln[k] * detall[1 - iab][k] * cd[k];
        psidn_st[i] = d;
      }
    }
    return determ;
  }

  // ---- ECP: gauss_pot / getvps_gauss (vmc/readps_gauss.f90:6-92) ----
  void gauss_pot(double r, int l /*1-based CHAMP channel*/, int ict, double &vpot, double &dvpot) const {
    double v = 0, dv = 0, rsq = r * r;
    int nt = s->necp_term[ict * CW_MPS_L + (l - 1)];
    for (int i = 0; i < nt; i++) {
      int idx = (ict * CW_MPS_L + (l - 1)) * CW_MGAUSS + i;
      int pw = s->necp_power[idx];
      double p, dpv;
      if (pw != 2) {
        p = std::pow(r, pw - 2);
        dpv = (pw - 2) * p / r;
      } else {
        p = 1.0;
        dpv = 0.0;
      }
      double e;
      if (s->ecp_exponent[idx] * rsq > 7.0e2) e = 0.0;
      else e = s->ecp_coef[idx] * std::exp(-s->ecp_exponent[idx] * rsq);
      v += p * e;
      dv += (dpv - 2 * p * s->ecp_exponent[idx] * r) * e;
    }
    vpot = v;
    dvpot = dv;
  }
  void getvps_gauss(int iel) {
    for (int ic = 0; ic < M; ic++) {
      int ict = s->iwctype[ic];
      double r = std::max(1.0e-10, r_en[iel + N * ic]);
      double ri = 1.0 / r;
      double vpot, dvpot;
      int lp = s->lpot[ict];
      gauss_pot(r, lp, ict, vpot, dvpot);
      vpot = vpot - s->znuc[ict] * ri;
      vps[iel + N * (ic + M * (lp - 1))] = vpot;
      for (int l = 1; l <= lp - 1; l++) {
        gauss_pot(r, l, ict, vpot, dvpot);
        vps[iel + N * (ic + M * (l - 1))] = vpot;
      }
    }
  }
  static double yl0(int l, double costh) {
    if (l == 1) return 1.0;
    if (l == 2) return 3.0 * costh;
    if (l == 3) return 2.5 * (3 * costh * costh - 1);
    return 3.5 * (5 * costh * costh * costh - 3 * costh);
  }
  // psinl / psianl / psibnl (vmc/nonlpsi.f90), ijas=4
  double psinl(double u, double rri, double rrj, int it) const {
    if (rri == s->asymp_r && rrj == s->asymp_r) return 0.0;
    const int nordj = std::max(std::max(s->norda, s->nordb), s->nordc);
    double uu[16], ri[16], rj[16], ss[16], tt[16];
    (void)nordj;
    uu[1] = 1 - s->scalek * u;
    ri[1] = 1 - s->scalek * rri;
    rj[1] = 1 - s->scalek * rrj;
    uu[0] = 1; ri[0] = 1; rj[0] = 1; ss[0] = 2; tt[0] = 1;
    for (int jp = 1; jp <= s->nordc; jp++) {
      uu[jp] = uu[1] * uu[jp - 1];
      ri[jp] = ri[1] * ri[jp - 1];
      rj[jp] = rj[1] * rj[jp - 1];
      ss[jp] = ri[jp] + rj[jp];
      tt[jp] = ri[jp] * rj[jp];
    }
    double v = 0;
    int ll = 0;
    for (int n = 2; n <= s->nordc; n++)
      for (int k = n - 1; k >= 0; k--) {
        int l_hi = (k == 0) ? n - k - 2 : n - k;
        for (int l = l_hi; l >= 0; l--) {
          int m = (n - k - l) / 2;
          if (2 * m == n - k - l) {
            v += s->C(ll, it) * uu[k] * ss[l] * tt[m];
            ll++;
          }
        }
      }
    return v;
  }
  double psianl(double rri, int it) const {
    if (rri == s->asymp_r) return 0.0;
    double v = s->A4(0, it) * rri / (1.0 + s->A4(1, it) * rri) - s->asymp_jasa[it];
    double rrip = rri;
    for (int i = 2; i <= s->norda; i++) {
      rrip *= rri;
      v += s->A4(i, it) * rrip;
    }
    return v;
  }
  double psibnl(double u, int isb, int ipar, double sspinn) const {
    if (u == s->asymp_r) return 0.0;
    double fee = s->B(0, isb) * u / (1 + s->B(1, isb) * u);
    double v = sspinn * fee - s->asymp_jasb[ipar];
    double uu = u;
    for (int i = 2; i <= s->nordb; i++) {
      uu *= u;
      v += s->B(i, isb) * uu;
    }
    return v;
  }

  // ---- nonloc_pot + nonloc (vmc/nonloc_pot.f90:3, vmc/nonloc.f90:5) ----
  void nonloc_pot(const double *x, double &pe, double *vpsp_det) {
    for (int i = 0; i < N; i++) getvps_gauss(i);
    for (int ic = 0; ic < M; ic++)
      for (int i = 0; i < N; i++) pe += vps[i + N * (ic + M * (s->lpot[s->iwctype[ic]] - 1))];
    nonloc(x, vpsp_det);
  }
  void nonloc(const double *x, double *vpsp_det) {
    vpsp_det[0] = vpsp_det[1] = 0;
    std::fill(tvpsp.begin(), tvpsp.end(), 0.0);
    tq_iel.clear(); tq_ic.clear(); tq_iq.clear(); tq_trj.clear(); btq.clear();
    // enumerate quadrature points (iel outer, ic middle, iq inner)
    struct QP { int iel, ic, iq; double costh, x[3]; };
    vector<QP> qp;
    for (int i = 0; i < N; i++)
      for (int ic = 0; ic < M; ic++) {
        int ict = s->iwctype[ic];
        int iskip = 1;
        for (int l = 1; l <= s->lpot[ict] - 1; l++)
          if (std::fabs(vps[i + N * (ic + M * (l - 1))]) > 1.0e-4) iskip = 0;
        if (iskip) continue;
        double ri = 1.0 / r_en[i + N * ic];
        for (int iq = 0; iq < s->nquad; iq++) {
          QP p;
          p.iel = i; p.ic = ic; p.iq = iq;
          p.costh = rvec_en[0 + 3 * (i + N * ic)] * xq[iq] + rvec_en[1 + 3 * (i + N * ic)] * yq[iq] +
                    rvec_en[2 + 3 * (i + N * ic)] * zq[iq];
          p.costh = p.costh * ri;
          p.x[0] = r_en[i + N * ic] * xq[iq] + s->cent[0 + 3 * ic];
          p.x[1] = r_en[i + N * ic] * yq[iq] + s->cent[1 + 3 * ic];
          p.x[2] = r_en[i + N * ic] * zq[iq] + s->cent[2 + 3 * ic];
          qp.push_back(p);
        }
      }
    int nxq = (int)qp.size();
    if (nxq == 0) return;
    // distance_quad (vmc/nonloc.f90:364) + r_en_quad(nxquad,ic)=r_en(i,ic)
    vector<double> rq((size_t)nxq * M), rvq((size_t)3 * nxq * M);
    for (int q = 0; q < nxq; q++)
      for (int jc = 0; jc < M; jc++) {
        double rr = 0;
        for (int k = 0; k < 3; k++) {
          double d = qp[q].x[k] - s->cent[k + 3 * jc];
          rvq[k + 3 * (q + (size_t)nxq * jc)] = d;
        }
        for (int k = 0; k < 3; k++) rr += rvq[k + 3 * (q + (size_t)nxq * jc)] * rvq[k + 3 * (q + (size_t)nxq * jc)];
        rq[q + (size_t)nxq * jc] = std::sqrt(rr);
      }
    for (int q = 0; q < nxq; q++) rq[q + (size_t)nxq * qp[q].ic] = r_en[qp[q].iel + N * qp[q].ic];
    // orbitals_quad (ider=0) + nonlocd_quad
    vector<double> ph((size_t)K * nxq);
    basis_fns(*s, 0, nxq, nxq, rvq.data(), rq.data(), 0, ph.data(), nullptr, nullptr);
    vector<double> det_ratio(nxq), orbq(O), orbq_all(s->ndet > 1 ? (size_t)nxq * O : 0);
    for (int q = 0; q < nxq; q++) {
      for (int iorb = 0; iorb < O; iorb++) {
        double a = 0;
        for (int m = 0; m < K; m++) a += s->COEF(m, iorb) * ph[m + (size_t)K * q];
        orbq[iorb] = a;
      }
      if (s->ndet > 1) std::copy(orbq.begin(), orbq.end(), orbq_all.begin() + (size_t)O * q);
      int iel = qp[q].iel;
      int iab = iel < s->nup ? 0 : 1, nel = nel_of(iab), ish = iab == 0 ? 0 : s->nup;
      int ikel = nel * (iel - ish);
      double r = 0;
      for (int j = 0; j < nel; j++) r += slmi[iab][j + ikel] * orbq[occ(j + ish)];
      det_ratio[q] = r;
    }
    // nonlocj_quad4 (vmc/nonloc.f90:656)
    vector<double> rr_en((size_t)N * M), rr_en_quad(M), ratio_jn(nxq);
    for (int ic = 0; ic < M; ic++)
      for (int i = 0; i < N; i++) scale_dist0(*s, r_en[i + N * ic], rr_en[i + N * ic]);
    for (int q = 0; q < nxq; q++) {
      int iel = qp[q].iel;
      for (int ic = 0; ic < M; ic++) scale_dist0(*s, rq[q + (size_t)nxq * ic], rr_en_quad[ic]);
      double fsum = 0;
      if (N >= 2) {
        for (int jj = 0; jj < N; jj++) {
          if (jj == iel) continue;
          int i = jj < iel ? iel : jj, j = jj < iel ? jj : iel;
          double sspinn = 1;
          int ipar = 0, isb = 0;
          if (i < s->nup || j >= s->nup) {
            if (s->nspin2b == 2) isb = 1;
            else if (s->nocuspb == 0) sspinn = 0.5;
            ipar = 1;
          }
          double dx[3], rij = 0;
          for (int k = 0; k < 3; k++) dx[k] = x[k + 3 * jj] - qp[q].x[k];
          for (int k = 0; k < 3; k++) rij += dx[k] * dx[k];
          rij = std::sqrt(rij);
          double u;
          scale_dist0(*s, rij, u);
          double f = psibnl(u, isb, ipar, sspinn);
          if (s->nordc > 1)
            for (int ic = 0; ic < M; ic++) f += psinl(u, rr_en_quad[ic], rr_en[jj + N * ic], s->iwctype[ic]);
          fsum = fsum + f - fso[FI(i, j, N)];
        }
      }
      double fen = 0;
      for (int ic = 0; ic < M; ic++) fen += psianl(rr_en_quad[ic], s->iwctype[ic]);
      fsum = fsum + fen - fso[FI(iel, iel, N)];
      ratio_jn[q] = fsum;
    }
    for (int q = 0; q < nxq; q++) {
      int iel = qp[q].iel, ic = qp[q].ic, ict = s->iwctype[ic];
      int iab = iel < s->nup ? 0 : 1;
      double term = 0;
      for (int l = 1; l <= s->lpot[ict] - 1; l++) term += yl0(l, qp[q].costh) * vps[iel + N * (ic + M * (l - 1))];
      double trj = term * s->wq[qp[q].iq] * std::exp(ratio_jn[q]);
      vpsp_det[iab] += trj * det_ratio[q];
      // transition matrix element of a T-move to this point (nonloc.f90:296-298)
      tvpsp[((size_t)iel * s->nquad + qp[q].iq) * M + ic] = det_ratio[q] * trj;
      tq_iel.push_back(iel);
      tq_ic.push_back(ic);
      tq_iq.push_back(qp[q].iq);
      tq_trj.push_back(trj);
      if (s->ndet > 1)  // b_t (nonloc.f90:299-301) for multideterminant_tmove
        for (int iorb = 0; iorb < O; iorb++) btq.push_back(orbq_all[iorb + (size_t)O * q] * trj);
      // pseudopotential contribution to the B matrix (nonloc.f90:271-273)
      if (s->ndet > 1)
        for (int iorb = 0; iorb < O; iorb++) bmat[iorb + (size_t)O * iel] += trj * orbq_all[iorb + (size_t)O * q];
    }
  }

  // pot_local (vmc/pot_local.f90:3)
  double pot_local() const {
    double pe = s->pecent;
    if (s->nloc == 0)
      for (int i = 0; i < N; i++)
        for (int ic = 0; ic < M; ic++) pe += -s->znuc[s->iwctype[ic]] / r_en[i + N * ic];
    int ij = 0;
    for (int i = 1; i < N; i++)
      for (int j = 0; j < i; j++, ij++) pe += 1 / r_ee[ij];
    return pe;
  }

  // multideterminant_hpsi (vmc/multideterminant.f90:3) with bxmatrix
  // (vmc/bxmatrices.f90:3) and the Y-matrix energy of hpsi (vmc/hpsi.f90:220-238):
  // aa = A^-1 Phi, tildem = A^-1 B - X Phi with X = A^-1 B_occ A^-1, the
  // excitation tables, every detiab, both Y matrices, psid and the energy
  // corrections denergy / dekin.
  bool multideterminant_hpsi(double &psid, double &denergy, double &dekin) {
    vector<double> tild[2], tildk[2];
    for (int iab = 0; iab < 2; iab++) {
      const int nel = nel_of(iab), ish = iab == 0 ? 0 : s->nup;
      tild[iab].assign((size_t)std::max(nel, 1) * O, 0.0);
      tildk[iab].assign((size_t)std::max(nel, 1) * O, 0.0);
      if (nel == 0) continue;
      const vector<double> &sl = slmi[iab];
      // xmat from B restricted to the reference orbitals (multiply_slmi_mderiv_simple)
      auto xmat_of = [&](const vector<double> &bb, vector<double> &xm) {
        vector<double> bt((size_t)nel * nel), work(nel);
        for (int i = 0; i < nel; i++)
          for (int j = 0; j < nel; j++) bt[j + (size_t)nel * i] = bb[occ(j + ish) + (size_t)O * (i + ish)];
        xm.assign((size_t)nel * nel, 0.0);
        for (int mm = 0; mm < nel; mm++) {
          for (int j = 0; j < nel; j++) {
            work[j] = 0;
            for (int i = 0; i < nel; i++) work[j] = work[j] + bt[i + (size_t)nel * j] * sl[i + (size_t)nel * mm];
          }
          for (int n = 0; n < nel; n++) {
            double x = 0;
            for (int j = 0; j < nel; j++) x = x + work[j] * sl[n + (size_t)nel * j];
            xm[mm + (size_t)nel * n] = x;
          }
        }
      };
      vector<double> xm, xmk;
      xmat_of(bmat, xm);
      xmat_of(bkin, xmk);
      for (int jrep = 0; jrep < O; jrep++)
        for (int irep = 0; irep < nel; irep++) {
          double d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0;
          for (int i = 0; i < nel; i++) {
            const double o = orb[(i + ish) + (size_t)N * jrep];
            d1 += sl[irep + (size_t)nel * i] * o;
            d2 += sl[irep + (size_t)nel * i] * bmat[jrep + (size_t)O * (i + ish)];
            d3 += xm[i + (size_t)nel * irep] * o;
            d4 += sl[irep + (size_t)nel * i] * bkin[jrep + (size_t)O * (i + ish)];
            d5 += xmk[i + (size_t)nel * irep] * o;
          }
          aa[iab][irep + (size_t)nel * jrep] = d1;
          tild[iab][irep + (size_t)nel * jrep] = d2 - d3;
          tildk[iab][irep + (size_t)nel * jrep] = d4 - d5;
        }
    }
    for (int iab = 0; iab < 2; iab++) {
      if (!md_tables(iab, aa[iab].data(), wfmat[iab].data(), ddet[iab].data())) return false;
      md_unroll(iab, detiab[iab], ddet[iab].data(), detall[iab].data());
    }
    compute_ymat(0, detall[0].data(), detall[1].data(), wfmat[0].data(), ymat[0].data());
    if (s->ndn > 0) compute_ymat(1, detall[0].data(), detall[1].data(), wfmat[1].data(), ymat[1].data());
    psid = 0.0;
    for (int k = 0; k < s->ndet; k++) psid = psid + detall[0][k] * detall[1][k] * s->cdet[k];
    // optci_deloc (vmc/optci.f90:49-51): ciprim = D_k / psid, here times the
    // orbital-order sign so that it is d ln psi / d c_k of the input coefficients
    ci_o.resize(s->ndet);
    for (int k = 0; k < s->ndet; k++) ci_o[k] = s->detsign[k] * (detall[0][k] * detall[1][k] / psid);
    denergy = 0;
    dekin = 0;
    for (int iab = 0; iab < 2; iab++) {
      const int nel = nel_of(iab);
      const Sys::MdSpin &m = s->md[iab];
      for (int jrep = m.ivirt; jrep < O; jrep++)
        for (int irep = m.iactv; irep < nel; irep++) {
          denergy = denergy + ymat[iab][jrep + (size_t)O * irep] * tild[iab][irep + (size_t)nel * jrep];
          dekin = dekin + ymat[iab][jrep + (size_t)O * irep] * tildk[iab][irep + (size_t)nel * jrep];
        }
    }
    denergy = denergy * detiab[0] * detiab[1] / psid;
    dekin = dekin * detiab[0] * detiab[1] / psid;
    // further states (determinante.f90:134-230 with nstates > 1): the same
    // excitation ratios and tildem, each state's own Y and psi_D
    psid_st[0] = psid;
    den_st[0] = denergy;
    dek_st[0] = dekin;
    for (int st = 1; st < s->nstates; st++) {
      const double *cd = s->cdet_st.data() + (size_t)st * s->ndet;
      vector<double> ys[2];
      for (int iab = 0; iab < 2; iab++) {
        ys[iab].assign((size_t)O * std::max(nel_of(iab), 1), 0.0);
        if (nel_of(iab) > 0)
          compute_ymat(iab, detall[0].data(), detall[1].data(), wfmat[iab].data(), ys[iab].data(), cd);
      }
      double ps = 0.0;
      for (int k = 0; k < s->ndet; k++) ps = ps + detall[0][k] * detall[1][k] * cd[k];
      double de = 0, dk = 0;
      for (int iab = 0; iab < 2; iab++) {
        const int nel = nel_of(iab);
        const Sys::MdSpin &m = s->md[iab];
        for (int jrep = m.ivirt; jrep < O; jrep++)
          for (int irep = m.iactv; irep < nel; irep++) {
            de = de + ys[iab][jrep + (size_t)O * irep] * tild[iab][irep + (size_t)nel * jrep];
            dk = dk + ys[iab][jrep + (size_t)O * irep] * tildk[iab][irep + (size_t)nel * jrep];
          }
      }
      psid_st[st] = ps;
      den_st[st] = de * detiab[0] * detiab[1] / ps;
      dek_st[st] = dk * detiab[0] * detiab[1] / ps;
    }
    return true;
  }
  vector<double> den_st = vector<double>(1), dek_st = vector<double>(1);

  // ---- hpsi (vmc/hpsi.f90:3), single det; returns false if singular ----
  bool hpsi(const double *coord, double &psid, double &psij, double &ekin, double &energy,
            double *extra = nullptr) {
    const double hb = 0.5;
    distances(-1, coord);
    double pe = pot_local();
    jastrow_factor4();
    vj = fjo;
    double d2j = d2o;
    psij = fsumo;
    if (!determinant()) return false;
    if (s->ndet > 1) {
      // compute_bmatrices_kin (vmc/determinant.f90:196): B of the kinetic operator
      for (int i = 0; i < N; i++)
        for (int iorb = 0; iorb < O; iorb++) {
          const double bk = -hb * (ddorb[iorb + O * i] + 2 * (vj[0 + 3 * i] * dorb[iorb + O * (i + N * 0)] +
                                                            vj[1 + 3 * i] * dorb[iorb + O * (i + N * 1)] +
                                                            vj[2 + 3 * i] * dorb[iorb + O * (i + N * 2)]));
          bkin[iorb + (size_t)O * i] = bk;
          bmat[iorb + (size_t)O * i] = bk;
        }
    }
    double vpsp[2] = {0, 0};
    if (s->nloc > 0) nonloc_pot(coord, pe, vpsp);
    double ekin_det[2], eloc_det[2];
    for (int iab = 0; iab < 2; iab++) {
      int nel = nel_of(iab), ish = iab == 0 ? 0 : s->nup;
      ekin_det[iab] = 0;
      for (int i = 0; i < nel; i++) {
        int e = i + ish;
        double tmp = -hb * (d2dx2[e] + 2.0 * (vj[0 + 3 * e] * ddx[0 + 3 * e] + vj[1 + 3 * e] * ddx[1 + 3 * e] +
                                              vj[2 + 3 * e] * ddx[2 + 3 * e]));
        ekin_det[iab] += tmp;
      }
      eloc_det[iab] = ekin_det[iab] + vpsp[iab];
    }
    double ekin_other = -hb * d2j;
    for (int i = 0; i < N; i++)
      ekin_other += -hb * (vj[0 + 3 * i] * vj[0 + 3 * i] + vj[1 + 3 * i] * vj[1 + 3 * i] + vj[2 + 3 * i] * vj[2 + 3 * i]);
    double e_other = ekin_other + pe;
    double denergy = 0, dekin = 0;
    if (s->ndet == 1) {
      psid = detiab[0] * detiab[1] * s->cdet[0];
    } else {
      den_st.resize(s->nstates);
      dek_st.resize(s->nstates);
      psid_st.resize(s->nstates);
      if (!multideterminant_hpsi(psid, denergy, dekin)) return false;
    }
    energy = denergy + eloc_det[0] + eloc_det[1] + e_other;
    ekin = dekin + ekin_det[0] + ekin_det[1] + ekin_other;
    if (s->nstates > 1) {
      e_st.resize(s->nstates);
      ekin_st.resize(s->nstates);
      for (int st = 0; st < s->nstates; st++) {
        e_st[st] = den_st[st] + eloc_det[0] + eloc_det[1] + e_other;
        ekin_st[st] = dek_st[st] + ekin_det[0] + ekin_det[1] + ekin_other;
      }
    }
    if (extra) {
      extra[0] = pe;
      extra[1] = vpsp[0] + vpsp[1];
    }
    return true;
  }

  // rotqua (vmc/rotqua.f90:357)
  void rotqua() {
    double x1, x2, x3, xsum;
    do {
      x1 = 1.0 - 2.0 * rng.uniform();
      x2 = 1.0 - 2.0 * rng.uniform();
      xsum = x1 * x1 + x2 * x2;
    } while (xsum >= 1.0);
    double xsum2 = 2.0 * std::sqrt(std::fabs(1.0 - xsum));
    x1 = x1 * xsum2;
    x2 = x2 * xsum2;
    x3 = 1.0 - 2.0 * xsum;
    double theta = std::acos(x3), sthet = std::sin(theta), cfi, sfi;
    if (sthet < 1.0e-05) {
      cfi = 1; sfi = 0; x1 = 0; x2 = 0; x3 = 1; sthet = 0;
    } else {
      cfi = x1 / sthet;
      sfi = x2 / sthet;
    }
    double yy1 = x3 * cfi, yy2 = x3 * sfi, yy3 = -sthet;
    double zz1 = -sfi, zz2 = cfi, zz3 = 0.0;
    double u1, u2, usum;
    do {
      u1 = rng.uniform() * 2.0 - 1.0;
      u2 = rng.uniform() * 2.0 - 1.0;
      usum = u1 * u1 + u2 * u2;
    } while (usum >= 1.0);
    double uu = std::sqrt(usum);
    u1 = u1 / uu;
    u2 = u2 / uu;
    double y1 = yy1 * u1 + zz1 * u2, y2 = yy2 * u1 + zz2 * u2, y3 = yy3 * u1 + zz3 * u2;
    double z1 = yy1 * u2 - zz1 * u1, z2 = yy2 * u2 - zz2 * u1, z3 = yy3 * u2 - zz3 * u1;
    for (int iq = 0; iq < s->nquad; iq++) {
      xq[iq] = s->xq0[iq] * x1 + s->yq0[iq] * y1 + s->zq0[iq] * z1;
      yq[iq] = s->xq0[iq] * x2 + s->yq0[iq] * y2 + s->zq0[iq] * z2;
      zq[iq] = s->xq0[iq] * x3 + s->yq0[iq] * y3 + s->zq0[iq] * z3;
    }
  }

  // zerest (vmc/acuest.f90:179): initial hpsi with the unrotated grid
  bool zerest() {
    zero_estimators();
    xq = s->xq0; yq = s->yq0; zq = s->zq0;
    double psid, psij, ekin, e;
    if (!hpsi(xold.data(), psid, psij, ekin, e)) return false;
    psido = psid; psijo = psij; eold = e; ekino = ekin;
    psi2o = 2 * (std::log(std::fabs(psido)) + psijo);
    if (s->iguiding > 0) {  // zerest after guiding (vmc/acuest.f90:273-278)
      psid_cur = psid_st;
      psi2o = std::log(std::fabs(psig_of(psid_cur.data()))) + 2 * (std::log(std::fabs(psido)) + psijo);
    }
    distances(-1, xold.data());
    for (int i = 0; i < N; i++) {
      rmino[i] = 99.0e9;
      for (int ic = 0; ic < M; ic++)
        if (r_en[i + N * ic] < rmino[i]) {
          rmino[i] = r_en[i + N * ic];
          nearesto[i] = ic;
        }
      for (int k = 0; k < 3; k++) rvmino[k + 3 * i] = rvec_en[k + 3 * (i + N * nearesto[i])];
    }
    xnew = xold;
    return true;
  }

  double thetamx(double r, double z) const {
    return s->deltat + (2.0 - s->deltat) / (1.0 + (z * r) * (z * r));
  }

  // ---- metrop6 (vmc/metrop_mov1_slat.f90:3) ----
  bool metrop6();
};

// gammai (vmc/gammai.f90:3)
double gammai(double a, double x, double xae, int &iflag) {
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
  } else {
    iflag = -1;
    double a0 = 1, a1 = x, b0 = 0, b1 = 1, fac = 1, g = 0;
    int iter = std::max(20 + (int)std::lround(a - x), 7);
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
}

// Transition-area integral used twice in metrop6 (forward and reverse).
double t_area(double zeta, double co, double rbot, double rtop, double bot) {
  const double d5b2 = 2.5, d2b3 = .666666666666667, g5b2 = 1.329340388179137;
  double rzero = -1.0 / co;
  double zrbot = zeta * rbot, zrtop = zeta * rtop;
  double zebot = std::sqrt(zrbot * zrbot * zrbot) * std::exp(-zrbot);
  double zetop = std::sqrt(zrtop * zrtop * zrtop) * std::exp(-zrtop);
  int iflagb, iflagt, iflagz;
  double g52bot = gammai(d5b2, zrbot, zrbot * zebot, iflagb);
  double g52top = gammai(d5b2, zrtop, zrtop * zetop, iflagt);
  if (rzero < rbot || rzero > rtop) {
    double g52dif = (iflagb * iflagt == 1) ? g52top - g52bot : g52top - g52bot + g5b2;
    double g32dif = d2b3 * (g52dif + zetop - zebot);
    return std::fabs(g32dif + co * g52dif / zeta) / (bot * std::sqrt(zeta * zeta * zeta));
  }
  double zrzer = zeta * rzero;
  double zezer = std::sqrt(zrzer * zrzer * zrzer) * std::exp(-zrzer);
  double g52zer = gammai(d5b2, zrzer, zrzer * zezer, iflagz);
  double g52dif1 = (iflagb * iflagz == 1) ? g52zer - g52bot : g52zer - g52bot + g5b2;
  double g32dif1 = d2b3 * (g52dif1 + zezer - zebot);
  double g52dif2 = (iflagt * iflagz == 1) ? g52top - g52zer : g52top - g52zer + g5b2;
  double g32dif2 = d2b3 * (g52dif2 + zetop - zezer);
  return (std::fabs(g32dif1 + co * g52dif1 / zeta) + std::fabs(g32dif2 + co * g52dif2 / zeta)) /
         (bot * std::sqrt(zeta * zeta * zeta));
}

bool Walker::metrop6() {
  const double zero = 0, one = 1, two = 2, four = 4, half = 0.5, d3b2 = 1.5, eps = 1.0e-10;
  const double deltar = s->deltar, fbias = s->fbias;
  double deltri = one / deltar;
  for (int i = 0; i < N; i++) {
    double *vo = &vold[3 * i];
    grad(i, 1, vo);
    double fxop = one;
    int nearo = nearesto[i];
    double zcusp = (s->nloc == 0) ? s->znuc[s->iwctype[nearo]] : zero;
    rmino[i] = std::sqrt(rvmino[0 + 3 * i] * rvmino[0 + 3 * i] + rvmino[1 + 3 * i] * rvmino[1 + 3 * i] +
                         rvmino[2 + 3 * i] * rvmino[2 + 3 * i]);
    double rbot = rmino[i] * deltri, rtop = rmino[i] * deltar;
    double voldr = zero;
    for (int ic = 0; ic < 3; ic++) voldr += vo[ic] * rvmino[ic + 3 * i];
    voldr = voldr / rmino[i];
    double voldp = zero, xaxis[3], yaxis[3], zaxis[3];
    for (int ic = 0; ic < 3; ic++) {
      zaxis[ic] = rvmino[ic + 3 * i] / rmino[i];
      xaxis[ic] = vo[ic] - voldr * zaxis[ic];
      voldp += xaxis[ic] * xaxis[ic];
    }
    voldp = std::sqrt(voldp);
    if (voldp < eps) {
      xaxis[0] = eps * (one - zaxis[0] * zaxis[0]);
      xaxis[1] = eps * (-zaxis[0] * zaxis[1]);
      xaxis[2] = eps * (-zaxis[0] * zaxis[2]);
      voldp = eps * std::sqrt(one - zaxis[0] * zaxis[0]);
    }
    for (int ic = 0; ic < 3; ic++) xaxis[ic] = xaxis[ic] / voldp;
    double znear = s->znuc[s->iwctype[nearo]];
    voldr = std::max(voldr, -2 * znear);
    yaxis[0] = zaxis[1] * xaxis[2] - zaxis[2] * xaxis[1];
    yaxis[1] = zaxis[2] * xaxis[0] - zaxis[0] * xaxis[2];
    yaxis[2] = zaxis[0] * xaxis[1] - zaxis[1] * xaxis[0];
    voldp = voldp * fbias;
    double root = (zcusp + voldr) * (zcusp + voldr - four / rmino[i]), zeta;
    if (root >= zero) {
      root = std::sqrt(root);
      zeta = half * (zcusp - voldr - root);
      if (zeta <= zero) zeta = half * (zcusp - voldr + root);
      if (zeta <= zero) zeta = eps;
    } else {
      zeta = (voldr < zero) ? -voldr - eps : one;
    }
    double co = (zeta + voldr) / (one - (zeta + voldr) * rmino[i]);
    root = std::sqrt((d3b2 * co - zeta) * (d3b2 * co - zeta) + two * zeta * co);
    double rmax1 = (d3b2 * co - zeta + root) / (two * zeta * co);
    if (rmax1 < rbot) rmax1 = rbot;
    if (rmax1 > rtop) rmax1 = rtop;
    double fmax = std::sqrt(rmax1) * std::fabs(one + co * rmax1) * std::exp(-zeta * rmax1);
    if (co < zero) {
      double rmax2 = (d3b2 * co - zeta - root) / (two * zeta * co);
      if (rmax2 < rbot) rmax2 = rbot;
      if (rmax2 > rtop) rmax2 = rtop;
      double fmax2 = std::sqrt(rmax2) * std::fabs(one + co * rmax2) * std::exp(-zeta * rmax2);
      fmax = std::max(fmax, fmax2);
    }
    double bot = std::sqrt(rmino[i]) * std::fabs(one + co * rmino[i]) * std::exp(-zeta * rmino[i]);
    double rtry, top;
    for (;;) {
      rtry = ((deltar - deltri) * rng.uniform() + deltri) * rmino[i];
      top = std::sqrt(rtry) * std::fabs(one + co * rtry) * std::exp(-zeta * rtry);
      double ratio = top / fmax;
      if (ratio > rng.uniform()) break;
    }
    fxop = fxop * top / bot;
    double areao = t_area(zeta, co, rbot, rtop, bot);
    double raver = half * (rmino[i] + rtry);
    double deltt = thetamx(raver, znear);
    double costht = one - deltt * rng.uniform();
    double zprime = rtry * costht;
    double sintht = std::sqrt(one - costht * costht);
    areao = areao * deltt;
    double term = std::min(voldp * raver * sintht, one);
    fmax = one + term;
    double phitry, cosphi;
    for (;;) {
      phitry = PI * rng.uniform();
      cosphi = std::cos(phitry);
      top = one + term * cosphi;
      if (top > rng.uniform() * fmax) break;
    }
    fxop = fxop * top;
    double xprime = rtry * sintht * std::cos(phitry);
    double yprime = std::sqrt(std::max(zero, rtry * rtry - xprime * xprime - zprime * zprime));
    if (rng.uniform() < half) yprime = -yprime;
    for (int ic = 0; ic < 3; ic++) {
      rvminno[ic + 3 * i] = xaxis[ic] * xprime + yaxis[ic] * yprime + zaxis[ic] * zprime;
      xnew[ic + 3 * i] = rvminno[ic + 3 * i] + s->cent[ic + 3 * nearo];
    }
    rminno[i] = rtry;
    // geometrical rejection
    rminn[i] = 99.0e9;
    for (int j = 0; j < M; j++) {
      double dist = zero;
      for (int ic = 0; ic < 3; ic++) dist += (xnew[ic + 3 * i] - s->cent[ic + 3 * j]) * (xnew[ic + 3 * i] - s->cent[ic + 3 * j]);
      if (dist < rminn[i]) {
        rminn[i] = dist;
        nearestn[i] = j;
      }
    }
    int nearn = nearestn[i];
    rminn[i] = std::sqrt(rminn[i]);
    rminon[i] = zero;
    double dot = zero;
    for (int ic = 0; ic < 3; ic++) {
      rvminn[ic + 3 * i] = xnew[ic + 3 * i] - s->cent[ic + 3 * nearn];
      rvminon[ic + 3 * i] = xold[ic + 3 * i] - s->cent[ic + 3 * nearn];
      rminon[i] += rvminon[ic + 3 * i] * rvminon[ic + 3 * i];
      dot += rvminn[ic + 3 * i] * rvminon[ic + 3 * i];
    }
    rminon[i] = std::sqrt(rminon[i]);
    dot = dot / (rminn[i] * rminon[i]);
    costht = dot;
    sintht = std::sqrt(one - costht * costht);
    double ravern = half * (rminn[i] + rminon[i]);
    delttn[i] = thetamx(ravern, s->znuc[s->iwctype[nearn]]);
    int igeometrical = 0;
    double p = zero, psi2n = 0, psidn = 0, psijn = 0;
    double vn[3] = {0, 0, 0};
    if (rminon[i] > rminn[i] * deltar || dot < one - delttn[i]) {
      igeometrical = 1;
      p = zero;
    } else {
      double rratio = rminno[i] / rminon[i];
      psidn = psie(i, xnew.data(), psijn, 0);
      if (psidn == 0.0) {
        // psi2g computed as 1 (iguiding=0): only psid==0 (detn==0) rejects
      }
      bool zero_psi = (detn == 0.0);
      if (zero_psi) {
        p = zero;
      } else {
        grad(i, 0, vn);
        for (int k = 0; k < 3; k++) vnew[k + 3 * i] = vn[k];
        const double psi2g = s->iguiding > 0 ? psig_of(psidn_st.data()) : 1.0;
        psi2n = std::log(std::fabs(psi2g)) + 2 * (std::log(std::fabs(psidn)) + psijn);
        double fxnp = one;
        rbot = rminn[i] * deltri;
        rtop = rminn[i] * deltar;
        double vnewr = zero;
        for (int ic = 0; ic < 3; ic++) vnewr += vn[ic] * rvminn[ic + 3 * i];
        vnewr = vnewr / rminn[i];
        double vnewp = zero;
        for (int ic = 0; ic < 3; ic++) {
          xaxis[ic] = vn[ic] - vnewr * rvminn[ic + 3 * i] / rminn[i];
          vnewp += xaxis[ic] * xaxis[ic];
        }
        vnewp = std::sqrt(vnewp);
        if (vnewp < eps) {
          xaxis[0] = eps * (one - rvminn[0 + 3 * i] * rvminn[0 + 3 * i]);
          xaxis[1] = eps * (-rvminn[0 + 3 * i] * rvminn[1 + 3 * i]);
          xaxis[2] = eps * (-rvminn[0 + 3 * i] * rvminn[2 + 3 * i]);
          vnewp = eps * std::sqrt(one - rvminn[0 + 3 * i] * rvminn[0 + 3 * i] * (two - rminn[i] * rminn[i]));
        }
        for (int ic = 0; ic < 3; ic++) xaxis[ic] = xaxis[ic] / vnewp;
        double zc = (s->nloc == 0) ? s->znuc[s->iwctype[nearn]] : zero;
        vnewr = std::max(vnewr, -2 * s->znuc[s->iwctype[nearn]]);
        vnewp = vnewp * fbias;
        root = (zc + vnewr) * (zc + vnewr - four / rminn[i]);
        if (root >= zero) {
          root = std::sqrt(root);
          zeta = half * (zc - vnewr - root);
          if (zeta <= zero) zeta = half * (zc - vnewr + root);
          if (zeta <= zero) zeta = eps;
        } else {
          zeta = (vnewr < zero) ? -vnewr - eps : one;
        }
        co = (zeta + vnewr) / (one - (zeta + vnewr) * rminn[i]);
        bot = std::sqrt(rminn[i]) * std::fabs(one + co * rminn[i]) * std::exp(-zeta * rminn[i]);
        top = std::sqrt(rminon[i]) * std::fabs(one + co * rminon[i]) * std::exp(-zeta * rminon[i]);
        fxnp = fxnp * top / bot;
        double arean = t_area(zeta, co, rbot, rtop, bot);
        arean = arean * delttn[i];
        term = std::min(vnewp * ravern * sintht, one);
        cosphi = zero;
        double rnorm = zero;
        for (int ic = 0; ic < 3; ic++) {
          double term2 = rvminon[ic + 3 * i] / rminon[i] - costht * rvminn[ic + 3 * i] / rminn[i];
          rnorm += term2 * term2;
          cosphi += term2 * xaxis[ic];
        }
        cosphi = cosphi / std::sqrt(rnorm);
        fxnp = fxnp * (one + term * cosphi);
        p = rratio * rratio * std::exp(psi2n - psi2o) * std::fabs((fxnp * areao) / (fxop * arean));
        p = std::min(one, p);
      }
    }
    if (rng.uniform() < p) {
      rmino[i] = rminn[i];
      nearesto[i] = nearestn[i];
      psi2o = psi2n;
      for (int ic = 0; ic < 3; ic++) {
        xold[ic + 3 * i] = xnew[ic + 3 * i];
        rvmino[ic + 3 * i] = rvminn[ic + 3 * i];
      }
      psido = psidn;
      psijo = psijn;
      if (s->iguiding > 0) psid_cur = psidn_st;
      acc = acc + one;
      jassav(i, 0);
      detsav(i);
    } else {
      for (int ic = 0; ic < 3; ic++) xnew[ic + 3 * i] = xold[ic + 3 * i];
      if (igeometrical == 0) distancese_restore(i);
    }
    update_ymat(i);
    if (singular) return false;
  }
  // primary configuration: full recompute
  double ekin, e;
  if (!hpsi(xold.data(), psido, psijo, ekin, e)) return false;
  eold = e;
  ekino = ekin;
  psi2o = 2 * (std::log(std::fabs(psido)) + psijo);
  double psi2g = 1.0;
  if (s->iguiding > 0) {  // metrop6 :652-657, :732
    psid_cur = psid_st;
    psi2g = psig_of(psid_cur.data());
    psi2o = std::log(std::fabs(psi2g)) + 2 * (std::log(std::fabs(psido)) + psijo);
  }
  double wtg_sqrt = psido / psido * std::exp(psijo - psijo) / std::sqrt(psi2g);
  double wtg = wtg_sqrt * wtg_sqrt;
  esum1 = eold;
  wsum += wtg;
  esum += eold * wtg;
  pesum += (eold - ekino) * wtg;
  tpbsum += ekino * wtg;
  // acues1 + acusig
  ecum1 += esum1 * wtg;
  ecm21 += esum1 * esum1 * wtg;
  ecum1s += eold * wtg;
  ecm21s += eold * eold * wtg;
  // every state, reweighted to the sampled distribution (metrop6 :678-690)
  for (int st = 0; s->nstates > 1 && st < s->nstates; st++) {
    const double ws = psid_st[st] / psid_st[0] * std::exp(psijo - psijo) / std::sqrt(psi2g);
    const double wt = ws * ws;
    wsum_st[st] += wt;
    esum_st[st] += e_st[st] * wt;
    pesum_st[st] += (e_st[st] - ekin_st[st]) * wt;
    tpbsum_st[st] += ekin_st[st] * wt;
  }
  // SR sums of the CI derivatives (optwf_store's sr_o contracted per sample)
  if (opt_ci) {
    const int nd = s->ndet;
    if (sr_o.empty()) {
      sr_o.assign(nd, 0.0);
      sr_eo.assign(nd, 0.0);
      sr_oo.assign((size_t)nd * nd, 0.0);
    }
    sr_w += wtg;
    for (int k = 0; k < nd; k++) {
      sr_o[k] += wtg * ci_o[k];
      sr_eo[k] += wtg * eold * ci_o[k];
      for (int l = 0; l < nd; l++) sr_oo[(size_t)k * nd + l] += wtg * ci_o[k] * ci_o[l];
    }
  }
  return true;
}

struct Walkers {
  const Sys *s;
  vector<Walker> w;
  // global (rank-0) cumulative estimators after acuest_reduce
  double ecum = 0, ecm2 = 0, wcum = 0, pecum = 0, tpbcum = 0, pecm2 = 0, tpbcm2 = 0, acc = 0;
  double ecum1 = 0, ecm21 = 0, ecum1s = 0, ecm21s = 0;
  vector<double> wcum_st, ecum_st, ecm2_st, pecum_st, tpbcum_st;  // per state (acuest per istate)
  long iblk = 0, passes = 0;
  int nstep_last = 0;
  bool failed = false;
};


// ===========================================================================
// DMC: dmc_ps (dmc/dmc_ps_mov1.f90:4), calculate_fratio / calculate_reweight
// (dmc/branching.f90:27,111), splitj (dmc/splitj.f90:3), acues1
// (dmc/acues1.f90:3) and the block sums of acuest (dmc/acuest.f90).
// One population, as one CHAMP rank in dmc_one_mpi1.  Each walker slot owns
// a random stream for its moves; rotqua and splitj draw from the population
// stream, as CHAMP's rank does.
// ===========================================================================
struct DmcParams {
  double tau, etrial;
  int nconf, mwalk, nfprod;
  int icasula = 0;  // 0: no T-moves, -1: one T-move per walker and step (dmc_ps :701-795)
};

struct DmcPop {
  const Sys *s;
  DmcParams prm;
  vector<Walker> w;          // slots 0..mwalk-1, active 0..nwalk-1
  int nwalk;
  Rng pop;
  double eest, eigv, wdsumo, fprod;
  vector<double> ff;
  vector<double> wt, fratio;
  vector<int> iage;
  long ipass = 0;
  // per-step and per-block sums
  double wsum1 = 0, esum1 = 0, pesum = 0, tpbsum = 0, tausum = 0;
  double wgsum = 0, egsum = 0, wgcum = 0, egcum = 0, wgcm2 = 0, egcm2 = 0, taucum = 0;
  double pecum = 0, tpbcum = 0;
  double acc = 0, trymove = 0;
  long nacc = 0, nodecr = 0, nbrnch = 0, iblk = 0, nmove_casula = 0;
  vector<int> tmoved;  // [mwalk] walker made a T-move in this step
  bool failed = false;
};

bool tmove_walker(DmcPop &P, int iw);

double gauss_draw(Rng &r) {
  // gauss (vmc/gauss.f90:3): one normal from two uniforms, cos draw first
  double g = std::cos(2 * PI * r.uniform());
  return g * std::sqrt(-2 * std::log(r.uniform()));
}

// grad for every electron after hpsi (dmc_ps :516): vold(3,nelec)
void vold_all(Walker &w) {
  for (int i = 0; i < w.N; i++) w.grad(i, 1, &w.vold[3 * i]);
}

// nearest centre of a point: first minimum of the squared distance
int nearest_centre(const Sys *s, const double *x) {
  double best = 1.0e100;
  int iw = 0;
  for (int ic = 0; ic < s->M; ic++) {
    const double d0 = x[0] - s->cent[3 * ic], d1 = x[1] - s->cent[3 * ic + 1], d2 = x[2] - s->cent[3 * ic + 2];
    const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
    if (r2 < best) {
      best = r2;
      iw = ic;
    }
  }
  return iw;
}

// dmc_eloc_cutoff (dmc/branching.f90:201-275) -> fratio (icut_e=0).
// Pseudopotential runs (dmc_ps passes adrift = 0.5): the plain averaged
// drift; all-electron runs (dmc_ae passes adrift0 = 0.1): the drift of each
// electron with the adrift of its nearest nucleus.
double fratio_of(const Walker &w, double tau, double tratio) {
  const Sys *s = w.s;
  double vav2sum = 0, v2sum = 0;
  for (int i = 0; i < w.N; i++) {
    const double *v = &w.vold[3 * i];
    double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (s->nloc > 0) {
      const double adrift = 0.5;
      double vavvt = (std::sqrt(1.0 + 2.0 * adrift * v2 * tau * tratio) - 1.0) / (adrift * v2);
      double vavvn = vavvt / (tau * tratio);
      vav2sum += vavvn * vavvn * v2;
    } else {
      const double adrift = 0.1, half = 0.5, eps = 1.0e-10;
      const double *x = &w.xold[3 * i];
      const int ic = nearest_centre(s, x);
      double rmin = 0, vr = 0;
      for (int k = 0; k < 3; k++) {
        const double rv = x[k] - s->cent[3 * ic + k];
        rmin += rv * rv;
        vr += v[k] * rv;
      }
      rmin = std::sqrt(rmin);
      vr = vr / rmin;
      const double va = std::sqrt(v2);
      const double hafzr2 = (half * s->znuc[s->iwctype[ic]] * rmin) * (half * s->znuc[s->iwctype[ic]] * rmin);
      const double adriftn = (half * (1 + eps + vr / va)) + adrift * hafzr2 / (1 + hafzr2);
      const double vavvt = (std::sqrt(1.0 + 2.0 * adriftn * v2 * tau) - 1.0) / (adriftn * v2);
      const double vavvn = vavvt / (tau * tratio);
      vav2sum += vavvn * vavvn * v2;
    }
    v2sum += v2;
  }
  return std::sqrt(vav2sum / v2sum);
}

// The drifted point of dmc_ae's move for an electron at x with drift v
// (dmc/dmc_ae_mov1.f90:227-303 forward, :396-474 reverse): the local frame
// of the nearest nucleus (z along the electron, x along the angular part
// of the drift), the UNR93 drift with the nucleus-dependent adrift, and the
// probability qgaus of sampling the exponential around the nucleus instead
// of the Gaussian around the drifted point.
struct AeFrame {
  int ic;
  double zeta, qgaus, pgaus, xd[3];
};
AeFrame ae_frame(const Sys *s, const double *x, const double *v, double tau) {
  const double one = 1, two = 2, half = 0.5, eps = 1.0e-10, adrift0 = 0.1;
  AeFrame f;
  f.ic = nearest_centre(s, x);
  const double *c = &s->cent[3 * f.ic];
  const double z = s->znuc[s->iwctype[f.ic]];
  double rv[3], rmin = 0, vr = 0, v2 = 0;
  for (int k = 0; k < 3; k++) {
    rv[k] = x[k] - c[k];
    rmin += rv[k] * rv[k];
    vr += v[k] * rv[k];
    v2 += v[k] * v[k];
  }
  rmin = std::sqrt(rmin);
  vr = vr / rmin;
  const double va = std::sqrt(v2);
  f.zeta = std::sqrt(one / tau + z * z);
  double zaxis[3], xaxis[3], vp = 0;
  for (int k = 0; k < 3; k++) {
    zaxis[k] = rv[k] / rmin;
    xaxis[k] = v[k] - vr * zaxis[k];
    vp += xaxis[k] * xaxis[k];
  }
  vp = std::sqrt(vp);
  if (vp < eps) {
    xaxis[0] = eps * (one - zaxis[0] * zaxis[0]);
    xaxis[1] = eps * (-zaxis[0] * zaxis[1]);
    xaxis[2] = eps * (-zaxis[0] * zaxis[2]);
    vp = eps * std::sqrt(one + eps - zaxis[0] * zaxis[0]);
  }
  for (int k = 0; k < 3; k++) xaxis[k] = xaxis[k] / vp;
  const double hafzr2 = (half * z * rmin) * (half * z * rmin);
  const double adrift = (half * (1 + eps + vr / va)) + adrift0 * hafzr2 / (1 + hafzr2);
  const double vavvt = (std::sqrt(one + two * adrift * v2 * tau) - one) / (adrift * v2);
  const double rtry = rmin + vavvt * vr;
  if (rtry > 0) {
    f.qgaus = half * std::erfc(rtry / std::sqrt(two * tau));
    const double xprime = vavvt * vp * rtry / (half * (rmin + rtry));
    for (int k = 0; k < 3; k++) f.xd[k] = c[k] + xaxis[k] * xprime + zaxis[k] * rtry;
  } else {
    f.qgaus = half * (one + std::erf(-rtry / std::sqrt(two * tau)));
    for (int k = 0; k < 3; k++) f.xd[k] = c[k];
  }
  f.pgaus = one - f.qgaus;
  return f;
}

// one walker of dmc_ps: electron moves, hpsi, weight; returns false if singular
bool dmc_walker(DmcPop &P, int iw, double ffi, double &wsum1, double &esum1, double &pesum, double &tpbsum,
                double &tausum, double &acc, double &trymove, long &nacc, long &nodecr) {
  Walker &w = P.w[iw];
  const Sys *s = P.s;
  const double tau = P.prm.tau, rttau = std::sqrt(tau), adrift = 0.5, one = 1, two = 2, zero = 0;
  double dfus2ac = 0, dfus2un = 0, drifdif = 0, pp = 1;
  int iaccept = 0;
  const bool ae = s->nloc == 0;
  const double term = std::pow(std::sqrt(two * PI * tau), 3) / PI;  // dmc_ae :148
  for (int i = 0; i < w.N; i++) {
    double *vo = &w.vold[3 * i];
    w.grad(i, 1, vo);
    double dfus2o = zero, xnew[3], fnormo = one;
    const double *xo = &w.xold[3 * i];
    if (ae) {
      // dmc_ae (dmc/dmc_ae_mov1.f90:227-356): drift in the nucleus frame,
      // then a Gaussian around the drifted point with probability pgaus or
      // an exponential around the nucleus
      const AeFrame f = ae_frame(s, xo, vo, tau);
      const double *c = &s->cent[3 * f.ic];
      for (int k = 0; k < 3; k++) xnew[k] = f.xd[k];
      double dfusb;
      if (w.rng.uniform() < f.pgaus) {
        double dfus2b = zero;
        for (int k = 0; k < 3; k++) {
          double dfus = gauss_draw(w.rng) * rttau;
          dfus2o += dfus * dfus;
          xnew[k] = xnew[k] + dfus;
          dfus2b += (xnew[k] - c[k]) * (xnew[k] - c[k]);
        }
        dfusb = std::sqrt(dfus2b);
      } else {
        const double u1 = w.rng.uniform(), u2 = w.rng.uniform(), u3 = w.rng.uniform();
        dfusb = (-0.5 / f.zeta) * std::log(u1 * u2 * u3);
        const double costht = two * (w.rng.uniform() - 0.5);
        const double sintht = std::sqrt(one - costht * costht);
        const double phi = two * PI * w.rng.uniform();
        for (int k = 0; k < 3; k++) {
          const double dfus = k == 0 ? dfusb * sintht * std::cos(phi) : k == 1 ? dfusb * sintht * std::sin(phi) : dfusb * costht;
          dfus2o += (c[k] + dfus - xnew[k]) * (c[k] + dfus - xnew[k]);
          xnew[k] = c[k] + dfus;
        }
      }
      fnormo = f.pgaus + f.qgaus * term * f.zeta * f.zeta * f.zeta * std::exp(-two * f.zeta * dfusb + 0.5 * dfus2o / tau);
    } else {
      double v2old = vo[0] * vo[0] + vo[1] * vo[1] + vo[2] * vo[2];
      double vavvt = (std::sqrt(one + two * adrift * v2old * tau) - one) / (adrift * v2old);
      for (int k = 0; k < 3; k++) {
        double drift = vavvt * vo[k];
        double dfus = gauss_draw(w.rng) * rttau;
        double dx = drift + dfus;
        dfus2o += dfus * dfus;
        xnew[k] = xo[k] + dx;
      }
    }
    for (int k = 0; k < 3; k++) w.xnew[k + 3 * i] = xnew[k];
    double psijn;
    double psidn = w.psie(i, w.xnew.data(), psijn, 0);
    double vn[3];
    if (w.detn != 0.0) w.grad(i, 0, vn);
    else vn[0] = vn[1] = vn[2] = 0;
    if (psidn * w.psido <= zero) nodecr++;  // icross=1: counted, not rejected
    double dfus2n = zero, fnormn = one;
    if (ae) {
      // the reverse move (dmc_ae :396-474): the drifted point of the new
      // position and the density of returning to the old one
      const AeFrame f = ae_frame(s, xnew, vn, tau);
      const double *c = &s->cent[3 * f.ic];
      double dfus2b = zero;
      for (int k = 0; k < 3; k++) {
        dfus2b += (c[k] - xo[k]) * (c[k] - xo[k]);
        dfus2n += (f.xd[k] - xo[k]) * (f.xd[k] - xo[k]);
      }
      const double dfusb = std::sqrt(dfus2b);
      fnormn = f.pgaus + f.qgaus * term * f.zeta * f.zeta * f.zeta * std::exp(-two * f.zeta * dfusb + 0.5 * dfus2n / tau);
    } else {
      double v2new = vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2];
      double vavvt = (std::sqrt(one + two * adrift * v2new * tau) - one) / (adrift * v2new);
      for (int k = 0; k < 3; k++) {
        double drift = vavvt * vn[k];
        double xbac = xnew[k] + drift;
        double dfus = xbac - xo[k];
        dfus2n += dfus * dfus;
      }
    }
    double p = (psidn / w.psido) * (psidn / w.psido) * std::exp(2 * (psijn - w.psijo)) *
               std::exp((dfus2o - dfus2n) / (two * tau)) * fnormn / fnormo;
    if (P.iage[iw] > 50) p = p * std::pow(1.1, P.iage[iw] - 50);
    pp = pp * p;
    p = std::min(one, p);
    acc += p;
    trymove += 1;
    dfus2ac += p * dfus2o;
    dfus2un += dfus2o;
    if (w.rng.uniform() < p) {
      iaccept = 1;
      nacc++;
      P.iage[iw] = 0;
      for (int k = 0; k < 3; k++) {
        drifdif += (w.xold[k + 3 * i] - xnew[k]) * (w.xold[k + 3 * i] - xnew[k]);
        w.xold[k + 3 * i] = xnew[k];
      }
      w.psido = psidn;
      w.psijo = psijn;
      w.jassav(i, 0);
      w.detsav(i);
    } else {
      for (int k = 0; k < 3; k++) w.xnew[k + 3 * i] = w.xold[k + 3 * i];
      w.distancese_restore(i);
    }
    w.update_ymat(i);
    if (w.singular) return false;
  }
  double tauprim = tau * dfus2ac / dfus2un;
  double psidn, psijn, ekino, enew;
  if (!w.hpsi(w.xold.data(), psidn, psijn, ekino, enew)) return false;
  w.psido = psidn;  // dmc_ps :516 drifts with the hpsi value of psid
  vold_all(w);
  if (P.prm.icasula == -1 && s->nloc > 0) w.md_tmove(psidn);  // dmc_ps :473
  double taunow = tauprim * 1.0;
  double fration = fratio_of(w, tau, one);
  // calculate_reweight (icut_e=0, icut_br=0)
  double deo = P.eest - w.eold, den = P.eest - enew;
  double ewto = P.eest - deo * P.fratio[iw];
  double ewtn = P.eest - den * fration;
  double expon = (P.prm.etrial - 0.5 * (ewto + ewtn)) * taunow;
  double dwt = std::exp(expon);
  dwt = dwt * ffi;
  P.wt[iw] = P.wt[iw] * dwt;
  double wtnow = P.wt[iw];
  double wtg = wtnow * P.fprod;
  tausum += wtg * taunow;
  w.eold = enew;
  w.ekino = ekino;
  w.psido = psidn;
  w.psijo = psijn;
  P.fratio[iw] = fration;
  if (iaccept == 0) P.iage[iw]++;
  wsum1 += wtnow;
  esum1 += wtnow * w.eold;
  pesum += wtg * (w.eold - ekino);
  tpbsum += wtg * ekino;
  (void)pp;
  (void)drifdif;
  if (P.prm.icasula == -1 && s->nloc > 0) return tmove_walker(P, iw);
  return true;
}

// T-move of one walker (icasula = -1): nonloc_grid (dmc/nonloc_grid.f90:3)
// over every electron with the matrix elements of the last hpsi, then the
// move of the chosen electron to its quadrature point, always accepted
// (dmc_ps :701-735).  Returns false if the new point is singular.
bool tmove_walker(DmcPop &P, int iw) {
  Walker &w = P.w[iw];
  const Sys *s = P.s;
  const int N = w.N, M = w.M, NQ = s->nquad;
  const double tauprim = P.prm.tau;
  double t_norm = 0.0;
  for (int i = 0; i < N; i++)
    for (int iq = 0; iq < NQ; iq++)
      for (int ic = 0; ic < M; ic++) {
        double &t = w.tvpsp[((size_t)i * NQ + iq) * M + ic];
        if (t > 0.0) t = 0.0;
        t_norm = t_norm - t;
      }
  t_norm = 1.0 + t_norm * tauprim;
  if (t_norm == 1.0) return true;
  const double t_normi = 1.0 / t_norm;
  double t_cum = 0.0;
  const double p = w.rng.uniform();
  int iel = -1, icg = -1, iqg = -1;
  for (int i = 0; i < N && iel < 0; i++)
    for (int iq = 0; iq < NQ && iel < 0; iq++)
      for (int ic = 0; ic < M; ic++) {
        t_cum = t_cum - tauprim * w.tvpsp[((size_t)i * NQ + iq) * M + ic] * t_normi;
        if (t_cum > p) {
          iel = i;
          icg = ic;
          iqg = iq;
          break;
        }
      }
  if (iel < 0) return true;
  // distances of the walker at its current configuration (r_en of electron iel)
  w.distances(iel, w.xold.data());
  const double r = w.r_en[iel + N * icg];
  double xn[3] = {r * w.xq[iqg] + s->cent[0 + 3 * icg], r * w.yq[iqg] + s->cent[1 + 3 * icg],
                  r * w.zq[iqg] + s->cent[2 + 3 * icg]};
  for (int k = 0; k < 3; k++) w.xnew[k + 3 * iel] = xn[k];
  double psijn;
  const double psidn = w.psie(iel, w.xnew.data(), psijn, 0);
  if (w.singular) return false;
  for (int k = 0; k < 3; k++) w.xold[k + 3 * iel] = xn[k];
  w.psido = psidn;
  w.psijo = psijn;
  w.jassav(iel, 0);
  w.detsav(iel);
  // dmc_ps :726-727: the moved spin's phase ends, the other spin's Y sees it
  w.update_ymat(iel < s->nup ? s->nup - 1 : N - 1);
  P.iage[iw] = 0;
  P.tmoved[iw] = 1;
  return true;
}

// copy walker iw into slot iw2 (splitjdet/splitjjas and the dmc arrays);
// the slot keeps its own random stream
void copy_walker(DmcPop &P, int iw, int iw2) {
  Rng keep = P.w[iw2].rng;
  P.w[iw2] = P.w[iw];
  P.w[iw2].rng = keep;
  P.fratio[iw2] = P.fratio[iw];
}

// splitj (dmc/splitj.f90:3)
void splitj(DmcPop &P) {
  const double zero = 0, two = 2, half = 0.5;
  vector<int> iwundr;
  int ipair = 0, iw2 = 0;
  for (int iw = 0; iw < P.nwalk; iw++) {
    if (P.wt[iw] < half) {
      if (P.wt[iw] == zero) {
        P.nbrnch++;
        iwundr.push_back(iw);
      } else if (ipair == 0) {
        ipair = 1;
        iw2 = iw;
      } else {
        P.nbrnch++;
        ipair = 0;
        double wttot = P.wt[iw] + P.wt[iw2];
        if (P.pop.uniform() > (P.wt[iw] / wttot)) {
          P.wt[iw2] = wttot;
          iwundr.push_back(iw);
        } else {
          P.wt[iw] = wttot;
          iwundr.push_back(iw2);
        }
      }
    }
  }
  int nwalk2 = P.nwalk;
  for (int iw = 0; iw < P.nwalk; iw++) {
    if (P.wt[iw] >= two) {
      P.nbrnch++;
      int dst;
      if (!iwundr.empty()) {
        dst = iwundr.back();
        iwundr.pop_back();
      } else {
        dst = nwalk2++;
        if (nwalk2 > P.prm.mwalk) { P.failed = true; return; }
      }
      P.wt[iw] = P.wt[iw] * half;
      P.wt[dst] = P.wt[iw];
      P.iage[dst] = P.iage[iw];
      copy_walker(P, iw, dst);
    }
  }
  for (int j = (int)iwundr.size() - 1; j >= 0; j--) {
    int dst = iwundr[j];
    int src = nwalk2 - 1;
    nwalk2--;
    P.wt[dst] = P.wt[src];
    P.iage[dst] = P.iage[src];
    copy_walker(P, src, dst);
  }
  P.nwalk = nwalk2;
}

bool dmc_step(DmcPop &P, int nthreads) {
  const Sys *s = P.s;
  P.ipass++;
  if (s->nloc > 0) {
    // rotqua with the population stream, shared by every walker
    Walker tmp(s);
    tmp.rng = P.pop;
    tmp.rotqua();
    P.pop = tmp.rng;
    for (int iw = 0; iw < P.nwalk; iw++) {
      P.w[iw].xq = tmp.xq;
      P.w[iw].yq = tmp.yq;
      P.w[iw].zq = tmp.zq;
    }
  }
  const int ipmod = (int)(P.ipass % P.prm.nfprod);
  const double ginv = std::min(1.0, P.prm.tau);
  const double ffn = P.eigv * std::pow(P.wdsumo / P.prm.nconf, ginv);
  const double ffi = 1.0 / ffn;
  P.fprod = P.fprod * ffn / P.ff[ipmod];
  P.ff[ipmod] = ffn;
  const int W = P.nwalk;
  std::fill(P.tmoved.begin(), P.tmoved.end(), 0);
  vector<double> a_w(W), a_e(W), a_pe(W), a_tpb(W), a_tau(W), a_acc(W), a_try(W);
  vector<long> a_nacc(W), a_nod(W);
  vector<int> bad(W, 0);
  auto work = [&](int t) {
    for (int iw = t; iw < W; iw += nthreads) {
      double ws = 0, es = 0, pes = 0, tps = 0, tas = 0, ac = 0, tr = 0;
      long na = 0, nd = 0;
      if (!dmc_walker(P, iw, ffi, ws, es, pes, tps, tas, ac, tr, na, nd)) bad[iw] = 1;
      a_w[iw] = ws; a_e[iw] = es; a_pe[iw] = pes; a_tpb[iw] = tps; a_tau[iw] = tas;
      a_acc[iw] = ac; a_try[iw] = tr; a_nacc[iw] = na; a_nod[iw] = nd;
    }
  };
  if (nthreads <= 1) work(0);
  else {
    vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) th.emplace_back(work, t);
    for (auto &t : th) t.join();
  }
  for (int iw = 0; iw < W; iw++) P.nmove_casula += P.tmoved[iw];
  for (int iw = 0; iw < W; iw++) {
    if (bad[iw]) return false;
    P.wsum1 += a_w[iw]; P.esum1 += a_e[iw]; P.pesum += a_pe[iw]; P.tpbsum += a_tpb[iw];
    P.tausum += a_tau[iw]; P.acc += a_acc[iw]; P.trymove += a_try[iw]; P.nacc += a_nacc[iw];
    P.nodecr += a_nod[iw];
  }
  const double wgsum1 = P.wsum1 * P.fprod, egsum1 = P.esum1 * P.fprod;
  splitj(P);
  if (P.failed) return false;
  // acues1 (idmc=2)
  P.wgsum += wgsum1;
  P.egsum += egsum1;
  P.eest = (P.egcum + P.egsum) / (P.wgcum + P.wgsum);
  P.eigv = std::exp((P.prm.etrial - P.eest) * (P.taucum + P.tausum) / (P.wgcum + P.wgsum));
  P.wdsumo = P.wsum1;
  P.wsum1 = 0;
  P.esum1 = 0;
  return true;
}

void dmc_end_block(DmcPop &P) {
  // acuest (dmc/acuest.f90:112-255): block sums into the cumulative ones
  const double egnow = P.egsum / P.wgsum;
  P.egcm2 += P.egsum * egnow;
  P.wgcm2 += P.wgsum * P.wgsum;
  P.egcum += P.egsum;
  P.wgcum += P.wgsum;
  P.taucum += P.tausum;
  P.pecum += P.pesum;
  P.tpbcum += P.tpbsum;
  P.egsum = P.wgsum = P.tausum = P.pesum = P.tpbsum = 0;
  P.iblk++;
}

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
extern "C" {

int or_nterms4(int nordc) { return nterms4(nordc); }

// raw Jastrow parameter derivatives of one configuration x[N][3]
int or_jas_nraw(void *sysp) {
  const Sys *s = (const Sys *)sysp;
  return s->nctype * (s->norda + 1) + s->nspin2b * (s->nordb + 1) + s->nctype * s->nterms;
}
void or_jas_raw(void *sys, const double *x, double *out) {
  Walker w((const Sys *)sys);
  w.distances(-1, x);
  w.jas_raw(out);
}

// Orbital-rotation derivatives of one configuration x[N][3] for a single
// determinant: optorb_deriv's orbprim (vmc/optorb.f90:5-95) with the
// multideterminant terms absent (ymat = zmat = 0 for one determinant), i.e.
// for the variation phi_io -> phi_io + a phi_jo, d ln psi / d a =
// sum over the spins whose reference determinant holds io of
// aa(irep, jo) = sum_i slmi(irep + (i-1) nel) orb(i, jo)
// (multideterminant_hpsi, vmc/multideterminant.f90:66-82), irep the slot of
// io.  ideriv [nterm][2] holds 1-based (io, jo).  Returns 1 when the
// Slater matrix is singular.
int or_orb_o(void *sysp, const double *x, int nterm, const int *ideriv, double *out) {
  const Sys *s = (const Sys *)sysp;
  Walker w(s);
  double psid, psij, ekin, e;
  if (!w.hpsi(x, psid, psij, ekin, e)) return 1;
  const int N = s->N;
  for (int t = 0; t < nterm; t++) {
    const int io = ideriv[2 * t] - 1, jo = ideriv[2 * t + 1] - 1;
    double o = 0;
    for (int iab = 0; iab < 2; iab++) {
      const int nel = iab == 0 ? s->nup : s->ndn, ish = iab == 0 ? 0 : s->nup;
      int irep = -1;
      for (int j = 0; j < nel; j++)
        if (s->iworbd[ish + j] - 1 == io) irep = j;
      if (irep < 0) continue;
      double a = 0;
      for (int i = 0; i < nel; i++) a += w.slmi[iab][irep + nel * i] * w.orb[(ish + i) + N * jo];
      o += a;
    }
    out[t] = o;
  }
  if (s->ndet == 1) return 0;
  // expansions: optorb_deriv's orbprim (vmc/optorb.f90:46-95) adds
  // detratio * dorb_psi, dorb_psi = sum over spins of sum_i zmat(io,i) orb(i,jo)
  // (io virtual) - sum_i aaz(irep,i) orb(i,jo) (io in the reference), with
  // compute_zmat's (vmc/multideterminant.f90:491-560)
  // zmat(jrep,irep) = sum_{krep >= iactv} ymat(jrep,krep) slmi(krep,irep) and
  // aaz(jrep,irep) = sum_{krep >= ivirt} aa(jrep,krep) zmat(krep,irep)
  const int O = s->O;
  const double detratio = w.detiab[0] * w.detiab[1] / psid;
  vector<double> zmat[2], aaz[2];
  for (int iab = 0; iab < 2; iab++) {
    const int nel = iab == 0 ? s->nup : s->ndn;
    const Sys::MdSpin &m = s->md[iab];
    zmat[iab].assign((size_t)O * std::max(nel, 1), 0.0);
    aaz[iab].assign((size_t)std::max(nel, 1) * std::max(nel, 1), 0.0);
    if (nel == 0) continue;
    for (int irep = 0; irep < nel; irep++)
      for (int jrep = m.ivirt; jrep < O; jrep++) {
        double z = 0;
        for (int krep = m.iactv; krep < nel; krep++)
          z = z + w.ymat[iab][jrep + (size_t)O * krep] * w.slmi[iab][krep + (size_t)nel * irep];
        zmat[iab][jrep + (size_t)O * irep] = z;
      }
    for (int irep = 0; irep < nel; irep++)
      for (int jrep = 0; jrep < nel; jrep++) {
        double z = 0;
        for (int krep = m.ivirt; krep < O; krep++)
          z = z + w.aa[iab][jrep + (size_t)nel * krep] * zmat[iab][krep + (size_t)O * irep];
        aaz[iab][jrep + (size_t)nel * irep] = z;
      }
  }
  for (int t = 0; t < nterm; t++) {
    const int io = ideriv[2 * t] - 1, jo = ideriv[2 * t + 1] - 1;
    double dpsi = 0;
    for (int iab = 0; iab < 2; iab++) {
      const int nel = iab == 0 ? s->nup : s->ndn, ish = iab == 0 ? 0 : s->nup;
      if (nel == 0) continue;
      if (io >= s->md[iab].ivirt)
        for (int i = 0; i < nel; i++) dpsi = dpsi + zmat[iab][io + (size_t)O * i] * w.orb[(ish + i) + N * jo];
      int irep = -1;
      for (int j = 0; j < nel; j++)
        if (s->iworbd[ish + j] - 1 == io) irep = j;
      if (irep >= 0)
        for (int i = 0; i < nel; i++) dpsi = dpsi - aaz[iab][irep + (size_t)nel * i] * w.orb[(ish + i) + N * jo];
    }
    out[t] = dpsi * detratio + out[t];
  }
  return 0;
}

void *or_sys_create(const cw_system_desc *d) {
  Sys *s = new Sys();
  s->N = d->nelec; s->nup = d->nup; s->ndn = d->nelec - d->nup;
  s->M = d->ncent; s->nctype = d->nctype;
  s->iwctype.assign(d->iwctype, d->iwctype + d->ncent);
  s->cent.assign(d->cent, d->cent + 3 * d->ncent);
  s->znuc.assign(d->znuc, d->znuc + d->nctype);
  s->pecent = d->pecent;
  s->mrwf = d->mrwf; s->mpts = d->mrwf_pts;
  s->nrbas.assign(d->nrbas, d->nrbas + d->nctype);
  s->igrid.assign(d->igrid, d->igrid + d->nctype);
  s->nr.assign(d->nr, d->nr + d->nctype);
  s->arg.assign(d->arg, d->arg + d->nctype);
  s->r0.assign(d->r0, d->r0 + d->nctype);
  size_t nt = (size_t)d->nctype * d->mrwf;
  s->rwf.assign(d->rwf, d->rwf + nt * d->mrwf_pts);
  s->d2rwf.assign(d->d2rwf, d->d2rwf + nt * d->mrwf_pts);
  s->ce.assign(d->ce, d->ce + nt * CW_NCOEF);
  s->ae.assign(d->ae, d->ae + nt * 2);
  s->rmaxwf.assign(d->rmaxwf, d->rmaxwf + nt);
  s->mbastyp = d->mbastyp;
  s->nbastyp.assign(d->nbastyp, d->nbastyp + d->nctype);
  s->iwlbas.assign(d->iwlbas, d->iwlbas + (size_t)d->nctype * d->mbastyp);
  s->iwrwf.assign(d->iwrwf, d->iwrwf + (size_t)d->nctype * d->mbastyp);
  s->K = d->nbasis; s->O = d->norb; s->ndet = d->ndet;
  s->coef.assign(d->coef, d->coef + (size_t)d->nbasis * d->norb);
  s->cdet.assign(d->cdet, d->cdet + d->ndet);
  s->detsign.assign(d->ndet, 1.0);
  s->nstates = d->nstates > 1 ? d->nstates : 1;
  s->cdet_st.assign(d->cdet, d->cdet + (size_t)s->nstates * d->ndet);
  if (s->nstates > 1 && d->ndet < 2) {
    delete s;
    return nullptr;
  }
  s->iguiding = s->nstates > 1 ? d->iguiding : 0;
  if (s->iguiding > 0) {
    if (!d->weights_g) {
      delete s;
      return nullptr;
    }
    s->weights_g.assign(d->weights_g, d->weights_g + s->nstates);
  }
  s->iworbd.assign(d->iworbd, d->iworbd + d->nelec);
  s->iworbd_all.assign(d->iworbd, d->iworbd + (size_t)d->ndet * d->nelec);
  if (d->ndet > 1 && !multideterminants_define(*s)) {
    delete s;
    return nullptr;
  }
  s->norda = d->norda; s->nordb = d->nordb; s->nordc = d->nordc;
  s->isc = d->isc; s->nspin2b = d->nspin2b; s->nocuspb = d->nocuspb;
  s->scalek = d->scalek;
  s->nterms = nterms4(d->nordc);
  s->a4.assign(d->a4, d->a4 + (size_t)(d->norda + 1) * d->nctype);
  s->b.assign(d->b, d->b + (size_t)(d->nordb + 1) * d->nspin2b);
  if (s->nterms > 0) s->c.assign(d->c, d->c + (size_t)s->nterms * d->nctype);
  s->nloc = d->nloc;
  if (d->nloc > 0) {
    s->lpot.assign(d->lpot, d->lpot + d->nctype);
    s->necp_term.assign(d->necp_term, d->necp_term + (size_t)d->nctype * CW_MPS_L);
    size_t ng = (size_t)d->nctype * CW_MPS_L * CW_MGAUSS;
    s->necp_power.assign(d->necp_power, d->necp_power + ng);
    s->ecp_exponent.assign(d->ecp_exponent, d->ecp_exponent + ng);
    s->ecp_coef.assign(d->ecp_coef, d->ecp_coef + ng);
    s->nquad = d->nquad;
    s->xq0.assign(d->xq0, d->xq0 + d->nquad);
    s->yq0.assign(d->yq0, d->yq0 + d->nquad);
    s->zq0.assign(d->zq0, d->zq0 + d->nquad);
    s->wq.assign(d->wq, d->wq + d->nquad);
  } else {
    s->nquad = 0;
  }
  s->deltar = d->deltar; s->deltat = d->deltat; s->fbias = d->fbias;
  set_scale_dist(*s);
  return s;
}

void or_sys_destroy(void *sys) { delete (Sys *)sys; }

double or_pot_nn(int ncent, const double *cent, const double *znuc, const int32_t *iwctype) {
  // pot_nn: sum_{i<j} Z_i Z_j / r_ij, i outer 2..ncent, j inner 1..i-1
  double pe = 0;
  for (int i = 1; i < ncent; i++)
    for (int j = 0; j < i; j++) {
      double r = 0;
      for (int k = 0; k < 3; k++) r += (cent[k + 3 * i] - cent[k + 3 * j]) * (cent[k + 3 * i] - cent[k + 3 * j]);
      r = std::sqrt(r);
      pe += znuc[iwctype[i]] * znuc[iwctype[j]] / r;
    }
  return pe;
}

int or_matinv(double *a, int n, double *determinant) {
  // matinv (vmc/matinv.f90:22). n<=2 closed forms; else partial-pivot LU
  // (pivot = first entry of maximal |a| in the column, as idamax) with the
  // base-10 scaled determinant product, then the inverse from the LU factors.
  if (n == 0) return 0;
  if (n == 1) {
    *determinant = a[0];
    a[0] = 1.0 / a[0];
    return 0;
  }
  if (n == 2) {
    *determinant = a[0] * a[3] - a[2] * a[1];
    double deti = 1.0 / *determinant;
    double aux = a[0];
    a[0] = a[3] * deti;
    a[3] = aux * deti;
    a[1] = -a[1] * deti;
    a[2] = -a[2] * deti;
    return 0;
  }
  auto A = [&](int i, int j) -> double & { return a[i + n * j]; };
  vector<int> ipvt(n);
  for (int k = 0; k < n; k++) {
    int p = k;
    double amax = std::fabs(A(k, k));
    for (int i = k + 1; i < n; i++)
      if (std::fabs(A(i, k)) > amax) {
        amax = std::fabs(A(i, k));
        p = i;
      }
    ipvt[k] = p;
    if (A(p, k) == 0.0) return 1;
    if (p != k)
      for (int j = 0; j < n; j++) std::swap(A(k, j), A(p, j));
    double piv = 1.0 / A(k, k);
    for (int i = k + 1; i < n; i++) A(i, k) *= piv;
    for (int j = k + 1; j < n; j++) {
      double akj = A(k, j);
      if (akj != 0.0)
        for (int i = k + 1; i < n; i++) A(i, j) -= A(i, k) * akj;
    }
  }
  double det1 = 1.0, det2 = 0.0;
  const double ten = 10.0;
  for (int i = 0; i < n; i++) {
    if (ipvt[i] != i) det1 = -det1;
    det1 = A(i, i) * det1;
    if (det1 == 0.0) break;
    while (std::fabs(det1) < 1.0) { det1 = ten * det1; det2 = det2 - 1.0; }
    while (std::fabs(det1) >= ten) { det1 = det1 / ten; det2 = det2 + 1.0; }
  }
  *determinant = det1 * std::pow(10.0, det2);
  // inverse: inv(U) in place, then solve inv(A)*L = inv(U), then column swaps
  vector<double> col(n);
  for (int j = 0; j < n; j++) {
    A(j, j) = 1.0 / A(j, j);
    double ajj = -A(j, j);
    // column j of inv(U): inv(U)(0:j-1,0:j-1) * U(0:j-1,j) * (-1/U(j,j))
    for (int i = 0; i < j; i++) {
      double sum = 0;
      for (int k = i; k < j; k++) sum += A(i, k) * A(k, j);
      col[i] = sum;
    }
    for (int i = 0; i < j; i++) A(i, j) = col[i] * ajj;
  }
  vector<double> work(n);
  for (int j = n - 2; j >= 0; j--) {
    for (int i = j + 1; i < n; i++) {
      work[i] = A(i, j);
      A(i, j) = 0.0;
    }
    for (int i = 0; i < n; i++) {
      double sum = 0;
      for (int k = j + 1; k < n; k++) sum += A(i, k) * work[k];
      A(i, j) -= sum;
    }
  }
  for (int j = n - 2; j >= 0; j--) {
    int jp = ipvt[j];
    if (jp != j)
      for (int i = 0; i < n; i++) std::swap(A(i, j), A(i, jp));
  }
  return 0;
}

void or_rng_states(const int32_t *irn8, int nwalk, uint64_t *out) {
  Rng r;
  std::memcpy(r.s, irn8, 32);
  for (int w = 0; w < nwalk; w++) {
    std::memcpy(out + 4 * w, r.s, 32);
    r.jump();
  }
}

void or_rng_uniform(uint64_t *state, int n, double *out) {
  Rng r;
  std::memcpy(r.s, state, 32);
  for (int i = 0; i < n; i++) out[i] = r.uniform();
  std::memcpy(state, r.s, 32);
}

void or_gesqua(int *nq, double *xq, double *yq, double *zq, double *wq) {
  // gesqua (vmc/rotqua.f90:3), cases needed here: 4 (tetrahedron), 6, 18, 26
  // (octahedron family); other orders fall back to the closest of these.
  static const int iqs[4] = {4, 6, 18, 26};
  int best = 0;
  for (int c = 1; c < 4; c++)
    if (std::abs(*nq - iqs[c]) < std::abs(*nq - iqs[best])) best = c;
  int n = iqs[best];
  *nq = n;
  for (int j = 0; j < n; j++) xq[j] = yq[j] = zq[j] = wq[j] = 0;
  double p = 1.0 / std::sqrt(2.0), q = 1.0 / std::sqrt(3.0);
  if (n == 4) {
    for (int j = 0; j < 4; j++) {
      wq[j] = 0.25;
      xq[j] = (j + 1 > 2) ? -q : q;
      yq[j] = (j + 1 == 2 || j + 1 == 4) ? -q : q;
      zq[j] = (j + 1 == 2 || j + 1 == 3) ? -q : q;
    }
    return;
  }
  // weights ww(icase,k) for icase 2 (6), 4 (18), 5 (26) and octa counts 6,12,8
  double w1, w2, w3;
  if (n == 6) { w1 = 1.0 / 6.0; w2 = 0; w3 = 0; }
  else if (n == 18) { w1 = 1.0 / 30.0; w2 = 1.0 / 15.0; w3 = 0; }
  else { w1 = 1.0 / 21.0; w2 = 4.0 / 105.0; w3 = 27.0 / 840.0; }
  for (int j = 0; j < n; j++) wq[j] = j < 6 ? w1 : (j < 18 ? w2 : w3);
  int ip = 0, lp = 0;
  double si = -1.0;
  for (int ii = 0; ii < 2; ii++) {
    si = -si;
    xq[ii] = si;
    yq[2 + ii] = si;
    zq[4 + ii] = si;
    if (n > 6) {
      double sj = -1.0;
      for (int jj = 0; jj < 2; jj++) {
        sj = -sj;
        ip++;
        xq[5 + ip] = si * p;
        yq[5 + ip] = sj * p;
        yq[9 + ip] = si * p;
        zq[9 + ip] = sj * p;
        zq[13 + ip] = si * p;
        xq[13 + ip] = sj * p;
        if (n > 18) {
          double sk = -1.0;
          for (int kk = 0; kk < 2; kk++) {
            sk = -sk;
            lp++;
            xq[17 + lp] = si * q;
            yq[17 + lp] = sj * q;
            zq[17 + lp] = sk * q;
          }
        }
      }
    }
  }
}

void or_sites(void *sysp, uint64_t *state, double *x) {
  const Sys &s = *(const Sys *)sysp;
  Rng r;
  std::memcpy(r.s, state, 32);
  // nsite rule of mc_configs_start (vmc/mc_configs.f90:75-94), no charged atom
  vector<int> nsite(s.M);
  int l = 0;
  for (int i = 0; i < s.M; i++) {
    nsite[i] = (int)(s.znuc[s.iwctype[i]] + 0.5);
    l += nsite[i];
    if (l > s.N) {
      nsite[i] -= (l - s.N);
      l = s.N;
    }
  }
  if (l < s.N) nsite[0] += (s.N - l);
  // sites (vmc/sites.f90:3)
  l = 0;
  for (int ispin = 1; ispin <= 2; ispin++)
    for (int i = 0; i < s.M && l < s.N; i++) {
      int ju = (nsite[i] + 2 - ispin) / 2;
      for (int j = 1; j <= ju; j++) {
        l++;
        if (l > s.N) break;
        double z = s.znuc[s.iwctype[i]], sitsca;
        if (j == 1) sitsca = 1 / z;
        else if (j <= 5) sitsca = 2 / (z - 2);
        else sitsca = 3 / (z - 10);
        for (int ic = 0; ic < 3; ic++) {
          double site = -std::log(r.uniform());
          double sg = r.uniform() - 0.5;
          site = sg >= 0 ? std::fabs(site) : -std::fabs(site);
          x[ic + 3 * (l - 1)] = sitsca * site + s.cent[ic + 3 * i];
        }
      }
    }
  std::memcpy(state, r.s, 32);
}

void or_orbitals(void *sys, const double *x, double *orb, double *dorb, double *ddorb) {
  Walker w((const Sys *)sys);
  w.distances(-1, x);
  w.orbitals_all();
  if (orb) std::memcpy(orb, w.orb.data(), sizeof(double) * w.orb.size());
  if (dorb) std::memcpy(dorb, w.dorb.data(), sizeof(double) * w.dorb.size());
  if (ddorb) std::memcpy(ddorb, w.ddorb.data(), sizeof(double) * w.ddorb.size());
}

void or_jastrow(void *sys, const double *x, double *psij, double *v, double *d2j) {
  Walker w((const Sys *)sys);
  w.distances(-1, x);
  w.jastrow_factor4();
  if (psij) *psij = w.fsumo;
  if (v) std::memcpy(v, w.fjo.data(), sizeof(double) * w.fjo.size());
  if (d2j) *d2j = w.d2o;
}

int or_slater(void *sys, const double *x, double *slmi, double *det) {
  const Sys *s = (const Sys *)sys;
  Walker w(s);
  w.distances(-1, x);
  if (!w.determinant()) return 1;
  int nmax = std::max(s->nup, s->ndn);
  for (int iab = 0; iab < 2; iab++) {
    int nel = iab == 0 ? s->nup : s->ndn;
    if (slmi)
      for (int j = 0; j < nel * nel; j++) slmi[iab * nmax * nmax + j] = w.slmi[iab][j];
    if (det) det[iab] = w.detiab[iab];
  }
  return 0;
}

int or_hpsi(void *sys, const double *x, const double *xq, const double *yq, const double *zq, double *out) {
  const Sys *s = (const Sys *)sys;
  Walker w(s);
  if (xq) {
    w.xq.assign(xq, xq + s->nquad);
    w.yq.assign(yq, yq + s->nquad);
    w.zq.assign(zq, zq + s->nquad);
  }
  double psid, psij, ekin, e, extra[2];
  if (!w.hpsi(x, psid, psij, ekin, e, extra)) return 1;
  out[0] = e; out[1] = psid; out[2] = psij; out[3] = ekin; out[4] = extra[0]; out[5] = extra[1];
  return 0;
}

// T-move elements of one configuration (nonloc + multideterminant_tmove):
// every quadrature point of the last nonloc (up to cap), out rows
// (iel, ic, iq, term_radial_jas, t_vpsp); returns the count (-1: singular)
int or_tmove_elements(void *sys, const double *x, const double *xq, const double *yq, const double *zq, int cap,
                      double *out, double *psid_out) {
  const Sys *s = (const Sys *)sys;
  Walker w(s);
  if (xq) {
    w.xq.assign(xq, xq + s->nquad);
    w.yq.assign(yq, yq + s->nquad);
    w.zq.assign(zq, zq + s->nquad);
  }
  double psid, psij, ekin, e, extra[2];
  if (!w.hpsi(x, psid, psij, ekin, e, extra)) return -1;
  w.md_tmove(psid);
  *psid_out = psid;
  const int n = (int)w.tq_iel.size();
  for (int q = 0; q < n && q < cap; q++) {
    const int iel = w.tq_iel[q], ic = w.tq_ic[q], iq = w.tq_iq[q];
    double *o = out + 5 * (size_t)q;
    o[0] = iel; o[1] = ic; o[2] = iq; o[3] = w.tq_trj[q];
    o[4] = w.tvpsp[((size_t)iel * s->nquad + iq) * s->M + ic];
  }
  return n;
}

void *or_walkers_create(void *sysp, int nwalk, const double *x, const uint64_t *rng) {
  const Sys *s = (const Sys *)sysp;
  Walkers *ws = new Walkers();
  ws->s = s;
  ws->w.reserve(nwalk);
  for (int k = 0; k < nwalk; k++) {
    ws->w.emplace_back(s);
    Walker &w = ws->w.back();
    std::memcpy(w.rng.s, rng + 4 * k, 32);
    std::memcpy(w.xold.data(), x + (size_t)3 * s->N * k, sizeof(double) * 3 * s->N);
    if (!w.zerest()) ws->failed = true;
  }
  return ws;
}

void or_walkers_destroy(void *ws) { delete (Walkers *)ws; }

int or_zerest(void *wsp) {
  // zerest (vmc/acuest.f90:179) on every walker + the rank-0 cumulative sums
  Walkers *ws = (Walkers *)wsp;
  int bad = 0;
  for (Walker &w : ws->w)
    if (!w.zerest()) bad = 1;
  ws->ecum = ws->ecm2 = ws->wcum = ws->pecum = ws->tpbcum = ws->pecm2 = ws->tpbcm2 = ws->acc = 0;
  ws->ecum1 = ws->ecm21 = ws->ecum1s = ws->ecm21s = 0;
  ws->iblk = 0;
  ws->passes = 0;
  return bad;
}

int or_vmc_steps(void *wsp, int nstep, int nthreads) {
  Walkers *ws = (Walkers *)wsp;
  int W = (int)ws->w.size();
  if (nthreads < 1) nthreads = 1;
  vector<int> bad(W, 0);
  auto work = [&](int t) {
    for (int k = t; k < W; k += nthreads) {
      Walker &w = ws->w[k];
      for (int st = 0; st < nstep; st++) {
        if (ws->s->nloc > 0) w.rotqua();
        if (!w.metrop6()) { bad[k] = 1; break; }
      }
    }
  };
  if (nthreads == 1) work(0);
  else {
    vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) th.emplace_back(work, t);
    for (auto &t : th) t.join();
  }
  ws->passes += nstep;
  ws->nstep_last = nstep;
  for (int k = 0; k < W; k++)
    if (bad[k]) return 1;
  return 0;
}

void or_end_block(void *wsp, double *block_energy) {
  // acuest (vmc/acuest.f90:61) per walker then acuest_reduce's sum over ranks
  Walkers *ws = (Walkers *)wsp;
  double es = 0, wsm = 0;
  for (Walker &w : ws->w) {
    double enow = w.esum / w.wsum;
    ws->wcum += w.wsum;
    ws->ecum += w.esum;
    ws->ecm2 += w.esum * enow;
    double penow = w.pesum / w.wsum, tpbnow = w.tpbsum / w.wsum;
    ws->pecm2 += w.pesum * penow;
    ws->tpbcm2 += w.tpbsum * tpbnow;
    ws->pecum += w.pesum;
    ws->tpbcum += w.tpbsum;
    ws->acc += w.acc;
    ws->ecum1 += w.ecum1; ws->ecm21 += w.ecm21; ws->ecum1s += w.ecum1s; ws->ecm21s += w.ecm21s;
    const int ns = ws->s->nstates;
    if (ns > 1) {
      for (auto *v : {&ws->wcum_st, &ws->ecum_st, &ws->ecm2_st, &ws->pecum_st, &ws->tpbcum_st}) v->resize(ns, 0.0);
      for (int st = 0; st < ns; st++) {
        const double en = w.esum_st[st] / w.wsum_st[st];
        ws->wcum_st[st] += w.wsum_st[st];
        ws->ecum_st[st] += w.esum_st[st];
        ws->ecm2_st[st] += w.esum_st[st] * en;
        ws->pecum_st[st] += w.pesum_st[st];
        ws->tpbcum_st[st] += w.tpbsum_st[st];
        w.wsum_st[st] = w.esum_st[st] = w.pesum_st[st] = w.tpbsum_st[st] = 0;
      }
    }
    es += w.esum;
    wsm += w.wsum;
    w.esum = w.wsum = w.pesum = w.tpbsum = 0;
    w.acc = 0;
    w.ecum1 = w.ecm21 = w.ecum1s = w.ecm21s = 0;
  }
  ws->iblk += (long)ws->w.size();
  if (block_energy) *block_energy = es / wsm;
}

void or_results(void *wsp, double *out) {
  // finwrt (vmc/finwrt.f90:75-187) with the reduced (all-rank) sums
  Walkers *ws = (Walkers *)wsp;
  int W = (int)ws->w.size();
  double passes = (double)ws->passes * W;  // passes summed over ranks (finwrt uses nproc*passes)
  double efin = ws->ecum / ws->wcum;
  auto err = [&](double x, double x2) {
    return std::sqrt(std::fabs(x2 / ws->wcum - (x / ws->wcum) * (x / ws->wcum)) / (double)ws->iblk);
  };
  auto err1 = [&](double x, double x2) {
    return std::sqrt(std::fabs(x2 / ws->wcum - (x / ws->wcum) * (x / ws->wcum)) / passes);
  };
  double eerr = err(ws->ecum, ws->ecm2);
  double eerr1s = err1(ws->ecum1s, ws->ecm21s);
  double rtpass = std::sqrt(passes);
  double tcsq = eerr1s == 0 ? 0 : eerr / eerr1s;
  out[0] = efin;
  out[1] = eerr;
  out[2] = eerr1s * rtpass;
  out[3] = tcsq * tcsq;
  out[4] = ws->acc / (passes * ws->s->N);
  out[5] = ws->pecum / ws->wcum;
  out[6] = ws->tpbcum / ws->wcum;
  out[7] = (double)ws->iblk;
}

int or_results_state(void *wsp, int istate, double *out) {
  // finwrt per state from the reweighted cumulative sums of that state
  Walkers *ws = (Walkers *)wsp;
  if (istate < 0 || istate >= ws->s->nstates) return 1;
  if (ws->s->nstates == 1) {
    or_results(wsp, out);
    return 0;
  }
  const double wc = ws->wcum_st[istate], ec = ws->ecum_st[istate], e2 = ws->ecm2_st[istate];
  const double nan = std::nan("");
  out[0] = ec / wc;
  out[1] = std::sqrt(std::fabs(e2 / wc - (ec / wc) * (ec / wc)) / (double)ws->iblk);
  out[2] = out[3] = out[4] = nan;
  out[5] = ws->pecum_st[istate] / wc;
  out[6] = ws->tpbcum_st[istate] / wc;
  out[7] = (double)ws->iblk;
  return 0;
}

void or_state_energies(void *wsp, double *e, double *psid) {
  Walkers *ws = (Walkers *)wsp;
  const int ns = ws->s->nstates;
  for (size_t k = 0; k < ws->w.size(); k++)
    for (int st = 0; st < ns; st++) {
      const Walker &w = ws->w[k];
      e[k * ns + st] = ns > 1 ? w.e_st[st] : w.eold;
      psid[k * ns + st] = ns > 1 ? w.psid_st[st] : w.psido;
    }
}

void or_opt_ci(void *wsp, int enable) {
  Walkers *ws = (Walkers *)wsp;
  for (Walker &w : ws->w) {
    w.opt_ci = enable != 0;
    w.sr_o.clear(); w.sr_eo.clear(); w.sr_oo.clear();
    w.sr_w = 0;
  }
}

void or_ci_o(void *wsp, double *out) {
  Walkers *ws = (Walkers *)wsp;
  const int nd = ws->s->ndet;
  for (size_t k = 0; k < ws->w.size(); k++)
    for (int j = 0; j < nd; j++) out[k * nd + j] = j < (int)ws->w[k].ci_o.size() ? ws->w[k].ci_o[j] : 0.0;
}

void or_opt_ci_sums(void *wsp, double *o, double *eo, double *oo, double *wsum) {
  // the SR sums of all walkers (ranks) since the last call, in walker order
  Walkers *ws = (Walkers *)wsp;
  const int nd = ws->s->ndet;
  std::fill(o, o + nd, 0.0);
  std::fill(eo, eo + nd, 0.0);
  if (oo) std::fill(oo, oo + (size_t)nd * nd, 0.0);
  *wsum = 0;
  for (Walker &w : ws->w) {
    if (w.sr_o.empty()) continue;
    for (int k = 0; k < nd; k++) {
      o[k] += w.sr_o[k];
      eo[k] += w.sr_eo[k];
    }
    if (oo)
      for (size_t t = 0; t < (size_t)nd * nd; t++) oo[t] += w.sr_oo[t];
    *wsum += w.sr_w;
    std::fill(w.sr_o.begin(), w.sr_o.end(), 0.0);
    std::fill(w.sr_eo.begin(), w.sr_eo.end(), 0.0);
    std::fill(w.sr_oo.begin(), w.sr_oo.end(), 0.0);
    w.sr_w = 0;
  }
}

void or_get_walkers(void *wsp, double *x, uint64_t *rng) {
  Walkers *ws = (Walkers *)wsp;
  int N = ws->s->N;
  for (size_t k = 0; k < ws->w.size(); k++) {
    if (x) std::memcpy(x + 3 * N * k, ws->w[k].xold.data(), sizeof(double) * 3 * N);
    if (rng) std::memcpy(rng + 4 * k, ws->w[k].rng.s, 32);
  }
}

void or_get_sums(void *wsp, double *out) {
  Walkers *ws = (Walkers *)wsp;
  for (size_t k = 0; k < ws->w.size(); k++) {
    const Walker &w = ws->w[k];
    out[5 * k + 0] = w.wsum;
    out[5 * k + 1] = w.esum;
    out[5 * k + 2] = w.pesum;
    out[5 * k + 3] = w.tpbsum;
    out[5 * k + 4] = w.acc;
  }
}

void or_get_state(void *wsp, double *eold, double *psido, double *psijo) {
  Walkers *ws = (Walkers *)wsp;
  for (size_t k = 0; k < ws->w.size(); k++) {
    if (eold) eold[k] = ws->w[k].eold;
    if (psido) psido[k] = ws->w[k].psido;
    if (psijo) psijo[k] = ws->w[k].psijo;
  }
}


// ----------------------------------------------------------------------------
// Per-electron routines of walker k, for a driver that keeps metrop6 on the
// host: psie (vmc/hpsie.f90:3) at a point, compute_determinante_grad
// (vmc/determinante.f90:69), the accept branch of metrop6
// (vmc/metrop_mov1_slat.f90:592-619: jassav, detsav) or distancese_restore
// (:621-626), update_ymat (vmc/multideterminant.f90:562).
// ----------------------------------------------------------------------------
int or_w1_psie(void *wsp, int k, int iel, const double *xnew3, double *out) {
  Walker &w = ((Walkers *)wsp)->w[k];
  w.xnew = w.xold;
  for (int c = 0; c < 3; c++) w.xnew[c + 3 * iel] = xnew3[c];
  double psij = 0;
  const double psid = w.psie(iel, w.xnew.data(), psij, 0);
  out[0] = psid;
  out[1] = psij;
  return w.singular ? 1 : 0;
}

void or_w1_grad(void *wsp, int k, int iel, int iflag_move, double *vd) {
  ((Walkers *)wsp)->w[k].grad(iel, iflag_move, vd);
}

void or_w1_commit(void *wsp, int k, int iel, int accept, double psidn, double psijn) {
  Walker &w = ((Walkers *)wsp)->w[k];
  if (accept) {
    for (int c = 0; c < 3; c++) w.xold[c + 3 * iel] = w.xnew[c + 3 * iel];
    w.psido = psidn;
    w.psijo = psijn;
    w.jassav(iel, 0);
    w.detsav(iel);
  } else {
    for (int c = 0; c < 3; c++) w.xnew[c + 3 * iel] = w.xold[c + 3 * iel];
    w.distancese_restore(iel);
  }
}

void or_w1_update_ymat(void *wsp, int k, int iel) { ((Walkers *)wsp)->w[k].update_ymat(iel); }

// ----------------------------------------------------------------------------
// DMC
// ----------------------------------------------------------------------------
void *or_dmc_create(void *sysp, int nwalk, const double *x, const uint64_t *rng, const uint64_t *pop_rng,
                    double tau, double etrial, int mwalk, int nfprod) {
  const Sys *s = (const Sys *)sysp;
  DmcPop *P = new DmcPop();
  P->s = s;
  P->prm = DmcParams{tau, etrial, nwalk, std::max(mwalk, nwalk), nfprod};
  P->nwalk = nwalk;
  std::memcpy(P->pop.s, pop_rng, 32);
  P->w.reserve(P->prm.mwalk);
  for (int k = 0; k < P->prm.mwalk; k++) {
    P->w.emplace_back(s);
    std::memcpy(P->w[k].rng.s, rng + 4 * k, 32);
  }
  P->wt.assign(P->prm.mwalk, 0.0);
  P->tmoved.assign(P->prm.mwalk, 0);
  P->fratio.assign(P->prm.mwalk, 0.0);
  P->iage.assign(P->prm.mwalk, 0);
  P->ff.assign(nfprod, 1.0);
  // init (dmc/init.f90:60-150)
  P->eigv = 1.0;
  P->eest = etrial;
  P->fprod = 1.0;
  P->wdsumo = nwalk;
  for (int iw = 0; iw < nwalk; iw++) {
    Walker &w = P->w[iw];
    std::memcpy(w.xold.data(), x + (size_t)3 * s->N * iw, sizeof(double) * 3 * s->N);
    w.xq = s->xq0; w.yq = s->yq0; w.zq = s->zq0;
    double psid, psij, ekin, e;
    if (!w.hpsi(w.xold.data(), psid, psij, ekin, e)) P->failed = true;
    w.psido = psid; w.psijo = psij; w.eold = e; w.ekino = ekin;
    vold_all(w);
    w.xnew = w.xold;
    P->wt[iw] = 1.0;
    // first call of dmc_ps: fratio with tratio=1
    P->fratio[iw] = fratio_of(w, tau, 1.0);
  }
  return P;
}
void or_dmc_destroy(void *p) { delete (DmcPop *)p; }
// T-moves (icasula, dmc_ps :701): 0 off, -1 one T-move per walker and step;
// returns 1 for an unsupported value or a multideterminant wave function
int or_dmc_set_tmoves(void *p, int icasula) {
  DmcPop *P = (DmcPop *)p;
  if (icasula != 0 && icasula != -1) return 1;
  if (icasula != 0 && (P->s->nloc == 0 || P->s->nstates > 1)) return 1;
  P->prm.icasula = icasula;
  return 0;
}
long or_dmc_tmoves(void *p) { return ((DmcPop *)p)->nmove_casula; }
int or_dmc_steps(void *p, int nstep, int nthreads) {
  DmcPop *P = (DmcPop *)p;
  if (P->failed) return 1;
  for (int k = 0; k < nstep; k++)
    if (!dmc_step(*P, nthreads)) return 1;
  return 0;
}
void or_dmc_end_block(void *p) { dmc_end_block(*(DmcPop *)p); }
// out: [0] egave, [1] err, [2] nwalk, [3] eest, [4] acceptance, [5] taueff,
//      [6] pe, [7] ke, [8] nblocks, [9] fprod, [10] eigv, [11] wdsumo
void or_dmc_results(void *p, double *out) {
  DmcPop *P = (DmcPop *)p;
  double egave = P->egcum / P->wgcum;
  double rn = P->wgcum * P->wgcum / P->wgcm2;
  double err = std::sqrt(std::max((P->egcm2 / P->wgcum - egave * egave) / (rn - 1), 0.0));
  out[0] = egave; out[1] = P->iblk > 1 ? err : 0.0; out[2] = P->nwalk; out[3] = P->eest;
  out[4] = P->acc / std::max(P->trymove, 1.0); out[5] = P->taucum / P->wgcum;
  out[6] = P->pecum / P->wgcum; out[7] = P->tpbcum / P->wgcum; out[8] = (double)P->iblk;
  out[9] = P->fprod; out[10] = P->eigv; out[11] = P->wdsumo;
}
// walkers: x [nwalk][N][3], wt [nwalk], eold [nwalk]; returns nwalk
int or_dmc_walkers(void *p, double *x, double *wt, double *eold, uint64_t *rng) {
  DmcPop *P = (DmcPop *)p;
  int N = P->s->N;
  for (int iw = 0; iw < P->nwalk; iw++) {
    if (x) std::memcpy(x + (size_t)3 * N * iw, P->w[iw].xold.data(), sizeof(double) * 3 * N);
    if (wt) wt[iw] = P->wt[iw];
    if (eold) eold[iw] = P->w[iw].eold;
    if (rng) std::memcpy(rng + 4 * iw, P->w[iw].rng.s, 32);
  }
  return P->nwalk;
}

}  // extern "C"
