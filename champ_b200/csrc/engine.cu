// engine.cu — the C ABI of include/champ_b200.h on top of the move and
// local-energy kernels.  One translation unit so the __constant__ system
// block is shared by every kernel without relocatable device code.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include <cudaTypedefs.h>

#include "../../include/champ_b200.h"
#include "common.cuh"
#include "gemm.cuh"
#include "hpsi.cuh"
#include "move.cuh"
#include "dmc.cuh"
#include "hooks.cuh"
#include "mdet.cuh"
#include "optjas.cuh"
#include "peak.cuh"
#include "umma.cuh"
#include "ragged.cuh"


using namespace cw;

// Host side of a DMC population (one CHAMP rank's dmc arrays and scalars).
struct DmcHost {
  bool on = false;
  int mwalk = 0, nconf = 0, nfprod = 100;
  double tau = 0, etrial = 0;
  DRng pop{};                       // rotqua + splitj stream
  double eest = 0, eigv = 1, wdsumo = 0, fprod = 1;
  std::vector<double> ff;           // ff(0:nfprod-1)
  long ipass = 0;
  double wsum1 = 0, esum1 = 0, pesum = 0, tpbsum = 0, tausum = 0;
  double wgsum = 0, egsum = 0, wgcum = 0, egcum = 0, wgcm2 = 0, egcm2 = 0, taucum = 0;
  double pecum = 0, tpbcum = 0, acc = 0, trymove = 0;
  long nacc = 0, nodecr = 0, nbrnch = 0, iblk = 0;
  int icasula = 0;                  // 0: no T-moves, -1: one per walker and step
  long nmove_casula = 0;
  DmcBuf db{};
  std::vector<void *> allocs;
  double *h_acc = nullptr, *h_wt = nullptr;   // pinned, [mwalk][DA_NA] and [mwalk]
  int *h_iage = nullptr, *h_copy = nullptr;   // pinned, [mwalk] and [2][mwalk]
  WalkerRec rec{};
};

struct cw_ctx {
  int device = 0, precision = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // second stream of a captured sweep: the moved electron's basis and LCAO
  // run beside its move Jastrow (both need only the proposal)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_jas = nullptr;  // hpsi: the full Jastrow done (the expansion's kinetic rows need its gradient)
  std::string err;
  CSys h;                 // host copy of the constant block
  GSys g{};               // device tables
  std::vector<void *> sys_allocs;
  // walkers
  int W = 0;
  WState st{};
  MoveBuf mb{};
  HBuf hb{};
  std::vector<void *> w_allocs;
  size_t smem_jmove = 0, smem_jmove_f32 = 0, smem_jfull = 0, smem_jfull_f32 = 0, smem_sinv = 0, smem_ctil = 0, smem_ecp = 0, smem_basis = 0;
  size_t smem_commit = 0;  // k_commit_tile's dynamic shared memory (0: the untiled k_commit)
  unsigned long long *d_stamps = nullptr;  // device-clock stamps (cw_stamp), kStampCap slots
  int nstamp = 0;
  int commit_grid = 1;     // k_commit_tile's grid: the blocks resident at once
  int gemm_bn_move = 64, gemm_bn_all = 64;  // N tiles of the FP64 LCAO GEMMs (cw_autotune)
  int big_spin = 0;        // Slater inverse and c~ on global memory (spins too large for shared memory)
  int ecp_rr_global = 0;   // k_ecp's e-n distances on global memory (hb.ecp_rr)
  int *acc_list = nullptr, *acc_count = nullptr;  // accepted walkers of a move (k_accept_list)
  double *xstage = nullptr;  // [W][N][3] positions in the caller's layout (cw_set_walkers / cw_get_walkers)
  int ecp_warps = 1, ecp_naov = 0, ecp_minb = 1;
  size_t dev_bytes = 0;  // bytes of this context's cudaMalloc allocations
  std::unordered_map<void *, size_t> alloc_bytes;
  double *bocc = nullptr;  // [nmax][K] coefficients of the occupied orbitals (c~ GEMM)
  // Parameter derivatives for optimisation (optjas gvalue, optci ci_o) and
  // the SR sums over the optimisation vector [njas Jastrow | ndet CI]
  double *md_sgn = nullptr;                       // [ndet] orbital-order signs
  bool opt_ci = false, opt_oo = false;
  int opt_w = 0, opt_njas = 0, opt_np = 0, jas_nraw = 0;
  double *opt_o = nullptr, *opt_ot = nullptr;     // [W][np], [np][W]
  double *jas_raw = nullptr, *jas_map = nullptr;  // [W][nraw], [nraw][njas]
  double *sr_o = nullptr, *sr_eo = nullptr, *sr_oo = nullptr, *oo_tmp = nullptr;
  double sr_w = 0;
  std::vector<void *> opt_allocs;
  // CUDA graph of one VMC sweep (captured on first use)
  cudaGraph_t sweep_graph = nullptr;
  cudaGraphExec_t sweep_exec = nullptr;
  long sweep_gen = 0;      // captures of the sweep so far (a batch rebuilds on change)
  long sweep_launches = 0;
  int sweep_w = 0;
  int basis_warps = 4;
  // rank-0 cumulative estimators (acuest_reduce)
  double ecum = 0, ecm2 = 0, wcum = 0, pecum = 0, tpbcum = 0, pecm2 = 0, tpbcm2 = 0, acc = 0;
  std::vector<double> st_cum;  // several states: [nstates][5] wcum, ecum, ecm2, pecum, tpbcum
  double ecum1s = 0, ecm21s = 0;
  long iblk = 0, passes = 0;
  double last_ms = 0;
  // launch accounting and optional per-stage event timing
  long launches = 0;
  bool prof = false;
  std::vector<cudaEvent_t> evpool;
  std::vector<int> evstage;      // stage of event pair k
  size_t evused = 0;
  double stage_ms[CW_NSTAGE] = {0};
  long stage_n[CW_NSTAGE] = {0};
  DmcHost dmc;
  // multideterminant expansion
  bool md_on = false;
  MdTab mdt{};
  MdBuf md{};
  double *md_vall = nullptr;     // [W][N][3] drift corrections of every electron (DMC)
  size_t smem_md_hpsi = 0, smem_md_phase = 0, smem_md_move = 0, smem_md_drift = 0, smem_md_tmove = 0;
  // mixed precision: tensor-core LCAO (TF32 x3) operands and tensor maps
  bool mixed = false;
  int kp = 0, np = 0, umma_st = 0;
  size_t smem_umma = 0;
  float *coef_hi = nullptr, *coef_lo = nullptr;   // [Oa][kp]
  int *d_err = nullptr;                            // tensor-core stage error flags
  CUtensorMap tm_b_hi{}, tm_b_lo{}, tm_mv_hi{}, tm_mv_lo{}, tm_all_hi{}, tm_all_lo{};
  // per-electron routines (cw_psie, cw_grad, cw_commit, cw_update_ymat)
  double *hook_buf = nullptr;    // [W][3] points in, [W][3] values out (device)
  int *hook_acc = nullptr;       // [W] accept flags (device)
  int hook_psie_iel = -1;        // electron of the last cw_psie (-1: none since the last commit)
  int hook_md_iel = -1;          // electron whose multideterminant move tables are prepared
  // orbital-rotation derivatives (cw_opt_orb): host term list, the slot of
  // each electron's orbital in determinant 1, and the device tables of the
  // current optimisation set-up
  std::vector<int> orb_ideriv;   // [n][2] 1-based (io, jo)
  std::vector<int> ref_orb;      // [nelec] 0-based orbital of each slot of determinant 1
  bool orb_on = false;
  int orb_nv = 0;
  OrbTerm *orb_terms = nullptr;
  int *orb_vorb = nullptr;
  double *orb_vals = nullptr;    // [W][N][nv]
};

namespace {

int fail(cw_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(c, e_ == cudaErrorMemoryAllocation ? CW_ERR_OOM : CW_ERR_CUDA,        \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

int nterms4(int nord) {
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

template <typename T>
int dalloc(cw_ctx *c, std::vector<void *> &list, T **p, size_t n) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess)
    return fail(c, CW_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
  list.push_back(q);
  c->dev_bytes += std::max<size_t>(n, 1) * sizeof(T);
  c->alloc_bytes[q] = std::max<size_t>(n, 1) * sizeof(T);
  *p = (T *)q;
  return CW_OK;
}

#define DALLOC(list, p, n)                         \
  do {                                             \
    int rc_ = dalloc(c, list, &(p), (size_t)(n));  \
    if (rc_) return rc_;                           \
  } while (0)

void free_list(cw_ctx *c, std::vector<void *> &l) {
  for (void *p : l) {
    cudaFree(p);
    auto it = c->alloc_bytes.find(p);
    if (it != c->alloc_bytes.end()) {
      c->dev_bytes -= it->second;
      c->alloc_bytes.erase(it);
    }
  }
  l.clear();
}

// The dynamic shared-memory limit of a kernel is a property of the function
// on the device, shared by every context of the process; contexts of
// different systems need different sizes, so the limit only ever grows.
std::mutex g_smem_mu;
std::map<std::pair<int, const void *>, size_t> g_smem_max;
template <typename F>
cudaError_t raise_smem(const cw_ctx *c, F *func, size_t bytes) {
  std::lock_guard<std::mutex> lk(g_smem_mu);
  size_t &cur = g_smem_max[{c->device, (const void *)func}];
  if (bytes <= cur) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

// Bracket a launch with CUDA events when profiling; count it either way.
void stage_begin(cw_ctx *c, int stage) {
  c->launches++;
  if (!c->prof) return;
  const size_t k = c->evused;
  if (2 * k + 2 > c->evpool.size()) {
    for (int i = 0; i < 256; i++) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      c->evpool.push_back(e);
    }
    c->evstage.resize(c->evpool.size() / 2);
  }
  c->evstage[k] = stage;
  cudaEventRecord(c->evpool[2 * k], c->stream);
}
void stage_end(cw_ctx *c) {
  if (!c->prof) return;
  cudaEventRecord(c->evpool[2 * c->evused + 1], c->stream);
  c->evused++;
}
void stage_collect(cw_ctx *c) {
  if (!c->prof) return;
  cudaStreamSynchronize(c->stream);
  for (size_t k = 0; k < c->evused; k++) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->evpool[2 * k], c->evpool[2 * k + 1]);
    c->stage_ms[c->evstage[k]] += ms;
    c->stage_n[c->evstage[k]]++;
  }
  c->evused = 0;
}

// Every kernel receives its context's system block by value, so entry points
// only select the context's device; contexts of different systems on one
// device run their work side by side, each on its own stream.
int bind(cw_ctx *c) {
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fail(c, CW_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return CW_OK;
}

#define BIND(c)                 \
  do {                          \
    int rc_b = bind(c);         \
    if (rc_b) return rc_b;      \
  } while (0)

int launch_check(cw_ctx *c, const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, CW_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
  return CW_OK;
}

#define LCHK(name)                        \
  do {                                    \
    int rc_ = launch_check(c, name);      \
    if (rc_) return rc_;                  \
  } while (0)

template <int NORD>
void launch_jmove(cw_ctx *c, int iel) {
  const int warps = 4;
  dim3 grid((c->W + warps - 1) / warps);
  if (c->mixed)
    k_jastrow_move_f32<NORD, kJmF32Partners><<<grid, 32 * warps, c->smem_jmove_f32, c->stream>>>(c->h, c->st, c->mb, iel);
  else
    k_jastrow_move<NORD><<<grid, 32 * warps, c->smem_jmove, c->stream>>>(c->h, c->st, c->mb, iel);
}
template <int NORD>
void launch_jfull(cw_ctx *c) {
  if (c->mixed)
    k_jastrow_full<NORD, float><<<c->W, 128, c->smem_jfull_f32, c->stream>>>(c->h, c->st, c->hb);
  else
    k_jastrow_full<NORD, double><<<c->W, 128, c->smem_jfull, c->stream>>>(c->h, c->st, c->hb);
}
template <int NORD>
void launch_ecp(cw_ctx *c) {
  const dim3 grid(c->W), block(32 * c->ecp_warps);
  if (c->mixed) {
    if (c->ecp_minb == 2) k_ecp<NORD, float, 2><<<grid, block, c->smem_ecp, c->stream>>>(c->h, c->st, c->hb, c->g);
    else k_ecp<NORD, float, 1><<<grid, block, c->smem_ecp, c->stream>>>(c->h, c->st, c->hb, c->g);
  } else {
    if (c->ecp_minb == 2) k_ecp<NORD, double, 2><<<grid, block, c->smem_ecp, c->stream>>>(c->h, c->st, c->hb, c->g);
    else k_ecp<NORD, double, 1><<<grid, block, c->smem_ecp, c->stream>>>(c->h, c->st, c->hb, c->g);
  }
}
template <int NORD>
int set_attrs(cw_ctx *c) {
  {
    // tiled commit: the spin's inverse (row stride nmax+1) and three vectors
    // in shared memory, for inverses up to 128 x 128 (140 KB)
    const int n = c->h.nmax;
    c->smem_commit = n <= 128 ? sizeof(double) * ((size_t)n * (n + 1) + 3 * n) : 0;
    if (c->smem_commit) {
      CK(raise_smem(c, k_commit_tile, c->smem_commit));
      // one wave of resident blocks loops over the accepted walkers
      int nsm = 0, per = 0;
      CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_commit_tile, 128, c->smem_commit));
      c->commit_grid = std::max(1, nsm * std::max(1, per));
    }
  }
  CK(raise_smem(c, k_jastrow_move<NORD>, (size_t)(c->smem_jmove)));
  CK(raise_smem(c, k_jastrow_move_f32<NORD, kJmF32Partners>, (size_t)(c->smem_jmove_f32)));
  CK(raise_smem(c, k_jastrow_full<NORD, double>, c->smem_jfull));
  CK(raise_smem(c, k_jastrow_full<NORD, float>, c->smem_jfull_f32));
  if (c->h.nloc > 0) {
    // warps per ECP block and register budget (two builds: one block per SM,
    // or two with at most 64 registers): the most resident warps per SM under
    // the shared memory (228 KB), register (64 K) and warp (64) limits; ties go
    // to the larger register budget, then to the larger block (fewer passes)
    const int tbytes = c->mixed ? 4 : 8, nb = 2 * ((een_nb(NORD) + 1) / 2);
    const int naov = c->ecp_naov;
    int best = 0;
    // the walker's scaled e-n distances go to global memory only when no
    // block shape fits them in shared memory
    for (int rrg = 0; rrg <= 1 && best == 0; rrg++)
    for (int minb = 1; minb <= 2; minb++) {
      cudaFuncAttributes fa;
      if (c->mixed)
        CK(minb == 2 ? cudaFuncGetAttributes(&fa, k_ecp<NORD, float, 2>) : cudaFuncGetAttributes(&fa, k_ecp<NORD, float, 1>));
      else
        CK(minb == 2 ? cudaFuncGetAttributes(&fa, k_ecp<NORD, double, 2>) : cudaFuncGetAttributes(&fa, k_ecp<NORD, double, 1>));
      const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
      for (int nw = 4; nw <= kEcpMaxWarps; nw++) {
        const size_t bytes = sizeof(double) * (ecp_base_doubles(c->h.N, c->h.M, 32 * nw, rrg) +
                                               (size_t)nw * ecp_warp_doubles(c->h.M, nb, tbytes, naov)) +
                             fa.sharedSizeBytes;
        if (bytes > 227 * 1024) continue;
        const int blocks = (int)std::min<size_t>({(size_t)(64 / nw), (228 * 1024) / (bytes + 1024),
                                                  (size_t)(65536 / (regs_warp * nw))});
        if (blocks > 0 && blocks * nw > best) {
          best = blocks * nw;
          c->ecp_warps = nw;
          c->ecp_minb = minb;
          c->smem_ecp = bytes - fa.sharedSizeBytes;
          c->ecp_rr_global = rrg;
        } else if (blocks > 0 && blocks * nw == best && minb == c->ecp_minb) {
          c->ecp_warps = nw;
          c->smem_ecp = bytes - fa.sharedSizeBytes;
        }
      }
    }
    if (best == 0) return fail(c, CW_ERR_UNSUPPORTED, "ECP stage shared memory too large");
    CK(raise_smem(c, k_ecp<NORD, double, 1>, c->smem_ecp));
    CK(raise_smem(c, k_ecp<NORD, float, 1>, c->smem_ecp));
    CK(raise_smem(c, k_ecp<NORD, double, 2>, c->smem_ecp));
    CK(raise_smem(c, k_ecp<NORD, float, 2>, c->smem_ecp));
  }
  return CW_OK;
}

// detsav + jassav of the accepted walkers (iel < 0: each walker's T-move electron);
// listed: k_decide has already listed them
void launch_commit(cw_ctx *c, int iel, bool listed = false) {
  if (c->smem_commit) {
    // the accepted walkers in order, then a fixed grid of blocks over them
    if (!listed) k_accept_list<<<1, 1024, 0, c->stream>>>(c->mb.ms, c->W, c->acc_list, c->acc_count);
    const int grid = std::max(1, std::min(c->W, c->commit_grid));
    k_commit_tile<<<grid, 128, c->smem_commit, c->stream>>>(c->h, c->st, c->mb, c->g, iel, c->acc_list, c->acc_count);
  } else {
    k_commit<<<c->W, 128, 0, c->stream>>>(c->h, c->st, c->mb, c->g, iel);
  }
}

#define NORD_DISPATCH(fn, ...)            \
  switch (c->h.nordc <= 1 ? 1 : c->h.nordc) { \
    case 1: fn<1>(__VA_ARGS__); break;    \
    case 2: fn<2>(__VA_ARGS__); break;    \
    case 3: fn<3>(__VA_ARGS__); break;    \
    case 4: fn<4>(__VA_ARGS__); break;    \
    case 5: fn<5>(__VA_ARGS__); break;    \
    case 6: fn<6>(__VA_ARGS__); break;    \
    default: fn<7>(__VA_ARGS__); break;   \
  }

int nord_attrs(cw_ctx *c) {
  switch (c->h.nordc <= 1 ? 1 : c->h.nordc) {
    case 1: return set_attrs<1>(c);
    case 2: return set_attrs<2>(c);
    case 3: return set_attrs<3>(c);
    case 4: return set_attrs<4>(c);
    case 5: return set_attrs<5>(c);
    case 6: return set_attrs<6>(c);
    default: return set_attrs<7>(c);
  }
}

// multideterminants_define (vmc/set_input_data.f90:46-414), kref = the
// first determinant: per spin the excitation (replaced reference slots in
// slot order, new orbitals in the determinant's order) of every
// determinant, the permutation sign folded into the coefficient, the unique
// spin-determinants ordered singles, doubles, rest (stable within each
// class), and for every determinant the unique index of each spin part
// (-1: the same as the reference).
int md_define(cw_ctx *c, const cw_system_desc *d, std::vector<int> &exc, std::vector<int> &kw,
              std::vector<double> &cdet, int nuniq[2], int ivirt[2], int iactv[2], int &numax,
              std::vector<double> &sgn) {
  const int N = d->nelec, nd = d->ndet, nup = d->nup, ndn = N - nup;
  auto IW = [&](int k, int i) { return d->iworbd[(size_t)k * N + i]; };
  for (size_t t = 0; t < (size_t)nd * N; t++)
    if (d->iworbd[t] < 1 || d->iworbd[t] > d->norb) return fail(c, CW_ERR_ARG, "iworbd entry out of range");
  std::vector<int> numrep((size_t)nd * 2, 0), irc((size_t)nd * 2 * N, 0), iro((size_t)nd * 2 * N, 0);
  const int ns = d->nstates > 1 ? d->nstates : 1;
  cdet.assign(d->cdet, d->cdet + (size_t)ns * nd);  // [nstates][ndet]
  sgn.assign(nd, 1.0);
  for (int k = 1; k < nd; k++) {
    int itot = 0;
    for (int iab = 0; iab < 2; iab++) {
      const int nel = iab == 0 ? nup : ndn, ish = iab == 0 ? 0 : nup;
      int nr = 0;
      for (int iref = 0; iref < nel; iref++) {
        bool in = false;
        for (int i = 0; i < nel; i++)
          if (IW(k, i + ish) == IW(0, iref + ish)) in = true;
        if (!in) irc[((size_t)k * 2 + iab) * N + nr++] = iref;
      }
      int isub = 0;
      for (int i = 0; i < nel; i++) {
        bool in = false;
        for (int iref = 0; iref < nel; iref++)
          if (IW(k, i + ish) == IW(0, iref + ish)) in = true;
        if (!in) iro[((size_t)k * 2 + iab) * N + isub++] = IW(k, i + ish) - 1;
      }
      if (isub != nr) return fail(c, CW_ERR_ARG, "determinant %d: inconsistent excitation", k + 1);
      numrep[k * 2 + iab] = nr;
      std::vector<int> sw(nel);
      for (int i = 0; i < nel; i++) sw[i] = IW(0, i + ish);
      for (int r = 0; r < nr; r++) sw[irc[((size_t)k * 2 + iab) * N + r]] = iro[((size_t)k * 2 + iab) * N + r] + 1;
      for (int i = 0; i < nel; i++)
        if (IW(k, i + ish) != sw[i])
          for (int l = i + 1; l < nel; l++)
            if (sw[l] == IW(k, i + ish)) {
              std::swap(sw[i], sw[l]);
              itot++;
            }
    }
    if (itot % 2) {
      sgn[k] = -1.0;
      for (int st = 0; st < ns; st++) cdet[(size_t)st * nd + k] = -cdet[(size_t)st * nd + k];
    }
  }
  kw.assign((size_t)nd * 2, -1);
  std::vector<std::vector<int>> order(2);
  for (int iab = 0; iab < 2; iab++) {
    const int nel = iab == 0 ? nup : ndn;
    iactv[iab] = nel;
    ivirt[iab] = iab == 0 ? nup : ndn;
    for (int k = 1; k < nd; k++)
      for (int r = 0; r < numrep[k * 2 + iab]; r++) {
        iactv[iab] = std::min(iactv[iab], irc[((size_t)k * 2 + iab) * N + r]);
        ivirt[iab] = std::min(ivirt[iab], iro[((size_t)k * 2 + iab) * N + r]);
      }
    auto same = [&](int a, int b) {
      if (numrep[a * 2 + iab] != numrep[b * 2 + iab]) return false;
      for (int r = 0; r < numrep[a * 2 + iab]; r++)
        if (irc[((size_t)a * 2 + iab) * N + r] != irc[((size_t)b * 2 + iab) * N + r] ||
            iro[((size_t)a * 2 + iab) * N + r] != iro[((size_t)b * 2 + iab) * N + r])
          return false;
      return true;
    };
    std::vector<int> iwun(nd, 0), uniq;
    for (int i = 1; i < nd; i++) {
      if (numrep[i * 2 + iab] == 0) continue;
      int j = 0;
      while (j != i && !same(j, i)) j++;
      iwun[i] = j;
      if (j == i) uniq.push_back(i);
    }
    // grouped by excitation order (1, 2, 3, then 4 and above), so that the
    // lanes of a warp, which take consecutive unique determinants, run the
    // same-size solve
    for (int pass = 0; pass < 4; pass++)
      for (int k : uniq) {
        const int nr = numrep[k * 2 + iab];
        if ((pass < 3 && nr == pass + 1) || (pass == 3 && nr > 3)) order[iab].push_back(k);
      }
    std::vector<int> kidx(nd, -1);
    for (size_t kk = 0; kk < order[iab].size(); kk++) kidx[order[iab][kk]] = (int)kk;
    for (int k = 1; k < nd; k++)
      if (numrep[k * 2 + iab] > 0) kw[(size_t)k * 2 + iab] = kidx[iwun[k]];
    nuniq[iab] = (int)order[iab].size();
  }
  numax = std::max(1, std::max(nuniq[0], nuniq[1]));
  const int stride = 1 + 2 * CW_MD_MEX;
  exc.assign((size_t)2 * numax * stride, 0);
  for (int iab = 0; iab < 2; iab++)
    for (int kk = 0; kk < nuniq[iab]; kk++) {
      const int k = order[iab][kk], nr = numrep[k * 2 + iab];
      if (nr > CW_MD_MEX)
        return fail(c, CW_ERR_UNSUPPORTED, "determinant %d: %d-fold excitation (at most %d supported)", k + 1, nr,
                    CW_MD_MEX);
      int *e = &exc[((size_t)iab * numax + kk) * stride];
      e[0] = nr;
      for (int r = 0; r < nr; r++) {
        e[1 + r] = irc[((size_t)k * 2 + iab) * N + r];
        e[1 + CW_MD_MEX + r] = iro[((size_t)k * 2 + iab) * N + r];
      }
    }
  return CW_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// 2-D FP32 tensor map over rows x K (row pitch kp floats), box 32 x box_rows,
// 128-byte swizzle; elements past K or past the last row read as zero.
int make_map(cw_ctx *c, CUtensorMap *map, const float *base, int K, long rows, int kp, int box_rows) {
  auto enc = tensor_map_encoder();
  if (!enc) return fail(c, CW_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t gdim[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t gstr[1] = {(cuuint64_t)kp * sizeof(float)};
  cuuint32_t box[2] = {32u, (cuuint32_t)box_rows};
  cuuint32_t est[2] = {1u, 1u};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)base, gdim, gstr, box, est,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(c, CW_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return CW_OK;
}

__global__ void k_split_rows(const double *src, int rows, int K, float *hi, float *lo, int kp) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)rows * kp) return;
  const int r = (int)(t / kp), k = (int)(t % kp);
  float h = 0.0f, l = 0.0f;
  if (k < K) split_tf32(src[(size_t)r * K + k], h, l);
  hi[t] = h;
  lo[t] = l;
}

// LCAO contraction of M basis rows: tensor cores (TF32 x3) in the mixed
// path, FP64 CUDA-core GEMM otherwise.
int lcao(cw_ctx *c, bool move, int M, const double *phi64, double *out, cudaStream_t strm = nullptr) {
  const CSys &h = c->h;
  cudaStream_t s = strm ? strm : c->stream;
  if (!c->mixed) {
    dgemm(s, M, h.Oa, h.K, phi64, c->g.coefT, out, move ? c->gemm_bn_move : c->gemm_bn_all);
    return launch_check(c, "dgemm");
  }
  const CUtensorMap &ahi = move ? c->tm_mv_hi : c->tm_all_hi;
  const CUtensorMap &alo = move ? c->tm_mv_lo : c->tm_all_lo;
  k_lcao_tf32x3<<<(M + 127) / 128, 128, c->smem_umma, s>>>(ahi, alo, c->tm_b_hi, c->tm_b_lo, M, h.K, c->np,
                                                           h.Oa, c->umma_st, out, h.Oa, c->d_err);
  return launch_check(c, "k_lcao_tf32x3");
}

// Multideterminant steps of a single-electron move (no-ops for one
// determinant): before the proposal (spin-phase G and Y, drift at the old
// position), after the LCAO (tables at the proposed position), after the
// commit (tables of an accepted move).
int md_before_propose(cw_ctx *c, int iel) {
  if (!c->md_on) return CW_OK;
  const CSys &h = c->h;
  const int W = c->W;
  if (iel == 0 || (iel == h.nup && h.ndn > 0)) {
    stage_begin(c, CW_ST_MDET);
    k_md_phase<<<W, 128, c->smem_md_phase, c->stream>>>(c->h, c->st, c->md, c->mdt, iel == 0 ? 0 : 1, nullptr);
    stage_end(c);
    LCHK("k_md_phase");
  }
  stage_begin(c, CW_ST_MDET);
  k_md_drift_old<<<W, 128, c->smem_md_drift, c->stream>>>(c->h, c->st, c->md, c->mdt, c->g, iel);
  stage_end(c);
  LCHK("k_md_drift_old");
  return CW_OK;
}
int md_after_lcao(cw_ctx *c, int iel, cudaStream_t strm = nullptr) {
  if (!c->md_on) return CW_OK;
  stage_begin(c, CW_ST_MDET);
  k_md_move<<<c->W, 128, c->smem_md_move, strm ? strm : c->stream>>>(c->h, c->st, c->mb, c->md, c->mdt, c->g, iel);
  stage_end(c);
  LCHK("k_md_move");
  return CW_OK;
}
int md_after_commit(cw_ctx *c, int iel) {
  if (!c->md_on) return CW_OK;
  stage_begin(c, CW_ST_MDET);
  k_md_commit<<<c->W, 128, 0, c->stream>>>(c->h, c->st, c->mb, c->md, c->mdt, iel);
  stage_end(c);
  LCHK("k_md_commit");
  return CW_OK;
}

// Full local energy of every walker (hpsi).  mode 1 also adds metrop6's sums.
template <int NORD>
void launch_jas_raw(cw_ctx *c) {
  k_jas_raw<NORD><<<c->W, kJasThreads, 0, c->stream>>>(c->h, c->st, c->jas_raw, c->jas_nraw);
}

// Parameter derivatives of every walker at the current configurations (the
// last hpsi): Jastrow part, then CI part of the optimisation vector
int opt_derivs(cw_ctx *c) {
  const int W = c->W;
  if (c->opt_njas > 0) {
    NORD_DISPATCH(launch_jas_raw, c);
    LCHK("k_jas_raw");
    const long n = (long)W * c->opt_njas;
    k_jas_o<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(W, c->jas_raw, c->jas_nraw, c->jas_map, c->opt_njas,
                                                                c->opt_np, c->opt_o, c->opt_ot);
    LCHK("k_jas_o");
  }
  if (c->opt_ci) {
    k_md_ci_o<<<W, 128, 0, c->stream>>>(c->h, c->st, c->md, c->mdt, c->md_sgn, c->opt_o, c->opt_ot, c->opt_np,
                                        c->opt_njas);
    LCHK("k_md_ci_o");
  }
  if (c->orb_on) {
    const int nt = (int)c->orb_ideriv.size() / 2;
    const long n = (long)W * nt;
    k_orb_o<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(c->h, c->st, nt, c->orb_terms, c->orb_nv, c->orb_vals,
                                                                c->opt_o, c->opt_ot, c->opt_np, c->opt_np - nt);
    LCHK("k_orb_o");
    if (c->md_on) {
      const size_t smem = sizeof(double) * ((size_t)c->h.Oa * c->h.nmax + (size_t)c->h.nmax * c->h.nmax);
      k_md_orb_o<<<W, 128, smem, c->stream>>>(c->h, c->st, c->md, nt, c->orb_terms, c->orb_nv, c->orb_vals, c->opt_o,
                                               c->opt_ot, c->opt_np, c->opt_np - nt);
      LCHK("k_md_orb_o");
    }
  }
  return CW_OK;
}

// Derivatives of every walker after a sweep's hpsi and the SR sums
int opt_accum(cw_ctx *c) {
  const int W = c->W, nd = c->opt_np;
  if (int rc = opt_derivs(c)) return rc;
  k_sr_accum<<<(nd + 127) / 128, 128, 0, c->stream>>>(c->st, c->opt_o, nd, c->sr_o, c->sr_eo);
  LCHK("k_sr_accum");
  if (c->opt_oo) {
    // sum_w O O^T as one GEMM over the walkers: [np x W] x [W x np]
    dgemm(c->stream, nd, nd, W, c->opt_ot, c->opt_o, c->oo_tmp);
    const size_t n = (size_t)nd * nd;
    k_add_inplace<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->sr_oo, c->oo_tmp, n);
    LCHK("k_add_inplace");
  }
  return CW_OK;  // the sample count is kept by cw_vmc_steps (this part may be a graph replay)
}

int run_hpsi(cw_ctx *c, int mode, double *d_e = nullptr, double *d_ekin = nullptr) {
  const CSys &h = c->h;
  const int W = c->W, N = h.N, M = h.M;
  // The full Jastrow and the orbital chain (basis, LCAO, scatter, Slater
  // inverse, c~) share no buffer: outside profiling the chain runs on the
  // side stream beside the Jastrow, joined before the ECP stage.  An
  // expansion's kinetic rows (k_md_scatter) use the Jastrow gradient, so
  // there the chain waits for the Jastrow before its first scatter.
  const bool fork = !c->prof;
  cudaStream_t os = fork ? c->side : c->stream;
  if (fork) {
    CK(cudaEventRecord(c->ev_fork, c->stream));
    CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
  }
  stage_begin(c, CW_ST_JASTROW_FULL);
  NORD_DISPATCH(launch_jfull, c);
  stage_end(c);
  LCHK("k_jastrow_full");
  if (fork && c->md_on) CK(cudaEventRecord(c->ev_jas, c->stream));
  // orbitals in electron chunks
  const int ec = c->hb.chunk;
  for (int e0 = 0; e0 < N; e0 += ec) {
    const int ne = std::min(ec, N - e0);
    const long nwarps = (long)W * ne;
    const int bw = c->basis_warps;
    stage_begin(c, CW_ST_BASIS_ALL);
    k_basis_all<<<(unsigned)((nwarps + bw - 1) / bw), 32 * bw, c->smem_basis, os>>>(c->h, c->st, c->hb, c->g, e0, ne);
    stage_end(c);
    LCHK("k_basis_all");
    stage_begin(c, CW_ST_LCAO_ALL);
    {
      int rc = lcao(c, false, W * ne * 5, c->hb.phi, c->hb.orball, os);
      stage_end(c);
      if (rc) return rc;
    }
    if (c->md_on) {
      const long nt = (long)W * ne * h.Oa;
      if (fork && e0 == 0) CK(cudaStreamWaitEvent(os, c->ev_jas, 0));
      stage_begin(c, CW_ST_SCATTER);
      k_md_scatter<<<(unsigned)((nt + 127) / 128), 128, 0, os>>>(c->h, c->st, c->md, c->hb.orball, e0, ne);
      stage_end(c);
      LCHK("k_md_scatter");
    }
    if (c->orb_on) {
      const long nv = (long)W * ne * c->orb_nv;
      k_orb_vals<<<(unsigned)((nv + 127) / 128), 128, 0, os>>>(W, N, e0, ne, h.Oa, c->hb.orball, c->orb_nv,
                                                               c->orb_vorb, c->orb_vals);
      LCHK("k_orb_vals");
    }
    const long ns = (long)W * ne * h.nmax;
    stage_begin(c, CW_ST_SCATTER);
    k_scatter_orbs<<<(unsigned)((ns + 127) / 128), 128, 0, os>>>(c->h, c->st, c->hb, c->g, e0, ne);
    stage_end(c);
    LCHK("k_scatter_orbs");
  }
  stage_begin(c, CW_ST_SLATER_INV);
  k_slater_inv<<<2 * W, 128, c->smem_sinv, os>>>(c->h, c->st, c->hb, c->big_spin);
  stage_end(c);
  LCHK("k_slater_inv");
  if (h.nloc > 0 && c->md_on) {
    const size_t np = (size_t)W * N * h.K;
    k_md_zero<<<(unsigned)((np + 255) / 256), 256, 0, os>>>(c->md.P, np);
    LCHK("k_md_zero");
  }
  if (h.nloc > 0) {
    const int nchunk = (h.K + 63) / 64;
    stage_begin(c, CW_ST_CTILDE);
    if (c->bocc)  // rows (walker, spin, slot) of slmi times the occupied coefficient rows
      dgemm(os, W * N, h.K, h.nmax, c->st.slmi, c->bocc, c->hb.ctilde);
    else
      k_ctilde<<<2 * W * nchunk, 256, c->smem_ctil, os>>>(c->h, c->st, c->hb, c->g, c->big_spin);
    stage_end(c);
    LCHK("k_ctilde");
  }
  if (fork) {
    CK(cudaEventRecord(c->ev_join, c->side));
    CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
  }
  if (h.nloc > 0) {
    stage_begin(c, CW_ST_ECP);
    NORD_DISPATCH(launch_ecp, c);
    stage_end(c);
    LCHK("k_ecp");
    if (c->md_on) {
      // pseudopotential B matrix of every orbital: P x coef
      stage_begin(c, CW_ST_LCAO_ALL);
      dgemm(c->stream, W * N, h.Oa, h.K, c->md.P, c->g.coefT, c->md.bnl);
      stage_end(c);
      LCHK("dgemm(bnl)");
    }
  }
  if (c->md_on) {
    stage_begin(c, CW_ST_MDET);
    k_md_hpsi<<<W, 128, c->smem_md_hpsi, c->stream>>>(c->h, c->st, c->md, c->mdt, c->g);
    stage_end(c);
    LCHK("k_md_hpsi");
  }
  stage_begin(c, CW_ST_ENERGY);
  k_energy<<<(W + 3) / 4, 128, 0, c->stream>>>(c->h, c->st, c->hb, mode, d_e, d_ekin);
  stage_end(c);
  LCHK("k_energy");
  return CW_OK;
}

int check_status(cw_ctx *c) {
  if (c->mixed) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (e) return fail(c, CW_ERR_CUDA, "tensor-core LCAO stage: a pipeline wait timed out (flags %d)", e);
  }
  std::vector<int> s(c->W);
  CK(cudaMemcpyAsync(s.data(), c->st.status, sizeof(int) * c->W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int w = 0; w < c->W; w++)
    if (s[w] & 1) return fail(c, CW_ERR_SINGULAR, "walker %d: singular Slater matrix", w);
  for (int w = 0; w < c->W; w++)
    if (s[w]) return fail(c, CW_ERR_STATE, "walker %d: non-finite state (status %d)", w, s[w]);
  return CW_OK;
}

void free_dmc(cw_ctx *c) {
  DmcHost &d = c->dmc;
  free_list(c, d.allocs);
  c->hb.tvpsp = c->hb.tvtrj = nullptr;  // held in d.allocs
  for (void *p : {(void *)d.h_acc, (void *)d.h_wt, (void *)d.h_iage, (void *)d.h_copy})
    if (p) cudaFreeHost(p);
  d = DmcHost();
}

void drop_sweep_graph(cw_ctx *c) {
  if (c->sweep_exec) cudaGraphExecDestroy(c->sweep_exec);
  if (c->sweep_graph) cudaGraphDestroy(c->sweep_graph);
  c->sweep_exec = nullptr;
  c->sweep_graph = nullptr;
}

// drop the optimisation buffers (sized for one population)
void opt_reset(cw_ctx *c) {
  free_list(c, c->opt_allocs);
  c->opt_ci = c->opt_oo = false;
  c->opt_njas = c->opt_np = c->jas_nraw = 0;
  c->opt_o = c->opt_ot = c->jas_raw = c->jas_map = nullptr;
  c->sr_o = c->sr_eo = c->sr_oo = c->oo_tmp = nullptr;
  c->sr_w = 0;
  c->orb_on = false;
  c->orb_nv = 0;
  c->orb_terms = nullptr;
  c->orb_vorb = nullptr;
  c->orb_vals = nullptr;
}

int alloc_walkers(cw_ctx *c, int W) {
  drop_sweep_graph(c);  // the captured sweep holds this population's buffers
  free_dmc(c);
  opt_reset(c);  // derivative buffers are sized for the old population
  free_list(c, c->w_allocs);
  const CSys &h = c->h;
  const int N = h.N, M = h.M, K = h.K, Oa = h.Oa, nmax = h.nmax, NQ = std::max(h.nquad, 1);
  auto &L = c->w_allocs;
  WState &s = c->st;
  s.W = W;
  DALLOC(L, s.x, (size_t)W * 3 * N);
  DALLOC(L, c->xstage, (size_t)W * 3 * N);
  DALLOC(L, s.rng, (size_t)W * 4);
  DALLOC(L, s.xq, (size_t)W * 3 * NQ);
  DALLOC(L, s.rmino, (size_t)W * N);
  DALLOC(L, s.nearesto, (size_t)W * N);
  DALLOC(L, s.rvmino, (size_t)W * 3 * N);
  DALLOC(L, s.psido, W);
  DALLOC(L, s.psijo, W);
  DALLOC(L, s.psi2o, W);
  DALLOC(L, s.eold, W);
  DALLOC(L, s.ekino, W);
  DALLOC(L, s.slmi, (size_t)W * 2 * nmax * nmax);
  DALLOC(L, s.detiab, (size_t)W * 2);
  DALLOC(L, s.orbs, (size_t)W * N * nmax);
  DALLOC(L, s.dorbs, (size_t)W * 3 * N * nmax);
  DALLOC(L, s.fso, (size_t)W * N * N);
  DALLOC(L, s.fijo, (size_t)W * 3 * N * N);
  DALLOC(L, s.fjo, (size_t)W * 3 * N);
  DALLOC(L, s.fsumo, W);
  DALLOC(L, s.enm, (size_t)W * 2 * M * N);
  s.enmf = nullptr;
  if (c->mixed) DALLOC(L, s.enmf, (size_t)W * 2 * M * N);
  DALLOC(L, s.sums, (size_t)W * 8);
  DALLOC(L, s.status, W);
  MoveBuf &m = c->mb;
  DALLOC(L, m.ms, W);
  DALLOC(L, m.fsn, (size_t)W * N);
  DALLOC(L, m.fijn_i, (size_t)W * 3 * N);
  DALLOC(L, m.fijn_j, (size_t)W * 3 * N);
  DALLOC(L, m.fsumn, W);
  DALLOC(L, m.vjn, (size_t)W * 3);
  DALLOC(L, m.phi, (size_t)W * 4 * K);
  DALLOC(L, m.orbn, (size_t)W * 4 * Oa);
  DALLOC(L, m.enn, (size_t)W * 2 * M);
  HBuf &b = c->hb;
  DALLOC(L, b.d2o, W);
  DALLOC(L, b.pe_ee, W);
  DALLOC(L, b.pe_ecp, W);
  DALLOC(L, b.vpsp, (size_t)W * 2);
  DALLOC(L, b.ddx, (size_t)W * N * 4);
  DALLOC(L, b.ddorbs, (size_t)W * N * nmax);
  // electron chunk of the all-electron orbital stage, bounded by a byte budget
  size_t budget = (size_t)1 << 30;
  if (const char *e = getenv("CW_CHUNK_BYTES")) budget = (size_t)atoll(e);
  const size_t per_e = (size_t)W * 5 * (K + Oa) * sizeof(double);
  int chunk = (int)std::max<size_t>(1, budget / std::max<size_t>(per_e, 1));
  chunk = std::min(chunk, N);
  b.chunk = chunk;
  DALLOC(L, b.phi, (size_t)W * chunk * 5 * K);
  DALLOC(L, b.orball, (size_t)W * chunk * 5 * Oa);
  m.phi_hi = m.phi_lo = nullptr;
  b.phi_hi = b.phi_lo = nullptr;
  if (c->mixed) {
    const int kp = c->kp;
    m.kp = b.kp = kp;
    DALLOC(L, m.phi_hi, (size_t)W * 4 * kp);
    DALLOC(L, m.phi_lo, (size_t)W * 4 * kp);
    DALLOC(L, b.phi_hi, (size_t)W * chunk * 5 * kp);
    DALLOC(L, b.phi_lo, (size_t)W * chunk * 5 * kp);
    int rc = make_map(c, &c->tm_mv_hi, m.phi_hi, K, (long)W * 4, kp, 128);
    if (!rc) rc = make_map(c, &c->tm_mv_lo, m.phi_lo, K, (long)W * 4, kp, 128);
    if (!rc) rc = make_map(c, &c->tm_all_hi, b.phi_hi, K, (long)W * chunk * 5, kp, 128);
    if (!rc) rc = make_map(c, &c->tm_all_lo, b.phi_lo, K, (long)W * chunk * 5, kp, 128);
    if (rc) return rc;
  }
  if (h.nloc > 0) DALLOC(L, b.ctilde, (size_t)W * N * K);
  m.md_velo = m.md_veln = m.md_psidn = nullptr;
  b.tvpsp = nullptr;
  b.tvtrj = nullptr;
  b.ecp_rr = nullptr;
  if (h.nloc > 0 && c->ecp_rr_global) DALLOC(L, b.ecp_rr, (size_t)W * N * (M | 1));
  b.md_P = nullptr;
  b.md_den = b.md_S = nullptr;
  b.md_S_ms = b.md_den_ms = nullptr;
  b.e_ms = b.psid_ms = b.sums_ms = nullptr;
  c->md.S_ms = c->md.den_ms = c->md.Sn_ms = c->md.psi2gn = nullptr;
  m.md_psi2g = nullptr;
  c->md_vall = nullptr;
  if (c->md_on) {
    MdBuf &d = c->md;
    const int nu = c->mdt.numax;
    DALLOC(L, d.aa, (size_t)W * 2 * nmax * Oa);
    DALLOC(L, d.ymat, (size_t)W * 2 * nmax * Oa);
    DALLOC(L, d.dd, (size_t)W * 2 * nu);
    DALLOC(L, d.G, (size_t)W * (h.iguiding ? h.nstates : 1) * (nu + 1));
    DALLOC(L, d.S, W);
    DALLOC(L, d.orbA, (size_t)W * N * Oa);
    DALLOC(L, d.dorbA, (size_t)W * 3 * N * Oa);
    DALLOC(L, d.bkin, (size_t)W * N * Oa);
    DALLOC(L, d.bnl, (size_t)W * N * Oa);
    CK(cudaMemsetAsync(d.bnl, 0, sizeof(double) * (size_t)W * N * Oa, c->stream));
    if (h.nloc > 0) DALLOC(L, d.P, (size_t)W * N * K);
    DALLOC(L, d.den, (size_t)W * 2);
    DALLOC(L, d.cvec, (size_t)W * nmax);
    DALLOC(L, d.wvec, (size_t)W * Oa);
    DALLOC(L, d.ddn, (size_t)W * nu);
    DALLOC(L, d.Sn, W);
    DALLOC(L, d.psidn, W);
    DALLOC(L, d.veln, (size_t)W * 3);
    DALLOC(L, d.velo, (size_t)W * 3);
    DALLOC(L, c->md_vall, (size_t)W * N * 3);
    m.md_velo = d.velo;
    m.md_veln = d.veln;
    m.md_psidn = d.psidn;
    b.md_P = d.P;
    b.md_den = d.den;
    b.md_S = d.S;
    if (h.nstates > 1) {
      const int ns = h.nstates;
      DALLOC(L, d.S_ms, (size_t)W * ns);
      DALLOC(L, d.den_ms, (size_t)W * ns * 2);
      DALLOC(L, b.e_ms, (size_t)W * ns);
      DALLOC(L, b.psid_ms, (size_t)W * ns);
      DALLOC(L, b.sums_ms, (size_t)W * ns * 4);
      CK(cudaMemsetAsync(b.sums_ms, 0, sizeof(double) * W * ns * 4, c->stream));
      b.md_S_ms = d.S_ms;
      b.md_den_ms = d.den_ms;
      if (h.iguiding) {
        DALLOC(L, d.Sn_ms, (size_t)W * ns);
        DALLOC(L, d.psi2gn, W);
        m.md_psi2g = d.psi2gn;
      }
    }
  }
  DALLOC(L, b.entab, (size_t)W * M * N * kEnFields);
  b.entabf = nullptr;
  if (c->mixed) DALLOC(L, b.entabf, (size_t)W * M * N * kEnFields);
  DALLOC(L, c->acc_list, W);
  DALLOC(L, c->acc_count, 1);
  DALLOC(L, c->hook_buf, (size_t)W * 6);
  DALLOC(L, c->hook_acc, W);
  c->hook_psie_iel = c->hook_md_iel = -1;
  CK(cudaMemsetAsync(s.status, 0, sizeof(int) * W, c->stream));
  CK(cudaMemsetAsync(s.sums, 0, sizeof(double) * W * 8, c->stream));
  c->W = W;
  return CW_OK;
}

int zerest(cw_ctx *c) {
  const CSys &h = c->h;
  const int W = c->W, NQ = h.nquad;
  if (NQ > 0) {
    k_xq_unrotated<<<(W + 127) / 128, 128, 0, c->stream>>>(c->h, c->st);
    LCHK("k_xq_unrotated");
  }
  int rc = run_hpsi(c, 0);
  if (rc) return rc;
  const long nt = (long)W * h.N;
  k_nearest<<<(unsigned)((nt + 127) / 128), 128, 0, c->stream>>>(c->h, c->st);
  LCHK("k_nearest");
  CK(cudaMemsetAsync(c->st.sums, 0, sizeof(double) * W * 8, c->stream));
  c->ecum = c->ecm2 = c->wcum = c->pecum = c->tpbcum = c->pecm2 = c->tpbcm2 = c->acc = 0;
  c->ecum1s = c->ecm21s = 0;
  c->st_cum.assign(h.nstates > 1 ? (size_t)h.nstates * 5 : 0, 0.0);
  c->iblk = 0;
  c->passes = 0;
  return check_status(c);
}

// one thread writes the device's global nanosecond clock when the stream
// reaches it
constexpr int kStampCap = 1 << 14;
__global__ void k_stamp(unsigned long long *slot) {
  unsigned long long ns;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(ns));
  *slot = ns;
}

}  // namespace

// ===========================================================================
extern "C" {

int cw_create(cw_ctx **out, const cw_system_desc *d, int device, int precision) {
  cw_ctx *c = nullptr;
  if (!out || !d) return CW_ERR_ARG;
  *out = nullptr;
  c = new cw_ctx();
  c->device = device;
  c->precision = precision;
  auto bad = [&](const char *msg) {
    c->err = msg;
    *out = c;
    return CW_ERR_ARG;
  };
  if (d->ncent > CW_MAX_CENT) return bad("ncent exceeds CW_MAX_CENT");
  if (d->nctype > CW_MAX_TYPES) return bad("nctype exceeds CW_MAX_TYPES");
  if (d->mrwf > CW_MAX_RWF) return bad("mrwf exceeds CW_MAX_RWF");
  if (d->nordc > CW_MAX_NORD || d->norda > CW_MAX_NORD || d->nordb > CW_MAX_NORD) return bad("Jastrow order > 7");
  if (d->ndet < 1) return bad("ndet must be at least 1");
  if (d->nloc != 0 && d->nloc != 4) return bad("nloc must be 0 or 4");
  if (d->nquad > 32) return bad("nquad > 32 not supported");
  if (d->isc < 2 || d->isc > 5) return bad("isc must be 2..5");
  const int ndn = d->nelec - d->nup;
  const int nmax = std::max(d->nup, ndn);
  if (nmax > 256) return bad("more than 256 electrons of one spin");
  if (precision != CW_PREC_FP64 && precision != CW_PREC_MIXED) return bad("unknown precision");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    c->err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
    *out = c;
    return CW_ERR_CUDA;
  }
  *out = c;
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&c->ev0));
  CK(cudaEventCreate(&c->ev1));
  CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&c->ev_jas, cudaEventDisableTiming));
  CSys &h = c->h;
  std::memset(&h, 0, sizeof h);
  h.N = d->nelec; h.nup = d->nup; h.ndn = ndn; h.M = d->ncent; h.nctype = d->nctype;
  h.K = d->nbasis; h.Oa = d->norb; h.nmax = nmax;
  h.norda = d->norda; h.nordb = d->nordb; h.nordc = d->nordc; h.isc = d->isc;
  h.nspin2b = d->nspin2b; h.nocuspb = d->nocuspb; h.nterms = nterms4(d->nordc);
  if (h.nterms > CW_MAX_TERMS) return fail(c, CW_ERR_ARG, "too many e-e-n terms");
  h.nloc = d->nloc; h.nquad = d->nloc ? d->nquad : 0;
  h.scalek = d->scalek;
  h.deltar = d->deltar; h.deltat = d->deltat; h.fbias = d->fbias; h.pecent = d->pecent;
  h.cdet = d->cdet[0];
  h.nstates = d->nstates > 1 ? d->nstates : 1;
  if (h.nstates > 1) {
    if (d->ndet < 2) return fail(c, CW_ERR_UNSUPPORTED, "several states need a multideterminant expansion");
    if (h.nstates > CW_MAX_STATES) return fail(c, CW_ERR_ARG, "at most %d states", CW_MAX_STATES);
    h.iguiding = d->iguiding > 0 ? d->iguiding : 0;
    if (h.iguiding) {
      if (!d->weights_g) return fail(c, CW_ERR_ARG, "iguiding > 0 needs weights_g");
      for (int i = 0; i < h.nstates; i++) h.wg[i] = d->weights_g[i];
      if (!(h.wg[0] > 0)) return fail(c, CW_ERR_ARG, "weights_g of state 1 must be positive");
    }
  }
  h.mrwf = d->mrwf; h.mpts = d->mrwf_pts; h.mbastyp = d->mbastyp;
  int m = 0;
  std::vector<int> ao_first(d->ncent + 1);
  for (int ic = 0; ic < d->ncent; ic++) {
    ao_first[ic] = m;
    m += d->nbastyp[d->iwctype[ic]];
  }
  ao_first[d->ncent] = m;
  if (m != d->nbasis) return fail(c, CW_ERR_ARG, "sum of nbastyp over centres (%d) != nbasis (%d)", m, d->nbasis);
  for (int it = 0; it < d->nctype; it++) {
    h.znuc[it] = d->znuc[it];
    h.nrbas[it] = d->nrbas[it]; h.igrid[it] = d->igrid[it]; h.nr[it] = d->nr[it];
    h.nbastyp[it] = d->nbastyp[it];
    h.arg[it] = d->arg[it]; h.r0[it] = d->r0[it];
    for (int irb = 0; irb < d->nrbas[it]; irb++) {
      const int src = irb + d->mrwf * it;
      h.rmaxwf[it * CW_MAX_RWF + irb] = d->rmaxwf[src];
      for (int k = 0; k < 5; k++) h.ce[(it * CW_MAX_RWF + irb) * 5 + k] = d->ce[src * CW_NCOEF + k];
      for (int k = 0; k < 2; k++) h.ae[(it * CW_MAX_RWF + irb) * 2 + k] = d->ae[src * 2 + k];
    }
    for (int k = 0; k <= d->norda; k++) h.a4[it * (d->norda + 1) + k] = d->a4[it * (d->norda + 1) + k];
    for (int k = 0; k < h.nterms; k++) {
      h.c[it * CW_MAX_TERMS + k] = d->c[it * h.nterms + k];
      h.cf[it * CW_MAX_TERMS + k] = (float)d->c[it * h.nterms + k];
    }
    if (d->nloc) {
      h.lpot[it] = d->lpot[it];
      for (int l = 0; l < CW_MPS_L; l++) {
        h.necp_term[it * 4 + l] = d->necp_term[it * CW_MPS_L + l];
        for (int k = 0; k < CW_MGAUSS; k++) {
          const int s = (it * CW_MPS_L + l) * CW_MGAUSS + k;
          h.necp_power[(it * 4 + l) * 16 + k] = d->necp_power[s];
          h.ecp_exponent[(it * 4 + l) * 16 + k] = d->ecp_exponent[s];
          h.ecp_coef[(it * 4 + l) * 16 + k] = d->ecp_coef[s];
        }
      }
    }
  }
  for (int isb = 0; isb < d->nspin2b; isb++)
    for (int k = 0; k <= d->nordb; k++) h.b[isb * (d->nordb + 1) + k] = d->b[isb * (d->nordb + 1) + k];
  for (int q = 0; q < h.nquad; q++) {
    h.xq0[q] = d->xq0[q]; h.yq0[q] = d->yq0[q]; h.zq0[q] = d->zq0[q]; h.wq[q] = d->wq[q];
  }
  // set_scale_dist (vmc/scale_dist.f90:3-55)
  h.asymp_r = 1.0 / h.scalek;
  for (int it = 0; it < d->nctype; it++) {
    const double *a = &h.a4[it * (d->norda + 1)];
    double v = a[0] * h.asymp_r / (1 + a[1] * h.asymp_r);
    for (int iord = 2; iord <= d->norda; iord++) v += a[iord] * std::pow(h.asymp_r, iord);
    h.asymp_jasa[it] = v;
  }
  for (int i = 0; i < 2; i++) {
    double sspinn;
    int isp;
    if (i == 0) { sspinn = 1; isp = 0; }
    else { sspinn = (d->nspin2b == 1 && d->nocuspb == 0) ? 0.5 : 1.0; isp = d->nspin2b - 1; }
    const double *bb = &h.b[isp * (d->nordb + 1)];
    double v = sspinn * bb[0] * h.asymp_r / (1 + bb[1] * h.asymp_r);
    for (int iord = 2; iord <= d->nordb; iord++) v += bb[iord] * std::pow(h.asymp_r, iord);
    h.asymp_jasb[i] = v;
  }
  {
    // Slm monomials (vmc/slm.f90 index table)
    static const int A[36] = {0, 0, 1, 0, 0, 2, 1, 1, 0, 0, 0, 3, 2, 2, 1, 1, 1, 0, 0, 0, 0,
                              4, 3, 3, 2, 2, 2, 1, 1, 1, 1, 0, 0, 0, 0, 0};
    static const int B[36] = {0, 0, 0, 1, 0, 0, 1, 0, 2, 1, 0, 0, 1, 0, 2, 1, 0, 3, 2, 1, 0,
                              0, 1, 0, 2, 1, 0, 3, 2, 1, 0, 4, 3, 2, 1, 0};
    static const int Cz[36] = {0, 0, 0, 0, 1, 0, 0, 1, 0, 1, 2, 0, 0, 1, 0, 1, 2, 0, 1, 2, 3,
                               0, 0, 1, 0, 1, 2, 0, 1, 2, 3, 0, 1, 2, 3, 4};
    const double cs_ = 0.28209479177387814, cp = 0.48860251190291992, cd1 = 0.630783130505040,
                 cd2 = 1.092548430592079, cf = 0.74635266518023078, cf2 = 1.66889529453113635,
                 cf3 = 2.89061144264055405, cg = 0.8462843753216345, cg2 = 2.2390579955406924,
                 cg3 = 2.890611442640554, cg4 = 5.006685883593409;
    const double K_[36] = {0,   cs_, cp,  cp,  cp,  cd1, cd2, cd2, cd1, cd2, cd1, cf,
                           cf2, cf2, cf2, cf3, cf2, cf,  cf2, cf2, cf,  cg,  cg2, cg2,
                           cg3, cg4, cg3, cg2, cg4, cg4, cg2, cg,  cg2, cg3, cg2, cg};
    for (int l = 0; l < 36; l++) {
      h.slm_a[l] = A[l];
      h.slm_b[l] = B[l];
      h.slm_c[l] = Cz[l];
      h.slm_k[l] = K_[l];
    }
  }
  // global tables
  auto &L = c->sys_allocs;
  {
    double *cent;
    int *iwct, *aof;
    DALLOC(L, cent, 3 * (size_t)d->ncent);
    DALLOC(L, iwct, d->ncent);
    DALLOC(L, aof, d->ncent + 1);
    CK(cudaMemcpy(cent, d->cent, 3 * (size_t)d->ncent * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(iwct, d->iwctype, d->ncent * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(aof, ao_first.data(), (d->ncent + 1) * sizeof(int), cudaMemcpyHostToDevice));
    h.cent = cent;
    h.iwctype = iwct;
    h.ao_first = aof;
  }
  const size_t nt = (size_t)d->nctype * d->mrwf * d->mrwf_pts;
  double *rwf, *d2rwf, *coefT;
  int *iwl, *iwr, *slot;
  DALLOC(L, rwf, nt);
  DALLOC(L, d2rwf, nt);
  CK(cudaMemcpy(rwf, d->rwf, nt * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d2rwf, d->d2rwf, nt * sizeof(double), cudaMemcpyHostToDevice));
  const size_t nb = (size_t)d->nctype * d->mbastyp;
  DALLOC(L, iwl, nb);
  DALLOC(L, iwr, nb);
  CK(cudaMemcpy(iwl, d->iwlbas, nb * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(iwr, d->iwrwf, nb * sizeof(int), cudaMemcpyHostToDevice));
  // coefT[m][o] = coef(m,o)
  std::vector<double> ct((size_t)d->nbasis * d->norb);
  for (int o = 0; o < d->norb; o++)
    for (int mm = 0; mm < d->nbasis; mm++) ct[(size_t)mm * d->norb + o] = d->coef[(size_t)o * d->nbasis + mm];
  DALLOC(L, coefT, ct.size());
  CK(cudaMemcpy(coefT, ct.data(), ct.size() * sizeof(double), cudaMemcpyHostToDevice));
  c->ref_orb.assign(d->iworbd, d->iworbd + d->nelec);
  for (int &v : c->ref_orb) v -= 1;
  std::vector<int> so(2 * nmax, 0);
  for (int j = 0; j < d->nup; j++) so[j] = d->iworbd[j] - 1;
  for (int j = 0; j < ndn; j++) so[nmax + j] = d->iworbd[d->nup + j] - 1;
  for (int v : so)
    if (v < 0 || v >= d->norb) return fail(c, CW_ERR_ARG, "iworbd entry out of range");
  DALLOC(L, slot, so.size());
  CK(cudaMemcpy(slot, so.data(), so.size() * sizeof(int), cudaMemcpyHostToDevice));
  // c~ as one GEMM over all walkers and both spins (slmi rows x occupied
  // coefficient rows) when both spins fill nmax slots with the same orbitals
  bool same_occ = d->nup == nmax && ndn == nmax && nmax % 2 == 0 && d->nbasis % 2 == 0;
  for (int j = 0; same_occ && j < nmax; j++) same_occ = so[j] == so[nmax + j];
  if (same_occ && d->nloc) {
    std::vector<double> bo((size_t)nmax * d->nbasis);
    for (int j = 0; j < nmax; j++)
      for (int mm = 0; mm < d->nbasis; mm++) bo[(size_t)j * d->nbasis + mm] = d->coef[(size_t)so[j] * d->nbasis + mm];
    DALLOC(L, c->bocc, bo.size());
    CK(cudaMemcpy(c->bocc, bo.data(), bo.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  // r0*arg^(jx-1) of every grid point (splfit's ref0 for igrid 2 and 3)
  std::vector<double> gpw((size_t)d->nctype * (d->mrwf_pts + 1), 0.0);
  for (int it = 0; it < d->nctype; it++)
    for (int jx = 1; jx <= d->mrwf_pts; jx++)
      gpw[(size_t)it * (d->mrwf_pts + 1) + jx] = d->r0[it] * std::pow(d->arg[it], jx - 1);
  double *gridpow;
  DALLOC(L, gridpow, gpw.size());
  CK(cudaMemcpy(gridpow, gpw.data(), gpw.size() * sizeof(double), cudaMemcpyHostToDevice));
  c->g.rwf = rwf; c->g.d2rwf = d2rwf; c->g.iwlbas = iwl; c->g.iwrwf = iwr; c->g.coefT = coefT; c->g.slot_orb = slot;
  c->g.gridpow = gridpow;
  std::vector<int4> aot(d->nbasis);
  for (int ic = 0; ic < d->ncent; ic++) {
    const int it = d->iwctype[ic];
    for (int ib = 0; ib < d->nbastyp[it]; ib++) {
      const int mm = ao_first[ic] + ib;
      aot[mm] = make_int4(ic, d->iwrwf[it * d->mbastyp + ib] - 1, it, d->iwlbas[it * d->mbastyp + ib]);
      if (aot[mm].w < 1 || aot[mm].w > 35 || aot[mm].y < 0 || aot[mm].y >= d->nrbas[it])
        return fail(c, CW_ERR_ARG, "basis pointer out of range (centre %d, AO %d)", ic, ib);
    }
  }
  int4 *aodev;
  DALLOC(L, aodev, aot.size());
  CK(cudaMemcpy(aodev, aot.data(), aot.size() * sizeof(int4), cudaMemcpyHostToDevice));
  c->g.ao = aodev;
  // per-AO radial-table offset, grid size, Slm exponents / constant, rmaxwf
  std::vector<int4> aox(d->nbasis);
  std::vector<double2> aok(d->nbasis);
  for (int mm = 0; mm < d->nbasis; mm++) {
    const int irb = aot[mm].y, it = aot[mm].z, l = aot[mm].w;
    aox[mm] = make_int4((irb + h.mrwf * it) * h.mpts, h.nr[it], h.slm_a[l] | (h.slm_b[l] << 8) | (h.slm_c[l] << 16), 0);
    aok[mm] = make_double2(h.slm_k[l], h.rmaxwf[it * CW_MAX_RWF + irb]);
  }
  int4 *aoxdev;
  double2 *aokdev;
  DALLOC(L, aoxdev, aox.size());
  DALLOC(L, aokdev, aok.size());
  CK(cudaMemcpy(aoxdev, aox.data(), aox.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(aokdev, aok.data(), aok.size() * sizeof(double2), cudaMemcpyHostToDevice));
  c->g.aox = aoxdev;
  c->g.aok = aokdev;
  std::vector<double2> cen(2 * (size_t)d->ncent);
  for (int ic = 0; ic < d->ncent; ic++) {
    cen[2 * ic] = make_double2(d->cent[3 * ic], d->cent[3 * ic + 1]);
    cen[2 * ic + 1] = make_double2(d->cent[3 * ic + 2], (double)d->iwctype[ic]);
  }
  double2 *cendev;
  DALLOC(L, cendev, cen.size());
  CK(cudaMemcpy(cendev, cen.data(), cen.size() * sizeof(double2), cudaMemcpyHostToDevice));
  c->g.cen = cendev;
  // dynamic shared memory sizes
  {
    const int nord = h.nordc <= 1 ? 1 : h.nordc;
    c->smem_jmove = sizeof(double) * 4 * (size_t)h.M * (8 + 2 * een_nb(nord));
    c->smem_jmove_f32 = sizeof(float) * 4 * (size_t)h.M * (8 + 2 * een_nbp(nord));
  }
  {
    const int nord = h.nordc <= 1 ? 1 : h.nordc;
    c->smem_jfull = sizeof(double) * (3 * (size_t)h.N + 1 + 2 * (size_t)h.M * 8 + 2 * (size_t)h.M * 4 * een_nb(nord));
    // FP32: the folded rows in floats, then the rows' fields in floats
    c->smem_jfull_f32 = sizeof(double) * (3 * (size_t)h.N + 1 + 2 * (size_t)h.M * 8) +
                        sizeof(float) * (2 * (size_t)h.M * 4 * een_nb(nord) + 2 * (size_t)h.M * 8);
  }
  // spins whose n x n inverse does not fit in shared memory (about 160
  // electrons and up): the inverse and c~ kernels work on global memory
  c->big_spin = sizeof(double) * ((size_t)nmax * nmax + (size_t)nmax * 64) > 200 * 1024 ? 1 : 0;
  c->smem_sinv = sizeof(double) * ((c->big_spin ? 0 : (size_t)nmax * nmax) + nmax);
  c->smem_ctil = sizeof(double) * ((c->big_spin ? 0 : (size_t)nmax * nmax) + (size_t)nmax * 64);
  {
    const int nord = h.nordc <= 1 ? 1 : h.nordc;
  }
  // warp-per-point basis kernels: as many warps per block as 4 records fit
  c->basis_warps = (int)std::max<size_t>(1, std::min<size_t>(4, (160 * 1024) / ((size_t)h.M * kCenRec * sizeof(double))));
  c->smem_basis = (size_t)c->basis_warps * h.M * kCenRec * sizeof(double);
  CK(raise_smem(c, k_basis_move, (size_t)(c->smem_basis)));
  CK(raise_smem(c, k_basis_all, (size_t)(c->smem_basis)));
  CK(raise_smem(c, k_slater_inv, (size_t)(c->smem_sinv)));
  CK(raise_smem(c, k_ctilde, (size_t)(c->smem_ctil)));
  CK(raise_smem(c, k_dgemm_mma<32>, mma_smem(32)));
  CK(raise_smem(c, k_dgemm_mma<48>, mma_smem(48)));
  CK(raise_smem(c, k_dgemm_mma<64>, mma_smem(64)));
  CK(raise_smem(c, k_dgemm_mma<80>, mma_smem(80)));
  c->mixed = precision == CW_PREC_MIXED;
  c->ecp_naov = d->ndet > 1 ? h.K : 0;  // the ECP stage keeps the point's basis values for the B matrix
  int rc = nord_attrs(c);
  if (rc) return rc;
  if (d->ndet > 1) {
    // compact multideterminant tables (multideterminants_define)
    std::vector<int> exc, kw;
    std::vector<double> cdet, sgn;
    int nuniq[2], ivirt[2], iactv[2], numax = 1;
    rc = md_define(c, d, exc, kw, cdet, nuniq, ivirt, iactv, numax, sgn);
    if (rc) return rc;
    h.ndet = d->ndet;
    for (int s2 = 0; s2 < 2; s2++) {
      h.md_nuniq[s2] = nuniq[s2];
      h.md_ivirt[s2] = ivirt[s2];
      h.md_iactv[s2] = iactv[s2];
    }
    int *dexc, *dkw;
    double *dcd;
    DALLOC(L, dexc, exc.size());
    DALLOC(L, dkw, kw.size());
    DALLOC(L, dcd, cdet.size());
    CK(cudaMemcpy(dexc, exc.data(), sizeof(int) * exc.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dkw, kw.data(), sizeof(int) * kw.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dcd, cdet.data(), sizeof(double) * cdet.size(), cudaMemcpyHostToDevice));
    c->mdt = MdTab{dexc, dkw, dcd, numax};
    DALLOC(L, c->md_sgn, sgn.size());
    CK(cudaMemcpy(c->md_sgn, sgn.data(), sizeof(double) * sgn.size(), cudaMemcpyHostToDevice));
    c->md_on = true;
    if (h.nloc > 0 && c->ecp_naov != h.K)  // the ECP block's basis-value rows must be sized
      return fail(c, CW_ERR_STATE, "ECP stage sized without multideterminant basis rows");
    const size_t O = h.Oa;
    c->smem_md_hpsi = sizeof(double) * (4 * (size_t)nmax * nmax + (h.nstates > 1 ? 3 : 1) * (size_t)nmax * O + numax + 1);
    c->smem_md_phase = sizeof(double) * ((size_t)numax + 1);
    c->smem_md_move = sizeof(double) * (2 * (size_t)nmax + 4 * O + (size_t)nmax * O + 3 * (size_t)nmax);
    c->smem_md_drift = sizeof(double) * ((size_t)nmax + 3 * O + (size_t)nmax * O + 3 * (size_t)nmax);
    c->smem_md_tmove = sizeof(double) * (2 * O + (size_t)nmax + h.K + (h.K & 1) + 4 * (size_t)h.M * kCenRec);
    const size_t lim = 227 * 1024;
    if (c->smem_md_hpsi > lim || c->smem_md_move > lim)
      return fail(c, CW_ERR_UNSUPPORTED, "multideterminant tables exceed shared memory (nmax %d, norb %d, %d unique)",
                  nmax, h.Oa, numax);
    CK(raise_smem(c, k_md_hpsi, (size_t)(c->smem_md_hpsi)));
    CK(raise_smem(c, k_md_phase, (size_t)(c->smem_md_phase)));
    CK(raise_smem(c, k_md_move, (size_t)(c->smem_md_move)));
    CK(raise_smem(c, k_md_drift_old, (size_t)(c->smem_md_drift)));
    {
      const size_t zs = sizeof(double) * ((size_t)O * nmax + (size_t)nmax * nmax);
      if (zs <= lim) CK(raise_smem(c, k_md_orb_o, zs));
    }
    if (c->smem_md_tmove <= lim) CK(raise_smem(c, k_md_tmove, (size_t)(c->smem_md_tmove)));
  }
  if (precision == CW_PREC_MIXED) {
    // tensor-core LCAO: coefficients split once into TF32 hi/lo, [Oa][kp]
    c->mixed = true;
    c->kp = (h.K + 31) / 32 * 32;
    c->np = (h.Oa + 15) / 16 * 16;
    if (c->np > 256) return fail(c, CW_ERR_UNSUPPORTED, "mixed precision: more than 256 orbitals");
    c->umma_st = umma_stages(c->np);
    c->smem_umma = umma_smem_bytes(c->np);
    CK(raise_smem(c, k_lcao_tf32x3, (size_t)(c->smem_umma)));
    double *cA;
    DALLOC(L, cA, (size_t)h.Oa * h.K);
    CK(cudaMemcpy(cA, d->coef, sizeof(double) * (size_t)h.Oa * h.K, cudaMemcpyHostToDevice));
    DALLOC(L, c->coef_hi, (size_t)h.Oa * c->kp);
    DALLOC(L, c->coef_lo, (size_t)h.Oa * c->kp);
    const long n = (long)h.Oa * c->kp;
    k_split_rows<<<(unsigned)((n + 255) / 256), 256>>>(cA, h.Oa, h.K, c->coef_hi, c->coef_lo, c->kp);
    LCHK("k_split_rows");
    CK(cudaDeviceSynchronize());
    DALLOC(L, c->d_err, 1);
    CK(cudaMemset(c->d_err, 0, sizeof(int)));
    rc = make_map(c, &c->tm_b_hi, c->coef_hi, h.K, h.Oa, c->kp, c->np);
    if (!rc) rc = make_map(c, &c->tm_b_lo, c->coef_lo, h.K, h.Oa, c->kp, c->np);
    if (rc) return rc;
  }
  return CW_OK;
}

void cw_destroy(cw_ctx *c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_dmc(c);
  free_list(c, c->w_allocs);
  drop_sweep_graph(c);
  free_list(c, c->opt_allocs);
  free_list(c, c->sys_allocs);
  if (c->d_stamps) cudaFree(c->d_stamps);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->ev_jas) cudaEventDestroy(c->ev_jas);
  for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char *cw_last_error(const cw_ctx *c) { return c ? c->err.c_str() : "null context"; }
size_t cw_device_bytes(const cw_ctx *c) { return c ? c->dev_bytes : 0; }

int cw_sync(cw_ctx *c) {
  if (!c) return CW_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  return CW_OK;
}

double cw_last_ms(const cw_ctx *c) { return c ? c->last_ms : 0.0; }

long cw_launches(const cw_ctx *c) { return c ? c->launches : 0; }

int cw_profile(cw_ctx *c, int enable) {
  if (!c) return CW_ERR_ARG;
  c->prof = enable != 0;
  for (int k = 0; k < CW_NSTAGE; k++) {
    c->stage_ms[k] = 0;
    c->stage_n[k] = 0;
  }
  c->evused = 0;
  return CW_OK;
}

int cw_stage_times(cw_ctx *c, double *ms, long *launches) {
  if (!c) return CW_ERR_ARG;
  for (int k = 0; k < CW_NSTAGE; k++) {
    if (ms) ms[k] = c->stage_ms[k];
    if (launches) launches[k] = c->stage_n[k];
  }
  return CW_OK;
}

int cw_set_walkers(cw_ctx *c, int nwalk, const double *x, const uint64_t *rng) {
  if (!c || nwalk <= 0 || !x || !rng) return fail(c, CW_ERR_ARG, "cw_set_walkers: bad arguments");
  BIND(c);
  if (nwalk != c->W) {
    int rc = alloc_walkers(c, nwalk);
    if (rc) return rc;
  }
  // the caller's array as it is (one copy; pinned memory goes straight to
  // the device), reordered on the device
  const int N = c->h.N;
  const long nt = (long)nwalk * N;
  CK(cudaMemcpyAsync(c->xstage, x, sizeof(double) * 3 * nt, cudaMemcpyHostToDevice, c->stream));
  k_x_from_host<<<(unsigned)((nt + 127) / 128), 128, 0, c->stream>>>(nwalk, N, c->xstage, c->st.x);
  LCHK("k_x_from_host");
  CK(cudaMemcpyAsync(c->st.rng, rng, sizeof(uint64_t) * 4 * nwalk, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->st.status, 0, sizeof(int) * nwalk, c->stream));
  return zerest(c);
}

int cw_autotune(cw_ctx *c, int reps, int32_t *choice) {
  if (!c) return CW_ERR_ARG;
  if (c->W == 0) return fail(c, CW_ERR_STATE, "cw_autotune: no walkers");
  BIND(c);
  const CSys &h = c->h;
  reps = std::max(1, reps);
  // N tile of the FP64 tensor-core LCAO for this context's two shapes (the
  // move's 4 rows per walker, the all-electron chunk's 5 rows per electron):
  // each candidate timed on the context's own scratch buffers, which every
  // sweep rewrites before reading, so the walk is untouched
  auto tune = [&](int M, const double *A, double *C, int &best) -> int {
    float tbest = 0;
    for (int bn : kMmaTiles) {
      dgemm(c->stream, M, h.Oa, h.K, A, c->g.coefT, C, bn);  // warm-up
      CK(cudaEventRecord(c->ev0, c->stream));
      for (int r = 0; r < reps; r++) dgemm(c->stream, M, h.Oa, h.K, A, c->g.coefT, C, bn);
      CK(cudaEventRecord(c->ev1, c->stream));
      CK(cudaEventSynchronize(c->ev1));
      LCHK("dgemm(autotune)");
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
      if (bn == kMmaTiles[0] || ms < tbest) {
        tbest = ms;
        best = bn;
      }
    }
    return CW_OK;
  };
  if (!c->mixed) {
    if (int rc = tune(c->W * 4, c->mb.phi, c->mb.orbn, c->gemm_bn_move)) return rc;
    if (int rc = tune(c->W * c->hb.chunk * 5, c->hb.phi, c->hb.orball, c->gemm_bn_all)) return rc;
  }
  drop_sweep_graph(c);  // the next sweep is captured with the chosen tiles
  if (choice) {
    choice[0] = c->gemm_bn_move;
    choice[1] = c->gemm_bn_all;
  }
  return CW_OK;
}

int cw_stamp(cw_ctx *c) {
  if (!c) return CW_ERR_ARG;
  BIND(c);
  if (!c->d_stamps) {
    CK(cudaMalloc(&c->d_stamps, sizeof(unsigned long long) * kStampCap));
    c->dev_bytes += sizeof(unsigned long long) * kStampCap;
  }
  if (c->nstamp >= kStampCap) return fail(c, CW_ERR_STATE, "more than %d stamps", kStampCap);
  k_stamp<<<1, 1, 0, c->stream>>>(c->d_stamps + c->nstamp);
  LCHK("k_stamp");
  c->nstamp++;
  return CW_OK;
}

int cw_stamps(cw_ctx *c, int64_t *ns, int n) {
  if (!c || (n > 0 && !ns)) return CW_ERR_ARG;
  const int m = std::min(n, c->nstamp);
  if (m > 0) {
    CK(cudaMemcpyAsync(ns, c->d_stamps, sizeof(int64_t) * m, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return c->nstamp;
}

int cw_walker_status(cw_ctx *c, int32_t *status) {
  if (!c || !status) return CW_ERR_ARG;
  if (c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  CK(cudaMemcpyAsync(status, c->st.status, sizeof(int) * c->W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CW_OK;
}

int cw_get_walkers(cw_ctx *c, double *x, uint64_t *rng) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  const int N = c->h.N, W = c->W;
  BIND(c);
  if (x) {
    const long nt = (long)W * N;
    k_x_to_host<<<(unsigned)((nt + 127) / 128), 128, 0, c->stream>>>(W, N, c->st.x, c->xstage);
    LCHK("k_x_to_host");
    CK(cudaMemcpyAsync(x, c->xstage, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost, c->stream));
  }
  if (rng) CK(cudaMemcpyAsync(rng, c->st.rng, sizeof(uint64_t) * 4 * W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CW_OK;
}

// ---------------------------------------------------------------------------
// Per-electron routines for a driver that keeps metrop6 on the host
// (psie, compute_determinante_grad, detsav + jassav, update_ymat), batched
// over the walkers of a VMC population.  Host arrays in, host arrays out.
// ---------------------------------------------------------------------------
int hook_check(cw_ctx *c, int iel, const char *what) {
  if (!c) return CW_ERR_ARG;
  if (c->W == 0) return fail(c, CW_ERR_STATE, "%s: no walkers", what);
  if (c->dmc.on) return fail(c, CW_ERR_STATE, "%s: the population is a DMC population", what);
  if (iel < 0 || iel >= c->h.N) return fail(c, CW_ERR_ARG, "%s: electron %d outside [0, %d)", what, iel, c->h.N);
  return CW_OK;
}

// multideterminant move tables of electron iel at the current configuration
// (spin-phase sums at the first electron of a spin, drift correction at the
// old position): what the engine's own sweep does before each proposal
int hook_md_prepare(cw_ctx *c, int iel) {
  if (!c->md_on || c->hook_md_iel == iel) return CW_OK;
  int rc = md_before_propose(c, iel);
  if (rc) return rc;
  c->hook_md_iel = iel;
  return CW_OK;
}

extern "C" int cw_psie(cw_ctx *c, int iel, const double *xnew, double *psid, double *psij) {
  if (int rc = hook_check(c, iel, "cw_psie")) return rc;
  if (!xnew) return fail(c, CW_ERR_ARG, "cw_psie: xnew is NULL");
  BIND(c);
  const int W = c->W;
  if (int rc = hook_md_prepare(c, iel)) return rc;
  CK(cudaMemcpyAsync(c->hook_buf, xnew, sizeof(double) * 3 * W, cudaMemcpyHostToDevice, c->stream));
  k_hook_place<<<(W + 127) / 128, 128, 0, c->stream>>>(c->h, c->st, c->mb, c->hook_buf);
  LCHK("k_hook_place");
  NORD_DISPATCH(launch_jmove, c, iel);
  LCHK("k_jastrow_move");
  const int bw = c->basis_warps;
  k_basis_move<<<(unsigned)((W + bw - 1) / bw), 32 * bw, c->smem_basis, c->stream>>>(c->h, c->st, c->mb, c->g);
  LCHK("k_basis_move");
  if (int rc = lcao(c, true, W * 4, c->mb.phi, c->mb.orbn)) return rc;
  if (int rc = md_after_lcao(c, iel)) return rc;
  double *out = c->hook_buf + (size_t)3 * W;
  k_hook_ratio<<<(W * kMoveGroup + 127) / 128, 128, 0, c->stream>>>(c->h, c->st, c->mb, c->g, iel, out);
  LCHK("k_hook_ratio");
  std::vector<double> h((size_t)2 * W);
  CK(cudaMemcpyAsync(h.data(), out, sizeof(double) * 2 * W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (int rc = check_status(c)) return rc;
  for (int w = 0; w < W; w++) {
    if (psid) psid[w] = h[2 * w];
    if (psij) psij[w] = h[2 * w + 1];
  }
  c->hook_psie_iel = iel;
  return CW_OK;
}

extern "C" int cw_grad(cw_ctx *c, int iel, int iflag_move, double *vd) {
  if (int rc = hook_check(c, iel, "cw_grad")) return rc;
  if (!vd) return fail(c, CW_ERR_ARG, "cw_grad: vd is NULL");
  if (iflag_move != 0 && iflag_move != 1)
    return fail(c, CW_ERR_ARG, "cw_grad: iflag_move %d (1: current position, 0: point of the last cw_psie)",
                iflag_move);
  if (iflag_move == 0 && c->hook_psie_iel != iel)
    return fail(c, CW_ERR_STATE, "cw_grad(iflag_move=0) of electron %d needs its cw_psie first", iel);
  BIND(c);
  const int W = c->W;
  if (iflag_move == 1) {
    if (int rc = hook_md_prepare(c, iel)) return rc;
  }
  double *out = c->hook_buf + (size_t)3 * W;
  k_hook_grad<<<(W * kMoveGroup + 127) / 128, 128, 0, c->stream>>>(c->h, c->st, c->mb, c->g, iel, iflag_move, out);
  LCHK("k_hook_grad");
  CK(cudaMemcpyAsync(vd, out, sizeof(double) * 3 * W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CW_OK;
}

extern "C" int cw_commit(cw_ctx *c, int iel, const int32_t *accept) {
  if (int rc = hook_check(c, iel, "cw_commit")) return rc;
  if (!accept) return fail(c, CW_ERR_ARG, "cw_commit: accept is NULL");
  if (c->hook_psie_iel != iel)
    return fail(c, CW_ERR_STATE, "cw_commit of electron %d needs its cw_psie first", iel);
  BIND(c);
  const int W = c->W;
  CK(cudaMemcpyAsync(c->hook_acc, accept, sizeof(int) * W, cudaMemcpyHostToDevice, c->stream));
  k_hook_accept<<<(W + 127) / 128, 128, 0, c->stream>>>(c->h, c->st, c->mb, iel, c->hook_acc);
  LCHK("k_hook_accept");
  launch_commit(c, iel);
  LCHK("k_commit");
  if (int rc = md_after_commit(c, iel)) return rc;
  // the walk's tables changed: a cw_graph-captured sweep stays valid (same
  // buffers), the prepared multideterminant tables of this electron do not
  c->hook_psie_iel = -1;
  c->hook_md_iel = -1;
  CK(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

extern "C" int cw_update_ymat(cw_ctx *c, int iel) {
  if (int rc = hook_check(c, iel, "cw_update_ymat")) return rc;
  if (!c->md_on || iel + 1 >= c->h.N) return CW_OK;
  BIND(c);
  if (int rc = hook_md_prepare(c, iel + 1)) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return CW_OK;
}

// One metrop6 sweep of every walker: rotqua, the single-electron moves of
// every electron, the sweep's hpsi and sums (and the optimisation sums).
int vmc_sweep(cw_ctx *c) {
  const CSys &h = c->h;
  const int W = c->W;
  if (h.nloc > 0) {
    stage_begin(c, CW_ST_ROTQUA);
    k_rotqua<<<(W + 127) / 128, 128, 0, c->stream>>>(c->h, c->st);
    stage_end(c);
    LCHK("k_rotqua");
  }
  for (int i = 0; i < h.N; i++) {
    if (int rc = md_before_propose(c, i)) return rc;
    stage_begin(c, CW_ST_PROPOSE);
    k_propose<<<(W * kMoveGroup + 127) / 128, 128, 0, c->stream>>>(c->h, c->st, c->mb, i,
                                                                  c->smem_commit ? c->acc_count : nullptr);
    stage_end(c);
    LCHK("k_propose");
    // the move Jastrow and the basis + LCAO of the proposed point depend only
    // on the proposal: outside profiling they run side by side (the basis
    // and LCAO on the side stream, joined before the decision)
    const bool fork = !c->prof;
    if (fork) {
      CK(cudaEventRecord(c->ev_fork, c->stream));
      CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    }
    stage_begin(c, CW_ST_JASTROW_MOVE);
    NORD_DISPATCH(launch_jmove, c, i);
    stage_end(c);
    LCHK("k_jastrow_move");
    cudaStream_t bs = fork ? c->side : c->stream;
    const int bw = c->basis_warps;
    stage_begin(c, CW_ST_BASIS_MOVE);
    k_basis_move<<<(unsigned)((W + bw - 1) / bw), 32 * bw, c->smem_basis, bs>>>(c->h, c->st, c->mb, c->g);
    stage_end(c);
    LCHK("k_basis_move");
    stage_begin(c, CW_ST_LCAO_MOVE);
    {
      int rc = lcao(c, true, W * 4, c->mb.phi, c->mb.orbn, bs);
      stage_end(c);
      if (rc) return rc;
    }
    if (int rc = md_after_lcao(c, i, bs)) return rc;  // needs the proposal and the LCAO only
    if (fork) {
      CK(cudaEventRecord(c->ev_join, c->side));
      CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    }
    stage_begin(c, CW_ST_ACCEPT);
    k_decide<<<(W * kMoveGroup + 127) / 128, 128, 0, c->stream>>>(c->h, c->st, c->mb, c->g, i,
                                                                 c->smem_commit ? c->acc_list : nullptr, c->acc_count);
    stage_end(c);
    LCHK("k_decide");
    stage_begin(c, CW_ST_COMMIT);
    launch_commit(c, i, true);
    stage_end(c);
    LCHK("k_commit");
    if (int rc = md_after_commit(c, i)) return rc;
  }
  int rc = run_hpsi(c, 1);
  if (rc) return rc;
  if (c->opt_np > 0) {
    rc = opt_accum(c);
    if (rc) return rc;
  }
  return CW_OK;
}

// The sweep's launch sequence is the same every sweep (pointers, electrons,
// shapes), so it is captured once into a CUDA graph and replayed: one launch
// per sweep instead of ~6N+20.  Profiling (per-stage events) runs the launches
// directly; a new population, optimisation sums or a restore re-capture.
// the sweep's launches captured into c->sweep_graph (and instantiated) if
// the population changed or nothing is captured yet
static int ensure_sweep_graph(cw_ctx *c) {
  if (c->sweep_exec && c->sweep_w != c->W) drop_sweep_graph(c);
  if (c->sweep_exec) return CW_OK;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  const long l0 = c->launches;
  int rc = vmc_sweep(c);
  cudaGraph_t gph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &gph);
  if (rc || e != cudaSuccess) {
    if (gph) cudaGraphDestroy(gph);
    if (rc) return rc;
    return fail(c, CW_ERR_CUDA, "sweep capture failed: %s", cudaGetErrorString(e));
  }
  c->sweep_graph = gph;
  c->sweep_launches = c->launches - l0;
  c->sweep_w = c->W;
  c->sweep_gen++;
  c->launches = l0;
  CK(cudaGraphInstantiate(&c->sweep_exec, c->sweep_graph, 0));
  return CW_OK;
}

int cw_vmc_steps(cw_ctx *c, int nstep) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  BIND(c);
  c->launches = 0;
  CK(cudaEventRecord(c->ev0, c->stream));
  if (c->prof) {
    for (int s = 0; s < nstep; s++) {
      int rc = vmc_sweep(c);
      if (rc) return rc;
      if (c->evused > 4096) stage_collect(c);
    }
  } else {
    if (int rc = ensure_sweep_graph(c)) return rc;
    for (int s = 0; s < nstep; s++) CK(cudaGraphLaunch(c->sweep_exec, c->stream));
    c->launches += (long)nstep * c->sweep_launches;
  }
  if (c->opt_np > 0) c->sr_w += (double)c->W * nstep;  // samples of the optimisation sums
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  c->passes += nstep;
  stage_collect(c);
  return check_status(c);
}

int cw_end_block(cw_ctx *c, double *block_energy) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  const int W = c->W;
  std::vector<double> s((size_t)W * 8);
  CK(cudaMemcpyAsync(s.data(), c->st.sums, sizeof(double) * s.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemsetAsync(c->st.sums, 0, sizeof(double) * s.size(), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double es = 0, wsm = 0;
  for (int w = 0; w < W; w++) {
    const double *v = &s[(size_t)w * 8];
    const double enow = v[1] / v[0];
    c->wcum += v[0];
    c->ecum += v[1];
    c->ecm2 += v[1] * enow;
    const double penow = v[2] / v[0], tpbnow = v[3] / v[0];
    c->pecm2 += v[2] * penow;
    c->tpbcm2 += v[3] * tpbnow;
    c->pecum += v[2];
    c->tpbcum += v[3];
    c->acc += v[4];
    c->ecum1s += v[5];
    c->ecm21s += v[6];
    es += v[1];
    wsm += v[0];
  }
  if (c->hb.sums_ms) {
    // acuest per state: the reweighted block sums of every walker
    const int ns = c->h.nstates;
    std::vector<double> q((size_t)W * ns * 4);
    CK(cudaMemcpyAsync(q.data(), c->hb.sums_ms, sizeof(double) * q.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemsetAsync(c->hb.sums_ms, 0, sizeof(double) * q.size(), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int w = 0; w < W; w++)
      for (int st = 0; st < ns; st++) {
        const double *v = &q[((size_t)w * ns + st) * 4];
        double *cu = &c->st_cum[(size_t)st * 5];
        const double en = v[1] / v[0];
        cu[0] += v[0];
        cu[1] += v[1];
        cu[2] += v[1] * en;
        cu[3] += v[2];
        cu[4] += v[3];
      }
  }
  c->iblk += W;
  if (block_energy) *block_energy = es / wsm;
  return CW_OK;
}

int cw_results_state(cw_ctx *c, int istate, double *out) {
  if (!c || !out) return fail(c, CW_ERR_ARG, "null argument");
  if (istate < 0 || istate >= c->h.nstates) return fail(c, CW_ERR_ARG, "state %d of %d", istate, c->h.nstates);
  if (c->h.nstates == 1) return cw_results(c, out);
  if (c->iblk == 0) return fail(c, CW_ERR_STATE, "no completed blocks");
  const double *cu = &c->st_cum[(size_t)istate * 5];
  const double ef = cu[1] / cu[0];
  out[0] = ef;
  out[1] = std::sqrt(std::fabs(cu[2] / cu[0] - ef * ef) / (double)c->iblk);
  out[2] = out[3] = out[4] = std::nan("");
  out[5] = cu[3] / cu[0];
  out[6] = cu[4] / cu[0];
  out[7] = (double)c->iblk;
  return CW_OK;
}

int cw_jas_nraw(cw_ctx *c, int *nraw) {
  if (!c || !nraw) return CW_ERR_ARG;
  const CSys &h = c->h;
  *nraw = h.nctype * (h.norda + 1) + h.nspin2b * (h.nordb + 1) + (h.nordc > 1 ? h.nctype * h.nterms : 0);
  return CW_OK;
}

int cw_opt_setup(cw_ctx *c, int ci, int njas, const double *jas_map, int with_overlap) {
  if (!c || njas < 0 || (njas > 0 && !jas_map)) return CW_ERR_ARG;
  BIND(c);
  drop_sweep_graph(c);  // the sweep gains or loses the derivative launches
  opt_reset(c);
  const int norbt = (int)c->orb_ideriv.size() / 2;
  if (!ci && njas == 0 && norbt == 0) return CW_OK;
  if (ci && !c->md_on) return fail(c, CW_ERR_UNSUPPORTED, "CI derivatives need a multideterminant expansion");
  if (c->h.nstates > 1) return fail(c, CW_ERR_UNSUPPORTED, "parameter derivatives of several states are not implemented");
  if (njas > 0 && (c->h.norda < 1 || c->h.nordb < 1))
    return fail(c, CW_ERR_UNSUPPORTED, "Jastrow derivatives need norda >= 1 and nordb >= 1 (Pade a(2), b(2))");
  if (c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  const int W = c->W, np = njas + (ci ? c->h.ndet : 0) + norbt;
  if (with_overlap && (size_t)np * np > ((size_t)1 << 27))
    return fail(c, CW_ERR_ARG, "overlap of %d parameters exceeds 2^27 entries", np);
  auto &L = c->opt_allocs;
  DALLOC(L, c->opt_o, (size_t)W * np);
  DALLOC(L, c->opt_ot, (size_t)W * np);
  DALLOC(L, c->sr_o, np);
  DALLOC(L, c->sr_eo, np);
  CK(cudaMemsetAsync(c->sr_o, 0, sizeof(double) * np, c->stream));
  CK(cudaMemsetAsync(c->sr_eo, 0, sizeof(double) * np, c->stream));
  if (with_overlap) {
    DALLOC(L, c->sr_oo, (size_t)np * np);
    DALLOC(L, c->oo_tmp, (size_t)np * np);
    CK(cudaMemsetAsync(c->sr_oo, 0, sizeof(double) * np * np, c->stream));
  }
  if (njas > 0) {
    int nraw = 0;
    cw_jas_nraw(c, &nraw);
    DALLOC(L, c->jas_raw, (size_t)W * nraw);
    DALLOC(L, c->jas_map, (size_t)nraw * njas);
    CK(cudaMemcpyAsync(c->jas_map, jas_map, sizeof(double) * nraw * njas, cudaMemcpyHostToDevice, c->stream));
    c->jas_nraw = nraw;
  }
  if (norbt > 0) {
    // rotation targets jo (each once) and per term the slots of io
    std::vector<int> vorb;
    std::vector<OrbTerm> terms(norbt);
    for (int t = 0; t < norbt; t++) {
      const int io = c->orb_ideriv[2 * t] - 1, jo = c->orb_ideriv[2 * t + 1] - 1;
      int v = -1;
      for (size_t k = 0; k < vorb.size(); k++)
        if (vorb[k] == jo) v = (int)k;
      if (v < 0) {
        v = (int)vorb.size();
        vorb.push_back(jo);
      }
      terms[t].v = v;
      terms[t].io = io;
      for (int iab = 0; iab < 2; iab++) {
        const int nel = iab == 0 ? c->h.nup : c->h.ndn, ish = iab == 0 ? 0 : c->h.nup;
        terms[t].slot[iab] = -1;
        for (int j = 0; j < nel; j++)
          if (c->ref_orb[ish + j] == io) terms[t].slot[iab] = j;
      }
    }
    c->orb_nv = (int)vorb.size();
    DALLOC(L, c->orb_terms, terms.size());
    DALLOC(L, c->orb_vorb, vorb.size());
    DALLOC(L, c->orb_vals, (size_t)W * c->h.N * c->orb_nv);
    CK(cudaMemcpyAsync(c->orb_terms, terms.data(), sizeof(OrbTerm) * terms.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->orb_vorb, vorb.data(), sizeof(int) * vorb.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->orb_on = true;
  }
  c->opt_ci = ci != 0;
  c->opt_njas = njas;
  c->opt_np = np;
  c->opt_oo = with_overlap != 0;
  c->opt_w = W;
  // derivatives at the current configurations (the last hpsi; with orbital
  // rotations the hpsi is repeated once so that it keeps the targets' values)
  if (c->orb_on)
    if (int rc = run_hpsi(c, 0)) return rc;
  if (int rc = opt_derivs(c)) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return CW_OK;
}

int cw_opt_ci(cw_ctx *c, int enable, int with_overlap) { return cw_opt_setup(c, enable, 0, nullptr, with_overlap); }

// columns [off, off+n) of the optimisation vector of every walker
static int opt_columns(cw_ctx *c, int off, int n, double *out) {
  BIND(c);
  CK(cudaMemcpy2DAsync(out, sizeof(double) * n, c->opt_o + off, sizeof(double) * c->opt_np, sizeof(double) * n,
                       c->W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CW_OK;
}

int cw_ci_o(cw_ctx *c, double *out) {
  if (!c || !out) return CW_ERR_ARG;
  if (!c->opt_ci || c->opt_w != c->W) return fail(c, CW_ERR_STATE, "CI derivatives not enabled for this population");
  return opt_columns(c, c->opt_njas, c->h.ndet, out);
}

int cw_jas_o(cw_ctx *c, double *out) {
  if (!c || !out) return CW_ERR_ARG;
  if (c->opt_njas == 0 || c->opt_w != c->W)
    return fail(c, CW_ERR_STATE, "Jastrow derivatives not enabled for this population");
  return opt_columns(c, 0, c->opt_njas, out);
}

int cw_opt_orb(cw_ctx *c, int norbterm, const int32_t *ideriv) {
  if (!c || norbterm < 0 || (norbterm > 0 && !ideriv)) return CW_ERR_ARG;
  if (norbterm > 0) {
    if (c->h.nstates > 1) return fail(c, CW_ERR_UNSUPPORTED, "orbital-rotation derivatives of several states");
    if (c->md_on && norbterm > 1024)
      return fail(c, CW_ERR_UNSUPPORTED, "orbital rotations of an expansion: at most 1024 pairs (%d)", norbterm);
    if (c->md_on && sizeof(double) * ((size_t)c->h.Oa * c->h.nmax + (size_t)c->h.nmax * c->h.nmax) > 227 * 1024)
      return fail(c, CW_ERR_UNSUPPORTED, "orbital rotations of an expansion: zmat tables exceed shared memory");
    for (int t = 0; t < norbterm; t++) {
      const int io = ideriv[2 * t], jo = ideriv[2 * t + 1];
      if (io < 1 || io > c->h.Oa || jo < 1 || jo > c->h.Oa || io == jo)
        return fail(c, CW_ERR_ARG, "orbital rotation %d: (%d, %d) outside 1..%d or io == jo", t, io, jo, c->h.Oa);
    }
  }
  c->orb_ideriv.assign(ideriv, ideriv + 2 * (size_t)norbterm);
  return CW_OK;
}

int cw_orb_o(cw_ctx *c, double *out) {
  if (!c || !out) return CW_ERR_ARG;
  if (!c->orb_on || c->opt_w != c->W)
    return fail(c, CW_ERR_STATE, "orbital-rotation derivatives not enabled for this population");
  const int nt = (int)c->orb_ideriv.size() / 2;
  return opt_columns(c, c->opt_np - nt, nt, out);
}

int cw_jas_raw(cw_ctx *c, double *out) {
  if (!c || !out) return CW_ERR_ARG;
  if (c->opt_njas == 0 || c->opt_w != c->W)
    return fail(c, CW_ERR_STATE, "Jastrow derivatives not enabled for this population");
  BIND(c);
  CK(cudaMemcpyAsync(out, c->jas_raw, sizeof(double) * c->W * c->jas_nraw, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CW_OK;
}

int cw_opt_sums(cw_ctx *c, double *o, double *eo, double *oo, double *wsum) {
  if (!c || !o || !eo || !wsum) return CW_ERR_ARG;
  if (c->opt_np == 0 || c->opt_w != c->W) return fail(c, CW_ERR_STATE, "optimisation sums not enabled for this population");
  if (oo && !c->opt_oo) return fail(c, CW_ERR_STATE, "overlap sums not enabled");
  BIND(c);
  const int nd = c->opt_np;
  CK(cudaMemcpyAsync(o, c->sr_o, sizeof(double) * nd, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(eo, c->sr_eo, sizeof(double) * nd, cudaMemcpyDeviceToHost, c->stream));
  if (oo) CK(cudaMemcpyAsync(oo, c->sr_oo, sizeof(double) * nd * nd, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemsetAsync(c->sr_o, 0, sizeof(double) * nd, c->stream));
  CK(cudaMemsetAsync(c->sr_eo, 0, sizeof(double) * nd, c->stream));
  if (c->opt_oo) CK(cudaMemsetAsync(c->sr_oo, 0, sizeof(double) * nd * nd, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *wsum = c->sr_w;
  c->sr_w = 0;
  return CW_OK;
}

int cw_opt_ci_sums(cw_ctx *c, double *o, double *eo, double *oo, double *wsum) {
  return cw_opt_sums(c, o, eo, oo, wsum);
}

int cw_state_energies(cw_ctx *c, double *energy, double *psid) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  BIND(c);
  const int W = c->W, ns = c->h.nstates;
  if (ns == 1) {
    if (energy) CK(cudaMemcpyAsync(energy, c->st.eold, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
    if (psid) CK(cudaMemcpyAsync(psid, c->st.psido, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
  } else {
    if (energy) CK(cudaMemcpyAsync(energy, c->hb.e_ms, sizeof(double) * W * ns, cudaMemcpyDeviceToHost, c->stream));
    if (psid) CK(cudaMemcpyAsync(psid, c->hb.psid_ms, sizeof(double) * W * ns, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return CW_OK;
}

int cw_results(cw_ctx *c, double *out) {
  if (!c || !out || c->iblk == 0) return fail(c, CW_ERR_STATE, "no completed blocks");
  const double passes = (double)c->passes * c->W;
  auto err = [&](double x, double x2) {
    return std::sqrt(std::fabs(x2 / c->wcum - (x / c->wcum) * (x / c->wcum)) / (double)c->iblk);
  };
  const double eerr = err(c->ecum, c->ecm2);
  const double eerr1s = std::sqrt(std::fabs(c->ecm21s / c->wcum - (c->ecum1s / c->wcum) * (c->ecum1s / c->wcum)) / passes);
  const double tcsq = eerr1s == 0 ? 0 : eerr / eerr1s;
  out[0] = c->ecum / c->wcum;
  out[1] = eerr;
  out[2] = eerr1s * std::sqrt(passes);
  out[3] = tcsq * tcsq;
  out[4] = c->acc / (passes * c->h.N);
  out[5] = c->pecum / c->wcum;
  out[6] = c->tpbcum / c->wcum;
  out[7] = (double)c->iblk;
  return CW_OK;
}

int cw_hpsi(cw_ctx *c, const double *xq, const double *yq, const double *zq, double *energy, double *psid,
            double *psij, double *ekin) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  BIND(c);
  const CSys &h = c->h;
  const int W = c->W, NQ = h.nquad;
  if (NQ > 0) {
    std::vector<double> t((size_t)W * 3 * NQ);
    for (int w = 0; w < W; w++)
      for (int q = 0; q < NQ; q++) {
        t[(size_t)w * 3 * NQ + q] = xq ? xq[q] : h.xq0[q];
        t[(size_t)w * 3 * NQ + NQ + q] = yq ? yq[q] : h.yq0[q];
        t[(size_t)w * 3 * NQ + 2 * NQ + q] = zq ? zq[q] : h.zq0[q];
      }
    CK(cudaMemcpyAsync(c->st.xq, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice, c->stream));
  }
  int rc = run_hpsi(c, 0);
  if (rc) return rc;
  rc = check_status(c);
  if (rc) return rc;
  return cw_get_state(c, energy, psid, psij) || (ekin && cudaMemcpy(ekin, c->st.ekino, sizeof(double) * W,
                                                                    cudaMemcpyDeviceToHost) != cudaSuccess)
             ? fail(c, CW_ERR_CUDA, "copy-out failed")
             : CW_OK;
}

int cw_get_state(cw_ctx *c, double *eold, double *psido, double *psijo) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  CK(cudaStreamSynchronize(c->stream));
  if (eold) CK(cudaMemcpy(eold, c->st.eold, sizeof(double) * c->W, cudaMemcpyDeviceToHost));
  if (psido) CK(cudaMemcpy(psido, c->st.psido, sizeof(double) * c->W, cudaMemcpyDeviceToHost));
  if (psijo) CK(cudaMemcpy(psijo, c->st.psijo, sizeof(double) * c->W, cudaMemcpyDeviceToHost));
  return CW_OK;
}

int cw_get_sums(cw_ctx *c, double *out) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  std::vector<double> s((size_t)c->W * 8);
  CK(cudaMemcpyAsync(s.data(), c->st.sums, sizeof(double) * s.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int w = 0; w < c->W; w++)
    for (int k = 0; k < 5; k++) out[(size_t)w * 5 + k] = s[(size_t)w * 8 + k];
  return CW_OK;
}

int cw_orbitals(cw_ctx *c, double *orb, double *dorb, double *ddorb) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  BIND(c);
  const CSys &h = c->h;
  const int W = c->W, N = h.N, M = h.M, Oa = h.Oa, K = h.K;
  const int ec = c->hb.chunk;
  std::vector<double> buf;
  for (int e0 = 0; e0 < N; e0 += ec) {
    const int ne = std::min(ec, N - e0);
    const long nwarps = (long)W * ne;
    const int bw = c->basis_warps;
    k_basis_all<<<(unsigned)((nwarps + bw - 1) / bw), 32 * bw, c->smem_basis, c->stream>>>(c->h, c->st, c->hb, c->g, e0, ne);
    LCHK("k_basis_all");
    {
      int rc = lcao(c, false, W * ne * 5, c->hb.phi, c->hb.orball);
      if (rc) return rc;
    }
    buf.resize((size_t)W * ne * 5 * Oa);
    CK(cudaMemcpyAsync(buf.data(), c->hb.orball, sizeof(double) * buf.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int w = 0; w < W; w++)
      for (int el = 0; el < ne; el++) {
        const int e = e0 + el;
        const double *ob = &buf[((size_t)w * ne + el) * 5 * Oa];
        for (int o = 0; o < Oa; o++) {
          if (orb) orb[((size_t)w * Oa + o) * N + e] = ob[o];
          if (dorb)
            for (int k = 0; k < 3; k++) dorb[(((size_t)w * 3 + k) * N + e) * Oa + o] = ob[(1 + k) * Oa + o];
          if (ddorb) ddorb[((size_t)w * N + e) * Oa + o] = ob[4 * Oa + o];
        }
      }
  }
  return CW_OK;
}

int cw_jastrow(cw_ctx *c, double *psij, double *v, double *d2j) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  BIND(c);
  NORD_DISPATCH(launch_jfull, c);
  LCHK("k_jastrow_full");
  const int W = c->W, N = c->h.N;
  CK(cudaStreamSynchronize(c->stream));
  if (psij) CK(cudaMemcpy(psij, c->st.fsumo, sizeof(double) * W, cudaMemcpyDeviceToHost));
  if (d2j) CK(cudaMemcpy(d2j, c->hb.d2o, sizeof(double) * W, cudaMemcpyDeviceToHost));
  if (v) {
    std::vector<double> t((size_t)W * 3 * N);
    CK(cudaMemcpy(t.data(), c->st.fjo, sizeof(double) * t.size(), cudaMemcpyDeviceToHost));
    for (int w = 0; w < W; w++)
      for (int e = 0; e < N; e++)
        for (int k = 0; k < 3; k++) v[((size_t)w * N + e) * 3 + k] = t[((size_t)w * 3 + k) * N + e];
  }
  return CW_OK;
}

int cw_slater(cw_ctx *c, double *slmi, double *det) {
  if (!c || c->W == 0) return fail(c, CW_ERR_STATE, "no walkers");
  BIND(c);
  int rc = run_hpsi(c, 0);
  if (rc) return rc;
  rc = check_status(c);
  if (rc) return rc;
  const int W = c->W, nmax = c->h.nmax;
  if (slmi) CK(cudaMemcpy(slmi, c->st.slmi, sizeof(double) * W * 2 * nmax * nmax, cudaMemcpyDeviceToHost));
  if (det) CK(cudaMemcpy(det, c->st.detiab, sizeof(double) * W * 2, cudaMemcpyDeviceToHost));
  return CW_OK;
}

int cw_fma_peak(int device, int fp64, double *tflops) {
  if (!tflops) return CW_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return CW_ERR_CUDA;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  void *out = nullptr;
  if (cudaMalloc(&out, 64) != cudaSuccess) return CW_ERR_OOM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = nsm * 8, threads = 256, iters = fp64 ? 8192 : 32768;
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0);
    if (fp64) k_fma_peak<double><<<blocks, threads>>>((double *)out, iters, 0.999999, 1e-7);
    else k_fma_peak<float><<<blocks, threads>>>((float *)out, iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = std::min(best, ms);
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return CW_ERR_CUDA;
  const double flops = 2.0 * 8 * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return CW_OK;
}

// --------------------------------------------------------------------------
// host-only helpers
// --------------------------------------------------------------------------
namespace {
struct HRng {
  uint64_t s[4];
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
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
    static const uint64_t J[] = {0x180ec6d33cfd0abaULL, 0xd5a61266f0c9392cULL, 0xa9582618e03fc9aaULL,
                                 0x39abdc4529b1661cULL};
    uint64_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    for (int i = 0; i < 4; i++)
      for (int b = 0; b < 64; b++) {
        if (J[i] & (1ULL << b)) {
          t0 ^= s[0]; t1 ^= s[1]; t2 ^= s[2]; t3 ^= s[3];
        }
        next();
      }
    s[0] = t0; s[1] = t1; s[2] = t2; s[3] = t3;
  }
};
}  // namespace

int cw_rng_states(const int32_t *irn8, int nwalk, uint64_t *out) {
  if (!irn8 || !out || nwalk < 0) return CW_ERR_ARG;
  HRng r;
  std::memcpy(r.s, irn8, 32);
  for (int w = 0; w < nwalk; w++) {
    std::memcpy(out + 4 * (size_t)w, r.s, 32);
    r.jump();
  }
  return CW_OK;
}

int cw_sites(const cw_system_desc *d, int nwalk, uint64_t *rng, double *x) {
  if (!d || !rng || !x || nwalk < 0) return CW_ERR_ARG;
  const int M = d->ncent, N = d->nelec;
  std::vector<int> nsite(M);
  int l = 0;
  for (int i = 0; i < M; i++) {
    nsite[i] = (int)(d->znuc[d->iwctype[i]] + 0.5);
    l += nsite[i];
    if (l > N) {
      nsite[i] -= (l - N);
      l = N;
    }
  }
  if (l < N) nsite[0] += (N - l);
  for (int w = 0; w < nwalk; w++) {
    HRng r;
    std::memcpy(r.s, rng + 4 * (size_t)w, 32);
    double *xw = x + (size_t)w * N * 3;
    l = 0;
    for (int ispin = 1; ispin <= 2; ispin++)
      for (int i = 0; i < M && l < N; i++) {
        const int ju = (nsite[i] + 2 - ispin) / 2;
        for (int j = 1; j <= ju; j++) {
          l++;
          if (l > N) break;
          const double z = d->znuc[d->iwctype[i]];
          double sitsca;
          if (j == 1) sitsca = 1 / z;
          else if (j <= 5) sitsca = 2 / (z - 2);
          else sitsca = 3 / (z - 10);
          for (int ic = 0; ic < 3; ic++) {
            double site = -std::log(r.uniform());
            const double sg = r.uniform() - 0.5;
            site = sg >= 0 ? std::fabs(site) : -std::fabs(site);
            xw[(size_t)(l - 1) * 3 + ic] = sitsca * site + d->cent[3 * i + ic];
          }
        }
      }
    std::memcpy(rng + 4 * (size_t)w, r.s, 32);
  }
  return CW_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free orbital evaluation at caller-given points.
//
// Some callers cannot call cudaMalloc while they run: a Fortran/OpenACC host
// whose device memory is pre-reserved by another allocator or pool, or a
// driver loop that cannot afford cudaMalloc's implicit device-wide
// synchronisation in the middle of a Monte Carlo step.  For them,
// cw_orbitals_noalloc evaluates the orbitals (value, gradient, Laplacian)
// at points the caller already holds on the device and writes them to a
// device buffer the caller provides.  The basis-function values it needs in
// between live in the fixed array below, reserved once when the library's
// device code is loaded on a GPU and kept until the process exits; the call
// itself allocates nothing.
// ===========================================================================
#define CW_NOALLOC_SCRATCH_DOUBLES (2u * 1024u * 1024u) /* 16 MiB per GPU */

static __device__ __align__(256) double cw_noalloc_phi[CW_NOALLOC_SCRATCH_DOUBLES];

namespace {
constexpr int kNoallocMaxDevices = 64;
double *g_noalloc_scratch[kNoallocMaxDevices] = {nullptr};
// the last call's completion on each device: the next call, from any
// context (any stream), waits for it before it writes the shared array
std::mutex g_noalloc_mu;
cudaEvent_t g_noalloc_done[kNoallocMaxDevices] = {nullptr};

// The array's name is only a host-side stand-in for the device symbol: its
// device address is looked up once per device, with that device current.
// The per-device cache below is written without a lock.  Two host threads
// whose first calls on one device race here both store the same address,
// so the race is benign.  The cache assumes the CUDA context of the device
// lives as long as the process: after a cudaDeviceReset the cached address
// is stale.
int noalloc_scratch(cw_ctx *c, double **p) {
  const int dev = c->device;
  if (dev < 0 || dev >= kNoallocMaxDevices) return fail(c, CW_ERR_ARG, "device index out of range");
  if (!g_noalloc_scratch[dev]) {
    void *addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, cw_noalloc_phi);
    if (e != cudaSuccess || !addr)
      return fail(c, CW_ERR_CUDA, "cudaGetSymbolAddress(cw_noalloc_phi) failed: %s", cudaGetErrorString(e));
    g_noalloc_scratch[dev] = (double *)addr;
  }
  *p = g_noalloc_scratch[dev];
  return CW_OK;
}

// basis functions (value, gradient, Laplacian) of npts points, thread per
// (point, centre); rows (p*5 + d) of phi, as k_basis_all writes them.
__global__ void k_basis_points(const __grid_constant__ CSys cs, GSys g, int npts, const double *__restrict__ xyz, double *__restrict__ phi) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int M = cs.M, K = cs.K;
  if (t >= (long)npts * M) return;
  const int ic = (int)(t % M);
  const long p = t / M;
  const double xc[3] = {xyz[3 * p] - cs.cent[3 * ic], xyz[3 * p + 1] - cs.cent[3 * ic + 1],
                        xyz[3 * p + 2] - cs.cent[3 * ic + 2]};
  double *row = phi + (size_t)p * 5 * K;
  basis_centre(cs, g, ic, xc, 2, [&](int a, int d, double v) { row[(size_t)d * K + a] = v; });
}
}  // namespace

extern "C" int cw_orbitals_noalloc(cw_ctx *c, int npts, const double *xyz, double *out) {
  if (!c) return CW_ERR_ARG;
  if (npts <= 0 || !xyz || !out) return fail(c, CW_ERR_ARG, "cw_orbitals_noalloc: bad arguments");
  const CSys &h = c->h;
  const size_t need = (size_t)npts * 5 * h.K;
  if (need > CW_NOALLOC_SCRATCH_DOUBLES)
    return fail(c, CW_ERR_ARG,
                "cw_orbitals_noalloc: %d points x 5 x %d basis functions exceed the fixed scratch of %u doubles "
                "(at most %u points per call for this basis)",
                npts, h.K, CW_NOALLOC_SCRATCH_DOUBLES, (unsigned)(CW_NOALLOC_SCRATCH_DOUBLES / (5u * h.K)));
  BIND(c);
  double *phi = nullptr;
  int rc = noalloc_scratch(c, &phi);
  if (rc) return rc;
  // calls on different contexts run on different streams: order them on the
  // device through the previous call's completion event (outside stream
  // capture; a captured call is ordered by its graph's launches)
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(c->stream, &cap));
  cudaEvent_t &done = g_noalloc_done[c->device];
  if (cap == cudaStreamCaptureStatusNone) {
    if (!done) CK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    CK(cudaStreamWaitEvent(c->stream, done, 0));
  }
  const long nt = (long)npts * h.M;
  k_basis_points<<<(unsigned)((nt + 127) / 128), 128, 0, c->stream>>>(c->h, c->g, npts, xyz, phi);
  LCHK("k_basis_points");
  dgemm(c->stream, npts * 5, h.Oa, h.K, phi, c->g.coefT, out);
  LCHK("dgemm(noalloc)");
  if (cap == cudaStreamCaptureStatusNone) CK(cudaEventRecord(done, c->stream));
  return CW_OK;
}

// ===========================================================================
// Batches of contexts (no CHAMP counterpart): the VMC sweeps of several
// systems as one CUDA graph whose child nodes are the contexts' own captured
// sweep graphs, with no edges between them, so one graph launch advances
// every system by one sweep and the device runs the systems side by side.
// ===========================================================================
struct cw_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, join = nullptr;
  std::vector<cw_ctx *> ctx;
  std::vector<long> gen;       // the contexts' sweep captures the graph was built from
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  float last_ms = 0;
  std::string err;
  // ragged mode: one launch per move stage over every system's walkers
  bool ragged = false;
  cudaEvent_t ev_fork = nullptr;  // ragged capture: start of the bands
  int rag_bn = 0;               // N tile of the grouped FP64 LCAO (timed at build)
  long rag_launches = 0;        // ragged launches per sweep
  long rag_ctx_launches = 0;    // the systems' own hpsi launches per sweep
  int rag_bands = 1;            // bands asked for (cw_batch_set_ragged)
  int rag_nband = 0;            // bands of the built graph
  std::vector<void *> rag_allocs;
  std::vector<cudaStream_t> rag_streams;  // each band's two streams
  std::vector<cudaEvent_t> rag_events;    // each band's fork, join and end events
  std::vector<cudaEvent_t> rag_fork, rag_done;  // per system: start and end of its hpsi branch
};

namespace {
int bfail(cw_batch *b, int code, const char *msg) {
  if (b) b->err = msg;
  return code;
}
}  // namespace

extern "C" int cw_batch_create(cw_batch **out, cw_ctx **ctxs, int n) {
  if (!out || !ctxs || n <= 0) return CW_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < n; i++)
    if (!ctxs[i] || ctxs[i]->device != ctxs[0]->device) return CW_ERR_ARG;
  cw_batch *b = new cw_batch();
  b->device = ctxs[0]->device;
  b->ctx.assign(ctxs, ctxs + n);
  b->gen.assign(n, -1);
  if (cudaSetDevice(b->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess) {
    delete b;
    return CW_ERR_CUDA;
  }
  *out = b;
  return CW_OK;
}

namespace {
void rag_free(cw_batch *b) {
  for (void *p : b->rag_allocs) cudaFree(p);
  b->rag_allocs.clear();
  for (cudaEvent_t e : b->rag_events) cudaEventDestroy(e);
  b->rag_events.clear();
  for (cudaStream_t st : b->rag_streams) cudaStreamDestroy(st);
  b->rag_streams.clear();
  for (cudaEvent_t e : b->rag_fork) cudaEventDestroy(e);
  for (cudaEvent_t e : b->rag_done) cudaEventDestroy(e);
  b->rag_fork.clear();
  b->rag_done.clear();
}
}  // namespace

extern "C" void cw_batch_destroy(cw_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  rag_free(b);
  for (cudaEvent_t e : {b->ev0, b->ev1, b->join, b->ev_fork})
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

extern "C" const char *cw_batch_last_error(const cw_batch *b) { return b ? b->err.c_str() : "null batch"; }

extern "C" float cw_batch_last_ms(const cw_batch *b) { return b ? b->last_ms : 0.0f; }

// ---------------------------------------------------------------------------
// Ragged mode: the moves of every system of the batch in one launch per move
// stage (ragged.cuh).  The systems are sorted by electron count, so the ones
// still moving at step k are a prefix of the slot array; after a system's
// last electron its hpsi (and optimisation sums) run on its own stream,
// forked from the batch's stream inside the same captured graph, while the
// larger systems keep moving.
// ---------------------------------------------------------------------------
namespace {

int nord_class(const cw_ctx *c) {
  const int n = c->h.nordc <= 1 ? 1 : c->h.nordc;
  return n > 7 ? 7 : n;
}

// why the batch's systems cannot advance as one ragged batch ("" if they can)
std::string rag_refusal(const cw_batch *b) {
  if (b->ctx.size() > (size_t)kRagMaxSlots) return "more than " + std::to_string(kRagMaxSlots) + " systems";
  const cw_ctx *c0 = b->ctx[0];
  for (size_t i = 0; i < b->ctx.size(); i++) {
    const cw_ctx *c = b->ctx[i];
    const std::string who = "system " + std::to_string(i) + ": ";
    if (c->W == 0) return who + "no walkers";
    if (c->dmc.on) return who + "a DMC population";
    if (c->md_on) return who + "a multideterminant expansion (one determinant only)";
    if (c->prof) return who + "profiling its launches";
    if (!c->smem_commit) return who + "a spin above 128 electrons";
    if (c->mixed != c0->mixed) return "the systems mix FP64 and mixed precision";
    if (nord_class(c) != nord_class(c0)) return "the systems' e-e-n orders differ";
  }
  return "";
}

template <class T>
T *rag_upload(cw_batch *b, const std::vector<T> &v) {
  void *p = nullptr;
  if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(1, v.size())) != cudaSuccess) return nullptr;
  b->rag_allocs.push_back(p);
  if (!v.empty() && cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return nullptr;
  return static_cast<T *>(p);
}

// blocks of `per` walkers for every slot: (slot, block of the slot); off[i] =
// blocks of the first i slots
std::vector<int2> rag_map(const std::vector<int> &W, int per, std::vector<int> &off) {
  std::vector<int2> m;
  off.assign(W.size() + 1, 0);
  for (size_t i = 0; i < W.size(); i++) {
    const int nb = (W[i] + per - 1) / per;
    for (int k = 0; k < nb; k++) m.push_back(make_int2((int)i, k));
    off[i + 1] = (int)m.size();
  }
  return m;
}

// the FP64 move LCAO of context c runs on the tensor cores when alone (dgemm's test)
bool rag_dmma_ok(const cw_ctx *c) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(c->mb.phi) | reinterpret_cast<uintptr_t>(c->g.coefT) |
                      reinterpret_cast<uintptr_t>(c->mb.orbn);
  return c->h.Oa > 16 && c->h.K % 2 == 0 && c->h.Oa % 2 == 0 && (a & 15) == 0;
}

std::vector<RagTile> rag_tiles(const std::vector<cw_ctx *> &sc, bool mixed, int bn, std::vector<int> &off) {
  std::vector<RagTile> t;
  off.assign(sc.size() + 1, 0);
  for (size_t i = 0; i < sc.size(); i++) {
    const cw_ctx *c = sc[i];
    const int M = 4 * c->W, N = c->h.Oa;
    if (mixed) {
      for (int m0 = 0; m0 < M; m0 += 128) t.push_back(RagTile{(int)i, 2, m0, 0});
    } else if (rag_dmma_ok(c)) {
      for (int n0 = 0; n0 < N; n0 += bn)
        for (int m0 = 0; m0 < M; m0 += kMmaBM) t.push_back(RagTile{(int)i, 0, m0, n0});
    } else {
      for (int n0 = 0; n0 < N; n0 += kRagSimtBN)
        for (int m0 = 0; m0 < M; m0 += kRagSimtBM) t.push_back(RagTile{(int)i, 1, m0, n0});
    }
    off[i + 1] = (int)t.size();
  }
  return t;
}

void rag_lcao(cudaStream_t s, bool mixed, int bn, int grid, size_t smem, const RagSlot *sl, const RagTile *t) {
  if (grid <= 0) return;
  if (mixed) {
    k_lcao_tf32x3_rag<<<grid, 128, smem, s>>>(sl, t);
    return;
  }
  switch (bn) {
    case 32: k_lcao_rag<32><<<grid, 128, smem, s>>>(sl, t); break;
    case 48: k_lcao_rag<48><<<grid, 128, smem, s>>>(sl, t); break;
    case 80: k_lcao_rag<80><<<grid, 128, smem, s>>>(sl, t); break;
    default: k_lcao_rag<64><<<grid, 128, smem, s>>>(sl, t); break;
  }
}

template <int NORD>
cudaError_t rag_jmove_attr(bool mixed, size_t smem) {
  if (mixed)
    return cudaFuncSetAttribute(k_jastrow_move_f32_rag<NORD, kJmF32Partners>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cudaFuncSetAttribute(k_jastrow_move_rag<NORD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}
template <int NORD>
void rag_jmove(cudaStream_t s, bool mixed, int grid, size_t smem, const CSys *csa, const RagSlot *sl, const int2 *map,
               int k) {
  if (mixed) k_jastrow_move_f32_rag<NORD, kJmF32Partners><<<grid, 128, smem, s>>>(csa, sl, map, k);
  else k_jastrow_move_rag<NORD><<<grid, 128, smem, s>>>(csa, sl, map, k);
}
#define RAG_NORD(nc, fn, ...)              \
  switch (nc) {                            \
    case 1: fn<1>(__VA_ARGS__); break;     \
    case 2: fn<2>(__VA_ARGS__); break;     \
    case 3: fn<3>(__VA_ARGS__); break;     \
    case 4: fn<4>(__VA_ARGS__); break;     \
    case 5: fn<5>(__VA_ARGS__); break;     \
    case 6: fn<6>(__VA_ARGS__); break;     \
    default: fn<7>(__VA_ARGS__); break;    \
  }
template <int NORD>
void rag_jmove_attr_v(cudaError_t &e, bool mixed, size_t smem) { e = rag_jmove_attr<NORD>(mixed, smem); }

#define RAG_CK(x, what)                                              \
  do {                                                               \
    cudaError_t e_ = (x);                                            \
    if (e_ != cudaSuccess)                                           \
      return bfail(b, CW_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e_)).c_str()); \
  } while (0)

// Device tables, launch shapes, the LCAO tile (timed) and the captured graph
// of one ragged sweep of every system.  Runs on the batch's stream, which
// already follows every context's queued work.
int rag_build(cw_batch *b) {
  rag_free(b);
  const int n = (int)b->ctx.size();
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->ctx[x]->h.N > b->ctx[y]->h.N; });
  std::vector<cw_ctx *> sc(n);
  std::vector<int> W(n), nel(n);
  for (int i = 0; i < n; i++) {
    sc[i] = b->ctx[order[i]];
    W[i] = sc[i]->W;
    nel[i] = sc[i]->h.N;
  }
  const bool mixed = sc[0]->mixed;
  const int ncls = nord_class(sc[0]);
  // constant blocks, tensor maps, slots
  std::vector<CSys> hcs(n);
  std::vector<CUtensorMap> htm(mixed ? 4 * n : 0);
  for (int i = 0; i < n; i++) {
    hcs[i] = sc[i]->h;
    if (mixed) {
      htm[4 * i + 0] = sc[i]->tm_mv_hi;
      htm[4 * i + 1] = sc[i]->tm_mv_lo;
      htm[4 * i + 2] = sc[i]->tm_b_hi;
      htm[4 * i + 3] = sc[i]->tm_b_lo;
    }
  }
  const CSys *d_cs = rag_upload(b, hcs);
  const CUtensorMap *d_tm = mixed ? rag_upload(b, htm) : nullptr;
  if (!d_cs || (mixed && !d_tm)) return bfail(b, CW_ERR_CUDA, "ragged batch: device tables");
  std::vector<RagSlot> hs(n);
  for (int i = 0; i < n; i++) {
    cw_ctx *c = sc[i];
    RagSlot &r = hs[i];
    r.st = c->st;
    r.mb = c->mb;
    r.g = c->g;
    r.acc_list = c->acc_list;
    r.acc_count = c->acc_count;
    r.W = c->W;
    r.K = c->h.K;
    r.Oa = c->h.Oa;
    r.tm = mixed ? d_tm + 4 * i : nullptr;
    r.np = c->np;
    r.stages = c->umma_st;
    r.err = c->d_err;
  }
  const RagSlot *d_slots = rag_upload(b, hs);
  if (!d_slots) return bfail(b, CW_ERR_CUDA, "ragged batch: slots");
  // launch shapes common to all bands
  int bw = 4;
  int maxM = 0;
  size_t smem_jm = 0, smem_commit = 0, smem_umma = 0;
  for (cw_ctx *c : sc) {
    bw = std::min(bw, c->basis_warps);
    maxM = std::max(maxM, c->h.M);
    smem_jm = std::max(smem_jm, mixed ? c->smem_jmove_f32 : c->smem_jmove);
    smem_commit = std::max(smem_commit, c->smem_commit);
    smem_umma = std::max(smem_umma, c->smem_umma);
  }
  const size_t smem_basis = (size_t)bw * maxM * kCenRec * sizeof(double);
  std::vector<int> offrot;
  std::vector<int> Wrot(n);
  for (int i = 0; i < n; i++) Wrot[i] = sc[i]->h.nloc > 0 ? W[i] : 0;
  const int2 *d_rot = rag_upload(b, rag_map(Wrot, 128, offrot));
  if (!d_rot) return bfail(b, CW_ERR_CUDA, "ragged batch: block maps");
  cudaError_t ea = cudaSuccess;
  RAG_NORD(ncls, rag_jmove_attr_v, ea, mixed, smem_jm);
  RAG_CK(ea, "ragged move Jastrow attributes");
  RAG_CK(cudaFuncSetAttribute(k_basis_move_rag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_basis),
         "ragged basis attributes");
  RAG_CK(cudaFuncSetAttribute(k_commit_rag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_commit),
         "ragged commit attributes");
  int nsm = 0, per = 0;
  RAG_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device), "device attributes");
  RAG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_commit_rag, 128, smem_commit), "commit occupancy");
  const int commit_grid = std::max(1, nsm * std::max(1, per));
  // LCAO tile: the N tile of the tensor-core tiles is timed over the whole
  // batch (every output sums its K slices in the same order whatever the tile)
  size_t smem_lcao = 0;
  if (mixed) {
    smem_lcao = smem_umma;
    RAG_CK(cudaFuncSetAttribute(k_lcao_tf32x3_rag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_lcao),
           "ragged tensor-core LCAO attributes");
    b->rag_bn = 0;
  } else {
    RAG_CK(cudaFuncSetAttribute(k_lcao_rag<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mma_smem(32)), "lcao");
    RAG_CK(cudaFuncSetAttribute(k_lcao_rag<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mma_smem(48)), "lcao");
    RAG_CK(cudaFuncSetAttribute(k_lcao_rag<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mma_smem(64)), "lcao");
    RAG_CK(cudaFuncSetAttribute(k_lcao_rag<80>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mma_smem(80)), "lcao");
    float best = 0;
    for (int bn : kMmaTiles) {
      std::vector<int> o;
      const RagTile *dt = rag_upload(b, rag_tiles(sc, false, bn, o));
      if (!dt) return bfail(b, CW_ERR_CUDA, "ragged batch: LCAO tiles");
      const int grid = o[n];
      rag_lcao(b->stream, false, bn, grid, mma_smem(bn), d_slots, dt);  // warm-up
      RAG_CK(cudaEventRecord(b->ev0, b->stream), "tile timing");
      for (int r = 0; r < 3; r++) rag_lcao(b->stream, false, bn, grid, mma_smem(bn), d_slots, dt);
      RAG_CK(cudaEventRecord(b->ev1, b->stream), "tile timing");
      RAG_CK(cudaEventSynchronize(b->ev1), "tile timing");
      RAG_CK(cudaGetLastError(), "ragged LCAO");
      float ms = 0;
      cudaEventElapsedTime(&ms, b->ev0, b->ev1);
      if (b->rag_bn == 0 || ms < best) {
        best = ms;
        b->rag_bn = bn;
      }
    }
    smem_lcao = mma_smem(b->rag_bn);
  }
  // bands: contiguous runs of the sorted systems with about equal moves per
  // sweep, each its own chain of ragged launches on its own streams
  std::vector<int> cut{0};
  {
    double tot = 0, acc = 0;
    for (int i = 0; i < n; i++) tot += (double)W[i] * nel[i];
    const int want = std::max(1, std::min(b->rag_bands, n));
    for (int i = 0; i < n; i++) {
      acc += (double)W[i] * nel[i];
      if ((int)cut.size() < want && i + 1 < n && acc >= tot * (double)cut.size() / want) cut.push_back(i + 1);
    }
    cut.push_back(n);
  }
  const int nband = (int)cut.size() - 1;
  struct Band {
    int s0, s1;
    std::vector<int> off16, off4, offbw, offt;
    const int2 *g16, *g4, *gbw;
    const RagTile *tiles;
    cudaStream_t main, side;
    cudaEvent_t fork, join, end;
  };
  std::vector<Band> band(nband);
  for (int g = 0; g < nband; g++) {
    Band &B = band[g];
    B.s0 = cut[g];
    B.s1 = cut[g + 1];
    const std::vector<int> Wg(W.begin() + B.s0, W.begin() + B.s1);
    const std::vector<cw_ctx *> scg(sc.begin() + B.s0, sc.begin() + B.s1);
    B.g16 = rag_upload(b, rag_map(Wg, 128 / kMoveGroup, B.off16));
    B.g4 = rag_upload(b, rag_map(Wg, 4, B.off4));
    B.gbw = rag_upload(b, rag_map(Wg, bw, B.offbw));
    B.tiles = rag_upload(b, rag_tiles(scg, mixed, b->rag_bn, B.offt));
    if (!B.g16 || !B.g4 || !B.gbw || !B.tiles) return bfail(b, CW_ERR_CUDA, "ragged batch: band maps");
    B.main = B.side = nullptr;
    B.fork = B.join = B.end = nullptr;
    RAG_CK(cudaStreamCreateWithFlags(&B.main, cudaStreamNonBlocking), "band streams");
    b->rag_streams.push_back(B.main);
    RAG_CK(cudaStreamCreateWithFlags(&B.side, cudaStreamNonBlocking), "band streams");
    b->rag_streams.push_back(B.side);
    for (cudaEvent_t *e : {&B.fork, &B.join, &B.end}) {
      RAG_CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "band events");
      b->rag_events.push_back(*e);
    }
  }
  // events of the systems' hpsi branches
  b->rag_fork.assign(n, nullptr);
  b->rag_done.assign(n, nullptr);
  for (int i = 0; i < n; i++) {
    RAG_CK(cudaEventCreateWithFlags(&b->rag_fork[i], cudaEventDisableTiming), "events");
    RAG_CK(cudaEventCreateWithFlags(&b->rag_done[i], cudaEventDisableTiming), "events");
  }
  // capture one sweep: rotqua of every system, then the bands side by side
  cudaStream_t s = b->stream;
  RAG_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "ragged capture");
  long nl = 0, nc = 0;
  int rc = CW_OK;
  std::string why;
  int forked = 0;
  if (offrot[n] > 0) {
    k_rotqua_rag<<<offrot[n], 128, 0, s>>>(d_cs, d_slots, d_rot);
    nl++;
  }
  cudaEventRecord(b->ev_fork, s);
  for (int g = 0; g < nband && rc == CW_OK; g++) {
    Band &B = band[g];
    const CSys *cs = d_cs + B.s0;
    const RagSlot *sl = d_slots + B.s0;
    const int nbs = B.s1 - B.s0;
    const int *ne = nel.data() + B.s0;
    cudaStream_t bm = B.main;
    if (cudaStreamWaitEvent(bm, b->ev_fork, 0) != cudaSuccess) {
      rc = CW_ERR_CUDA;
      why = "ragged capture: band fork";
      break;
    }
    int A = nbs;
    for (int k = 0; k < ne[0] && rc == CW_OK; k++) {
      while (A > 0 && ne[A - 1] <= k) A--;
      k_propose_rag<<<B.off16[A], 128, 0, bm>>>(cs, sl, B.g16, k);
      // the move Jastrow beside the basis + LCAO (both need only the proposal)
      cudaEventRecord(B.fork, bm);
      cudaStreamWaitEvent(B.side, B.fork, 0);
      RAG_NORD(ncls, rag_jmove, bm, mixed, B.off4[A], smem_jm, cs, sl, B.g4, k);
      k_basis_move_rag<<<B.offbw[A], 32 * bw, smem_basis, B.side>>>(cs, sl, B.gbw);
      rag_lcao(B.side, mixed, b->rag_bn, B.offt[A], smem_lcao, sl, B.tiles);
      cudaEventRecord(B.join, B.side);
      cudaStreamWaitEvent(bm, B.join, 0);
      k_decide_rag<<<B.off16[A], 128, 0, bm>>>(cs, sl, B.g16, k);
      k_commit_rag<<<commit_grid, 128, smem_commit, bm>>>(cs, sl, A, k);
      nl += 6;
      const cudaError_t le = cudaGetLastError();
      if (le != cudaSuccess) {
        rc = CW_ERR_CUDA;
        why = std::string("ragged launch: ") + cudaGetErrorString(le);
        break;
      }
      // the band's systems whose last electron just moved: hpsi on their own streams
      for (int j = A - 1; j >= 0 && ne[j] == k + 1; j--) {
        const int i = B.s0 + j;
        cw_ctx *c = sc[i];
        if (cudaEventRecord(b->rag_fork[i], bm) != cudaSuccess ||
            cudaStreamWaitEvent(c->stream, b->rag_fork[i], 0) != cudaSuccess) {
          rc = CW_ERR_CUDA;
          why = "ragged capture: fork";
          break;
        }
        forked++;
        const long l0 = c->launches;
        rc = run_hpsi(c, 1);
        if (rc == CW_OK && c->opt_np > 0) rc = opt_accum(c);
        nc += c->launches - l0;
        c->launches = l0;
        cudaEventRecord(b->rag_done[i], c->stream);
        if (rc) {
          why = "system " + std::to_string(order[i]) + ": " + c->err;
          break;
        }
      }
    }
    cudaEventRecord(B.end, bm);
  }
  // join every band and every system's hpsi branch
  for (int g = 0; g < nband; g++)
    if (band[g].end) cudaStreamWaitEvent(s, band[g].end, 0);
  for (int i = 0; i < n; i++) cudaStreamWaitEvent(s, b->rag_done[i], 0);
  cudaGraph_t gph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(s, &gph);
  if (rc != CW_OK || ee != cudaSuccess) {
    if (gph) cudaGraphDestroy(gph);
    cudaGetLastError();
    if (rc == CW_OK) {
      rc = CW_ERR_CUDA;
      why = std::string("ragged capture: ") + cudaGetErrorString(ee);
    }
    return bfail(b, rc, why.c_str());
  }
  if (forked != n) {
    cudaGraphDestroy(gph);
    return bfail(b, CW_ERR_STATE, "ragged capture: a system's hpsi was not scheduled");
  }
  b->rag_nband = nband;
  b->graph = gph;
  b->rag_launches = nl;
  b->rag_ctx_launches = nc;
  RAG_CK(cudaGraphInstantiate(&b->exec, b->graph, 0), "ragged graph instantiate");
  return CW_OK;
}

}  // namespace

// Ragged mode off (bands = 0) or on with that many bands of systems (each
// band its own chain of launches); refused (with the reason) when a system
// cannot join
extern "C" int cw_batch_set_ragged(cw_batch *b, int bands) {
  if (!b || bands < 0) return CW_ERR_ARG;
  if (bands) {
    const std::string why = rag_refusal(b);
    if (!why.empty()) return bfail(b, CW_ERR_UNSUPPORTED, ("ragged batch: " + why).c_str());
  }
  if (b->ragged != (bands != 0) || (bands && bands != b->rag_bands)) {
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, CW_ERR_CUDA, "cudaSetDevice failed");
    cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->ragged = bands != 0;
    if (bands) b->rag_bands = bands;
  }
  return CW_OK;
}

// [bands asked for (0: off), LCAO N tile, ragged launches per sweep, the
//  systems' own hpsi launches per sweep, bands of the built graph]
extern "C" int cw_batch_info(const cw_batch *b, int64_t *info) {
  if (!b || !info) return CW_ERR_ARG;
  info[0] = b->ragged ? b->rag_bands : 0;
  info[1] = b->rag_bn;
  info[2] = b->rag_launches;
  info[3] = b->rag_ctx_launches;
  info[4] = b->rag_nband;
  return CW_OK;
}

// nstep sweeps of every context of the batch: each context's sweep graph is
// (re)captured where needed, the batch graph rebuilt when any of them
// changed, then launched nstep times on the batch's stream, ordered after
// each context's queued work and before its next.  A context that reports a
// failure status names itself in the batch's error (its own cw_last_error
// has the detail).  In ragged mode the batch graph is the ragged sweep.
extern "C" int cw_batch_vmc_steps(cw_batch *b, int nstep) {
  if (!b || nstep < 0) return CW_ERR_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, CW_ERR_CUDA, "cudaSetDevice failed");
  bool stale = !b->exec;
  for (size_t i = 0; i < b->ctx.size(); i++) {
    cw_ctx *c = b->ctx[i];
    if (c->W == 0) return bfail(b, CW_ERR_STATE, "a context of the batch has no walkers");
    if (c->prof) return bfail(b, CW_ERR_STATE, "a context of the batch is profiling its launches");
    if (int rc = ensure_sweep_graph(c)) return bfail(b, rc, "a context's sweep capture failed");
    if (b->gen[i] != c->sweep_gen) stale = true;
  }
  if (b->ragged) {
    const std::string why = rag_refusal(b);
    if (!why.empty()) return bfail(b, CW_ERR_UNSUPPORTED, ("ragged batch: " + why).c_str());
  }
  // after every context's queued work ...
  for (cw_ctx *c : b->ctx) {
    if (cudaEventRecord(b->join, c->stream) != cudaSuccess || cudaStreamWaitEvent(b->stream, b->join, 0) != cudaSuccess)
      return bfail(b, CW_ERR_CUDA, "ordering the batch after its contexts failed");
  }
  if (stale) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    if (b->ragged) {
      if (int rc = rag_build(b)) return rc;
    } else {
      if (cudaGraphCreate(&b->graph, 0) != cudaSuccess) return bfail(b, CW_ERR_CUDA, "cudaGraphCreate failed");
      for (size_t i = 0; i < b->ctx.size(); i++) {
        cudaGraphNode_t node;
        if (cudaGraphAddChildGraphNode(&node, b->graph, nullptr, 0, b->ctx[i]->sweep_graph) != cudaSuccess)
          return bfail(b, CW_ERR_CUDA, "cudaGraphAddChildGraphNode failed");
      }
      if (cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess)
        return bfail(b, CW_ERR_CUDA, "cudaGraphInstantiate of the batch failed");
    }
    for (size_t i = 0; i < b->ctx.size(); i++) b->gen[i] = b->ctx[i]->sweep_gen;
  }
  cudaEventRecord(b->ev0, b->stream);
  for (int s = 0; s < nstep; s++)
    if (cudaGraphLaunch(b->exec, b->stream) != cudaSuccess) return bfail(b, CW_ERR_CUDA, "batch graph launch failed");
  cudaEventRecord(b->ev1, b->stream);
  // ... and before each context's next work
  cudaEventRecord(b->join, b->stream);
  for (cw_ctx *c : b->ctx)
    if (cudaStreamWaitEvent(c->stream, b->join, 0) != cudaSuccess)
      return bfail(b, CW_ERR_CUDA, "ordering the contexts after the batch failed");
  if (cudaEventSynchronize(b->ev1) != cudaSuccess) return bfail(b, CW_ERR_CUDA, "batch sweeps failed");
  cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
  for (size_t i = 0; i < b->ctx.size(); i++) {
    cw_ctx *c = b->ctx[i];
    c->passes += nstep;
    c->launches = b->ragged ? 0 : (long)nstep * c->sweep_launches;
    if (c->opt_np > 0) c->sr_w += (double)c->W * nstep;
    if (int rc = check_status(c)) {
      b->err = "context " + std::to_string(i) + ": " + c->err;
      return rc;
    }
  }
  return CW_OK;
}

// ===========================================================================
// Diffusion Monte Carlo: one population per context (CHAMP's per-rank dmc
// arrays).  Walker slots 0..mwalk-1 live in the walker arrays allocated for
// mwalk; kernels run over the nwalk active ones.
// ===========================================================================
namespace {

// splitj (dmc/splitj.f90:3) on the host weights and ages: pairs small
// weights, splits weights >= 2 and compacts the population.  Appends the
// (source, destination) slot copies in CHAMP's order; returns the new nwalk
// or -1 when mwalk would be exceeded.
int splitj_host(DmcHost &d, int nwalk, std::vector<std::pair<int, int>> &copies) {
  double *wt = d.h_wt;
  int *iage = d.h_iage;
  std::vector<int> iwundr;
  int ipair = 0, iw2 = 0;
  for (int iw = 0; iw < nwalk; iw++) {
    if (wt[iw] < 0.5) {
      if (wt[iw] == 0.0) {
        d.nbrnch++;
        iwundr.push_back(iw);
      } else if (ipair == 0) {
        ipair = 1;
        iw2 = iw;
      } else {
        d.nbrnch++;
        ipair = 0;
        const double wttot = wt[iw] + wt[iw2];
        if (d.pop.uniform() > (wt[iw] / wttot)) {
          wt[iw2] = wttot;
          iwundr.push_back(iw);
        } else {
          wt[iw] = wttot;
          iwundr.push_back(iw2);
        }
      }
    }
  }
  int nwalk2 = nwalk;
  for (int iw = 0; iw < nwalk; iw++) {
    if (wt[iw] >= 2.0) {
      d.nbrnch++;
      int dst;
      if (!iwundr.empty()) {
        dst = iwundr.back();
        iwundr.pop_back();
      } else {
        dst = nwalk2++;
        if (nwalk2 > d.mwalk) return -1;
      }
      wt[iw] = wt[iw] * 0.5;
      wt[dst] = wt[iw];
      iage[dst] = iage[iw];
      copies.emplace_back(iw, dst);
    }
  }
  for (int j = (int)iwundr.size() - 1; j >= 0; j--) {
    const int dst = iwundr[j], src = nwalk2 - 1;
    nwalk2--;
    wt[dst] = wt[src];
    iage[dst] = iage[src];
    copies.emplace_back(src, dst);
  }
  return nwalk2;
}

void add_field(WalkerRec &r, double *p, long len) {
  r.ptr[r.nfield] = p;
  r.len[r.nfield] = len;
  r.nfield++;
}

}  // namespace

int dmc_alloc(cw_ctx *c, int mwalk);

extern "C" int cw_dmc_init(cw_ctx *c, int nwalk, int mwalk, const double *x, const uint64_t *rng,
                           const uint64_t *pop_rng, double tau, double etrial, int nfprod) {
  if (!c || nwalk <= 0 || mwalk < nwalk || !x || !rng || !pop_rng || !(tau > 0) || nfprod < 1)
    return fail(c, CW_ERR_ARG, "cw_dmc_init: bad arguments");
  // several states: dmc_ps propagates and estimates state 1 alone (psidn(1),
  // enew(1)); the other CI vectors ride along unused.  Sampling a guiding
  // function is a VMC feature.
  if (c->h.nstates > 1 && c->h.iguiding > 0)
    return fail(c, CW_ERR_UNSUPPORTED, "cw_dmc_init: a guiding function (iguiding > 0) is a VMC feature");
  BIND(c);
  int rc = dmc_alloc(c, mwalk);
  if (rc) return rc;
  const CSys &h = c->h;
  const int N = h.N;
  DmcHost &d = c->dmc;
  DmcBuf &b = d.db;
  // active population
  c->W = nwalk;
  c->st.W = nwalk;
  std::vector<double> xt((size_t)nwalk * 3 * N);
  for (int w = 0; w < nwalk; w++)
    for (int e = 0; e < N; e++)
      for (int k = 0; k < 3; k++) xt[((size_t)w * 3 + k) * N + e] = x[((size_t)w * N + e) * 3 + k];
  CK(cudaMemcpyAsync(c->st.x, xt.data(), sizeof(double) * xt.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->st.rng, rng, sizeof(uint64_t) * 4 * mwalk, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->st.status, 0, sizeof(int) * mwalk, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // init: hpsi with the unrotated grid, then drift and fratio of every walker
  rc = zerest(c);
  if (rc) return rc;
  d.tau = tau;
  d.etrial = etrial;
  d.mwalk = mwalk;
  d.nconf = nwalk;
  d.nfprod = nfprod;
  d.pop.load(pop_rng);
  d.ff.assign(nfprod, 1.0);
  d.eigv = 1.0;
  d.eest = etrial;
  d.fprod = 1.0;
  d.wdsumo = nwalk;
  const DmcScalars sc{tau, etrial, d.eest, 1.0, 1.0};
  if (c->md_on) {
    k_md_drift_all<<<(unsigned)(((long)nwalk * N + 3) / 4), 128, 0, c->stream>>>(c->h, c->st, c->md, c->g, c->md_vall);
    LCHK("k_md_drift_all");
  }
  k_dmc_weights<<<(nwalk + 3) / 4, 128, 0, c->stream>>>(c->h, c->st, b, sc, 0, c->md_vall);
  LCHK("k_dmc_weights(init)");
  for (int w = 0; w < nwalk; w++) d.h_wt[w] = 1.0;
  CK(cudaMemcpyAsync(b.wt, d.h_wt, sizeof(double) * nwalk, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(b.iage, 0, sizeof(int) * mwalk, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  d.on = true;
  return CW_OK;
}

// Walker storage for mwalk slots plus the DMC arrays, pinned host buffers
// and the walker record of splitj copies.
int dmc_alloc(cw_ctx *c, int mwalk) {
  int rc = alloc_walkers(c, mwalk);
  if (rc) return rc;
  const CSys &h = c->h;
  const int N = h.N, nmax = h.nmax;
  DmcHost &d = c->dmc;
  DmcBuf &b = d.db;
  d.mwalk = mwalk;
  DALLOC(d.allocs, b.vold, (size_t)mwalk * 3 * N);
  DALLOC(d.allocs, b.wt, mwalk);
  DALLOC(d.allocs, b.fratio, mwalk);
  DALLOC(d.allocs, b.iage, mwalk);
  DALLOC(d.allocs, b.eprev, mwalk);
  DALLOC(d.allocs, b.acc, (size_t)mwalk * DA_NA);
  DALLOC(d.allocs, b.copy_src, mwalk);
  DALLOC(d.allocs, b.copy_dst, mwalk);
  CK(cudaMallocHost((void **)&d.h_acc, sizeof(double) * mwalk * DA_NA));
  CK(cudaMallocHost((void **)&d.h_wt, sizeof(double) * mwalk));
  CK(cudaMallocHost((void **)&d.h_iage, sizeof(int) * mwalk));
  CK(cudaMallocHost((void **)&d.h_copy, sizeof(int) * 2 * mwalk));
  // walker record of splitj copies
  WalkerRec &r = d.rec;
  r.nfield = 0;
  add_field(r, c->st.x, 3L * N);
  add_field(r, c->st.psido, 1);
  add_field(r, c->st.psijo, 1);
  add_field(r, c->st.psi2o, 1);
  add_field(r, c->st.eold, 1);
  add_field(r, c->st.ekino, 1);
  add_field(r, c->st.slmi, 2L * nmax * nmax);
  add_field(r, c->st.detiab, 2);
  add_field(r, c->st.orbs, (long)N * nmax);
  add_field(r, c->st.dorbs, 3L * N * nmax);
  add_field(r, c->st.fso, (long)N * N);
  add_field(r, c->st.fijo, 3L * N * N);
  add_field(r, c->st.fjo, 3L * N);
  add_field(r, c->st.fsumo, 1);
  add_field(r, c->st.enm, 2L * h.M * N);
  // 2MN floats per walker = MN doubles: the copy kernel moves doubles
  if (c->st.enmf) add_field(r, reinterpret_cast<double *>(c->st.enmf), (long)h.M * N);
  if (c->md_on) {
    add_field(r, c->md.aa, 2L * nmax * h.Oa);
    add_field(r, c->md.dd, 2L * c->mdt.numax);
    add_field(r, c->md.S, 1);
    add_field(r, c->md.dorbA, 3L * N * h.Oa);
  }
  add_field(r, b.vold, 3L * N);
  add_field(r, b.fratio, 1);
  return CW_OK;
}

extern "C" int cw_dmc_steps(cw_ctx *c, int nstep) {
  if (!c || !c->dmc.on) return fail(c, CW_ERR_STATE, "cw_dmc_steps: no DMC population (cw_dmc_init)");
  BIND(c);
  const CSys &h = c->h;
  DmcHost &d = c->dmc;
  DmcBuf &b = d.db;
  c->launches = 0;
  double total_ms = 0;
  std::vector<std::pair<int, int>> copies;
  std::vector<int> origin(d.mwalk), is_src(d.mwalk);
  for (int s = 0; s < nstep; s++) {
    const int W = c->W;
    CK(cudaEventRecord(c->ev0, c->stream));
    d.ipass++;
    if (h.nloc > 0) {
      double f[9];
      rotqua_frame(d.pop, f);
      QuadRot q;
      for (int iq = 0; iq < h.nquad; iq++) {
        q.x[iq] = h.xq0[iq] * f[0] + h.yq0[iq] * f[3] + h.zq0[iq] * f[6];
        q.y[iq] = h.xq0[iq] * f[1] + h.yq0[iq] * f[4] + h.zq0[iq] * f[7];
        q.z[iq] = h.xq0[iq] * f[2] + h.yq0[iq] * f[5] + h.zq0[iq] * f[8];
      }
      stage_begin(c, CW_ST_ROTQUA);
      k_set_quad<<<(W + 127) / 128, 128, 0, c->stream>>>(c->h, c->st, q);
      stage_end(c);
      LCHK("k_set_quad");
    }
    // population control factor (dmc_ps :148-160)
    const int ipmod = (int)(d.ipass % d.nfprod);
    const double ginv = std::min(1.0, d.tau);
    const double ffn = d.eigv * std::pow(d.wdsumo / d.nconf, ginv);
    const double ffi = 1.0 / ffn;
    d.fprod = d.fprod * ffn / d.ff[ipmod];
    d.ff[ipmod] = ffn;
    const DmcScalars sc{d.tau, d.etrial, d.eest, ffi, d.fprod};
    CK(cudaMemsetAsync(b.acc, 0, sizeof(double) * W * DA_NA, c->stream));
    CK(cudaMemcpyAsync(b.eprev, c->st.eold, sizeof(double) * W, cudaMemcpyDeviceToDevice, c->stream));
    for (int i = 0; i < h.N; i++) {
      if (int rc = md_before_propose(c, i)) return rc;
      stage_begin(c, CW_ST_PROPOSE);
      k_dmc_propose<<<(W + 63) / 64, 64, 0, c->stream>>>(c->h, c->st, c->mb, b, sc, i,
                                                        c->smem_commit ? c->acc_count : nullptr);
      stage_end(c);
      LCHK("k_dmc_propose");
      // move Jastrow beside basis + LCAO + multideterminant ratios (all need
      // only the proposal), joined before the decision; in order when profiling
      const bool fork = !c->prof;
      if (fork) {
        CK(cudaEventRecord(c->ev_fork, c->stream));
        CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
      }
      stage_begin(c, CW_ST_JASTROW_MOVE);
      NORD_DISPATCH(launch_jmove, c, i);
      stage_end(c);
      LCHK("k_jastrow_move");
      cudaStream_t bs = fork ? c->side : c->stream;
      const int bw = c->basis_warps;
      stage_begin(c, CW_ST_BASIS_MOVE);
      k_basis_move<<<(unsigned)((W + bw - 1) / bw), 32 * bw, c->smem_basis, bs>>>(c->h, c->st, c->mb, c->g);
      stage_end(c);
      LCHK("k_basis_move");
      stage_begin(c, CW_ST_LCAO_MOVE);
      {
        int rc = lcao(c, true, W * 4, c->mb.phi, c->mb.orbn, bs);
        stage_end(c);
        if (rc) return rc;
      }
      if (int rc = md_after_lcao(c, i, bs)) return rc;
      if (fork) {
        CK(cudaEventRecord(c->ev_join, c->side));
        CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
      }
      stage_begin(c, CW_ST_ACCEPT);
      k_dmc_decide<<<(W + 63) / 64, 64, 0, c->stream>>>(c->h, c->st, c->mb, c->g, b, sc, i,
                                                       c->smem_commit ? c->acc_list : nullptr, c->acc_count);
      stage_end(c);
      LCHK("k_dmc_decide");
      stage_begin(c, CW_ST_COMMIT);
      launch_commit(c, i, true);
      stage_end(c);
      LCHK("k_commit");
      if (int rc = md_after_commit(c, i)) return rc;
    }
    if (d.icasula == -1) {
      CK(cudaMemsetAsync(c->hb.tvpsp, 0, sizeof(double) * (size_t)W * h.N * h.nquad * h.M, c->stream));
      if (c->hb.tvtrj) CK(cudaMemsetAsync(c->hb.tvtrj, 0, sizeof(double) * (size_t)W * h.N * h.nquad * h.M, c->stream));
    }
    int rc = run_hpsi(c, 0);
    if (rc) return rc;
    if (d.icasula == -1 && c->md_on) {
      // the excitations' part of the T-move elements (dmc_ps :473), from hpsi's Y
      stage_begin(c, CW_ST_TMOVE);
      k_md_tmove<<<W, 128, c->smem_md_tmove, c->stream>>>(c->h, c->st, c->md, c->hb, c->g);
      stage_end(c);
      LCHK("k_md_tmove");
    }
    if (c->md_on) {
      stage_begin(c, CW_ST_MDET);
      k_md_drift_all<<<(unsigned)(((long)W * h.N + 3) / 4), 128, 0, c->stream>>>(c->h, c->st, c->md, c->g, c->md_vall);
      stage_end(c);
      LCHK("k_md_drift_all");
    }
    stage_begin(c, CW_ST_DMC_WEIGHTS);
    k_dmc_weights<<<(W + 3) / 4, 128, 0, c->stream>>>(c->h, c->st, b, sc, 1, c->md_vall);
    stage_end(c);
    LCHK("k_dmc_weights");
    if (d.icasula == -1) {
      // T-moves (dmc_ps :701-735): choice, then the forced move of each walker's electron
      stage_begin(c, CW_ST_TMOVE);
      k_tmove_select<<<(W + 3) / 4, 128, 0, c->stream>>>(c->h, c->st, c->mb, c->hb.tvpsp, sc);
      stage_end(c);
      LCHK("k_tmove_select");
      stage_begin(c, CW_ST_JASTROW_MOVE);
      NORD_DISPATCH(launch_jmove, c, -1);
      stage_end(c);
      LCHK("k_jastrow_move(tmove)");
      const int bw = c->basis_warps;
      stage_begin(c, CW_ST_BASIS_MOVE);
      k_basis_move<<<(unsigned)((W + bw - 1) / bw), 32 * bw, c->smem_basis, c->stream>>>(c->h, c->st, c->mb, c->g);
      stage_end(c);
      LCHK("k_basis_move(tmove)");
      stage_begin(c, CW_ST_LCAO_MOVE);
      {
        int rc2 = lcao(c, true, W * 4, c->mb.phi, c->mb.orbn);
        stage_end(c);
        if (rc2) return rc2;
      }
      if (c->md_on) {
        // psi_D of the expansion at each walker's point: G of the moved spin
        // (as at the start of its phase), then multideterminante
        stage_begin(c, CW_ST_MDET);
        k_md_phase<<<W, 128, c->smem_md_phase, c->stream>>>(c->h, c->st, c->md, c->mdt, -1, c->mb.ms);
        k_md_move<<<W, 128, c->smem_md_move, c->stream>>>(c->h, c->st, c->mb, c->md, c->mdt, c->g, -1);
        stage_end(c);
        LCHK("k_md_move(tmove)");
      }
      stage_begin(c, CW_ST_TMOVE);
      k_tmove_accept<<<(W + 63) / 64, 64, 0, c->stream>>>(c->h, c->st, c->mb, c->g, b, c->md_on ? c->md.psidn : nullptr);
      stage_end(c);
      LCHK("k_tmove_accept");
      stage_begin(c, CW_ST_COMMIT);
      launch_commit(c, -1);
      stage_end(c);
      LCHK("k_commit(tmove)");
      if (c->md_on) {
        stage_begin(c, CW_ST_MDET);
        k_md_commit<<<W, 128, 0, c->stream>>>(c->h, c->st, c->mb, c->md, c->mdt, -1);
        stage_end(c);
        LCHK("k_md_commit(tmove)");
      }
    }
    CK(cudaMemcpyAsync(d.h_acc, b.acc, sizeof(double) * W * DA_NA, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(d.h_wt, b.wt, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(d.h_iage, b.iage, sizeof(int) * W, cudaMemcpyDeviceToHost, c->stream));
    rc = check_status(c);  // synchronises the stream
    if (rc) return rc;
    // the step's sums, in walker order
    for (int w = 0; w < W; w++) {
      const double *a = d.h_acc + (size_t)w * DA_NA;
      d.wsum1 += a[DA_WSUM1];
      d.esum1 += a[DA_ESUM1];
      d.pesum += a[DA_PESUM];
      d.tpbsum += a[DA_TPBSUM];
      d.tausum += a[DA_TAUSUM];
      d.acc += a[DA_ACC];
      d.trymove += a[DA_TRY];
      d.nacc += (long)a[DA_NACC];
      d.nodecr += (long)a[DA_NODECR];
      d.nmove_casula += (long)a[DA_TMOVE];
    }
    const double wgsum1 = d.wsum1 * d.fprod, egsum1 = d.esum1 * d.fprod;
    // splitj: weights on the host, walker copies on the device
    copies.clear();
    const int nwalk2 = splitj_host(d, W, copies);
    if (nwalk2 < 0) return fail(c, CW_ERR_STATE, "SPLITJ: MWALK exceeded (mwalk=%d)", d.mwalk);
    for (int k = 0; k < d.mwalk; k++) {
      origin[k] = k;
      is_src[k] = 0;
    }
    for (auto &cp : copies) origin[cp.second] = origin[cp.first];
    int ncopy = 0;
    for (int k = 0; k < nwalk2; k++)
      if (origin[k] != k) {
        d.h_copy[ncopy] = origin[k];
        d.h_copy[d.mwalk + ncopy] = k;
        is_src[origin[k]] = 1;
        ncopy++;
      }
    for (int k = 0; k < ncopy; k++)
      if (is_src[d.h_copy[d.mwalk + k]])
        return fail(c, CW_ERR_STATE, "splitj: slot %d is both a copy source and a destination", d.h_copy[d.mwalk + k]);
    CK(cudaMemcpyAsync(b.wt, d.h_wt, sizeof(double) * nwalk2, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(b.iage, d.h_iage, sizeof(int) * nwalk2, cudaMemcpyHostToDevice, c->stream));
    if (ncopy > 0) {
      CK(cudaMemcpyAsync(b.copy_src, d.h_copy, sizeof(int) * ncopy, cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemcpyAsync(b.copy_dst, d.h_copy + d.mwalk, sizeof(int) * ncopy, cudaMemcpyHostToDevice, c->stream));
      stage_begin(c, CW_ST_SPLITJ);
      k_walker_copy<<<ncopy, 256, 0, c->stream>>>(d.rec, b, ncopy);
      stage_end(c);
      LCHK("k_walker_copy");
    }
    c->W = nwalk2;
    c->st.W = nwalk2;
    // acues1 (dmc/acues1.f90:3)
    d.wgsum += wgsum1;
    d.egsum += egsum1;
    d.eest = (d.egcum + d.egsum) / (d.wgcum + d.wgsum);
    d.eigv = std::exp((d.etrial - d.eest) * (d.taucum + d.tausum) / (d.wgcum + d.wgsum));
    d.wdsumo = d.wsum1;
    d.wsum1 = 0;
    d.esum1 = 0;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    total_ms += ms;
    if (c->prof) stage_collect(c);
  }
  c->last_ms = total_ms;
  c->passes += nstep;
  return CW_OK;
}

extern "C" int cw_dmc_end_block(cw_ctx *c) {
  if (!c || !c->dmc.on) return fail(c, CW_ERR_STATE, "cw_dmc_end_block: no DMC population");
  DmcHost &d = c->dmc;
  // acuest (dmc/acuest.f90:112-255): block sums into the cumulative ones
  const double egnow = d.egsum / d.wgsum;
  d.egcm2 += d.egsum * egnow;
  d.wgcm2 += d.wgsum * d.wgsum;
  d.egcum += d.egsum;
  d.wgcum += d.wgsum;
  d.taucum += d.tausum;
  d.pecum += d.pesum;
  d.tpbcum += d.tpbsum;
  d.egsum = d.wgsum = d.tausum = d.pesum = d.tpbsum = 0;
  d.iblk++;
  return CW_OK;
}

extern "C" int cw_dmc_results(cw_ctx *c, double *out) {
  if (!c || !out || !c->dmc.on) return fail(c, CW_ERR_STATE, "cw_dmc_results: no DMC population");
  const DmcHost &d = c->dmc;
  if (d.iblk == 0) return fail(c, CW_ERR_STATE, "cw_dmc_results: no completed blocks");
  // finwrt (dmc/finwrt.f90): error with the effective number of blocks
  const double egave = d.egcum / d.wgcum;
  const double rn = d.wgcum * d.wgcum / d.wgcm2;
  const double err = std::sqrt(std::max((d.egcm2 / d.wgcum - egave * egave) / (rn - 1), 0.0));
  out[0] = egave;
  out[1] = d.iblk > 1 ? err : 0.0;
  out[2] = c->W;
  out[3] = d.eest;
  out[4] = d.acc / std::max(d.trymove, 1.0);
  out[5] = d.taucum / d.wgcum;
  out[6] = d.pecum / d.wgcum;
  out[7] = d.tpbcum / d.wgcum;
  out[8] = (double)d.iblk;
  out[9] = d.fprod;
  out[10] = d.eigv;
  out[11] = d.wdsumo;
  return CW_OK;
}

extern "C" int cw_dmc_walkers(cw_ctx *c, int *nwalk, double *x, double *wt, double *eold, uint64_t *rng) {
  if (!c || !c->dmc.on) return fail(c, CW_ERR_STATE, "cw_dmc_walkers: no DMC population");
  const int W = c->W;
  if (nwalk) *nwalk = W;
  int rc = cw_get_walkers(c, x, rng);
  if (rc) return rc;
  if (wt) CK(cudaMemcpy(wt, c->dmc.db.wt, sizeof(double) * W, cudaMemcpyDeviceToHost));
  if (eold) CK(cudaMemcpy(eold, c->st.eold, sizeof(double) * W, cudaMemcpyDeviceToHost));
  return CW_OK;
}

// ===========================================================================
// Checkpoint / restart of the walker population and the accumulators: the
// role of CHAMP's dumper / startr (vmc/dumper.f90:51-106, dmc/dumper.f90:3,
// dmc/restart.f90:3).  The buffer holds what the Markov chain needs to
// continue — configurations, random streams, the rotated quadrature, the
// walkers' block sums and the global accumulators (for DMC: population,
// weights, ages, fratio, the population stream and the branching scalars);
// every derived table is rebuilt by hpsi on restore, so a restored run
// continues exactly as the uninterrupted one.
// ===========================================================================
namespace {

const char kCkMagic[8] = {'C', 'W', 'C', 'K', 'P', 'T', '0', '1'};

struct CkWriter {
  std::vector<uint8_t> b;
  template <typename T>
  void put(const T &v) {
    const uint8_t *p = reinterpret_cast<const uint8_t *>(&v);
    b.insert(b.end(), p, p + sizeof(T));
  }
  template <typename T>
  void put(const T *v, size_t n) {
    const uint8_t *p = reinterpret_cast<const uint8_t *>(v);
    b.insert(b.end(), p, p + n * sizeof(T));
  }
};
struct CkReader {
  const uint8_t *p;
  size_t n, off = 0;
  bool ok = true;
  template <typename T>
  T get() {
    T v{};
    if (off + sizeof(T) > n) { ok = false; return v; }
    std::memcpy(&v, p + off, sizeof(T));
    off += sizeof(T);
    return v;
  }
  template <typename T>
  void get(T *v, size_t cnt) {
    if (off + cnt * sizeof(T) > n) { ok = false; return; }
    std::memcpy(v, p + off, cnt * sizeof(T));
    off += cnt * sizeof(T);
  }
};

template <typename T>
int d2h(cw_ctx *c, std::vector<T> &v, const T *src, size_t n) {
  v.resize(n);
  CK(cudaMemcpyAsync(v.data(), src, sizeof(T) * n, cudaMemcpyDeviceToHost, c->stream));
  return CW_OK;
}

int ck_serialize(cw_ctx *c, std::vector<uint8_t> &out) {
  if (c->W == 0) return fail(c, CW_ERR_STATE, "checkpoint: no walkers");
  BIND(c);
  const CSys &h = c->h;
  const int W = c->W, N = h.N, NQ = std::max(h.nquad, 0);
  const bool dmc = c->dmc.on;
  const int slots = dmc ? c->dmc.mwalk : W;
  CkWriter o;
  o.put(kCkMagic, 8);
  const int64_t hdr[12] = {1, dmc ? 1 : 0, N, h.nup, h.K, h.Oa, h.M, h.ndet, NQ, W, slots, c->precision};
  o.put(hdr, 12);
  std::vector<double> x, xq, sums;
  std::vector<uint64_t> rng;
  int rc = d2h(c, x, c->st.x, (size_t)W * 3 * N);
  if (!rc) rc = d2h(c, rng, c->st.rng, (size_t)slots * 4);
  if (!rc && NQ > 0) rc = d2h(c, xq, c->st.xq, (size_t)W * 3 * NQ);
  if (!rc) rc = d2h(c, sums, c->st.sums, (size_t)W * 8);
  if (rc) return rc;
  std::vector<double> wt, fratio;
  std::vector<int> iage;
  if (dmc) {
    rc = d2h(c, wt, c->dmc.db.wt, (size_t)W);
    if (!rc) rc = d2h(c, fratio, c->dmc.db.fratio, (size_t)W);
    if (!rc) rc = d2h(c, iage, c->dmc.db.iage, (size_t)W);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  o.put(x.data(), x.size());
  o.put(rng.data(), rng.size());
  o.put(xq.data(), xq.size());
  o.put(sums.data(), sums.size());
  const double vg[10] = {c->ecum, c->ecm2, c->wcum, c->pecum, c->tpbcum, c->pecm2, c->tpbcm2, c->acc, c->ecum1s, c->ecm21s};
  o.put(vg, 10);
  const int64_t vi[2] = {c->iblk, c->passes};
  o.put(vi, 2);
  if (dmc) {
    const DmcHost &d = c->dmc;
    o.put(wt.data(), wt.size());
    o.put(fratio.data(), fratio.size());
    o.put(iage.data(), iage.size());
    uint64_t pop[4];
    d.pop.store(pop);
    o.put(pop, 4);
    const double ds[21] = {d.tau, d.etrial, d.eest, d.eigv, d.wdsumo, d.fprod, d.wsum1, d.esum1, d.pesum, d.tpbsum,
                           d.tausum, d.wgsum, d.egsum, d.wgcum, d.egcum, d.wgcm2, d.egcm2, d.taucum, d.pecum,
                           d.tpbcum, d.acc};
    o.put(ds, 21);
    const int64_t di[10] = {d.nconf, d.nfprod, d.ipass, d.nacc, d.nodecr, d.nbrnch, d.iblk, (int64_t)d.ff.size(),
                            d.icasula, d.nmove_casula};
    o.put(di, 10);
    o.put(d.trymove);
    o.put(d.ff.data(), d.ff.size());
  }
  if (h.nstates > 1) {
    // several states: cumulative and current-block sums of every state
    std::vector<double> q((size_t)W * h.nstates * 4);
    CK(cudaMemcpyAsync(q.data(), c->hb.sums_ms, sizeof(double) * q.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    o.put(c->st_cum.data(), c->st_cum.size());
    o.put(q.data(), q.size());
  }
  out.swap(o.b);
  return CW_OK;
}

int ck_restore(cw_ctx *c, const uint8_t *buf, size_t n) {
  const CSys &h = c->h;
  CkReader r{buf, n};
  char mg[8];
  r.get(mg, 8);
  if (!r.ok || std::memcmp(mg, kCkMagic, 8) != 0) return fail(c, CW_ERR_ARG, "restore: not a checkpoint buffer");
  int64_t hdr[12];
  r.get(hdr, 12);
  if (!r.ok || hdr[0] != 1) return fail(c, CW_ERR_ARG, "restore: unsupported checkpoint version");
  const bool dmc = hdr[1] == 1;
  if (hdr[2] != h.N || hdr[3] != h.nup || hdr[4] != h.K || hdr[5] != h.Oa || hdr[6] != h.M || hdr[7] != h.ndet ||
      hdr[8] != std::max(h.nquad, 0))
    return fail(c, CW_ERR_ARG, "restore: checkpoint of a different system");
  const int W = (int)hdr[9], slots = (int)hdr[10], N = h.N, NQ = std::max(h.nquad, 0);
  if (W <= 0 || slots < W) return fail(c, CW_ERR_ARG, "restore: bad walker counts");
  std::vector<double> x((size_t)W * 3 * N), xq((size_t)W * 3 * NQ), sums((size_t)W * 8);
  std::vector<uint64_t> rng((size_t)slots * 4);
  r.get(x.data(), x.size());
  r.get(rng.data(), rng.size());
  r.get(xq.data(), xq.size());
  r.get(sums.data(), sums.size());
  double vg[10];
  int64_t vi[2];
  r.get(vg, 10);
  r.get(vi, 2);
  std::vector<double> wt, fratio, ds(21), ff;
  std::vector<int> iage;
  uint64_t pop[4] = {0, 0, 0, 0};
  int64_t di[10] = {0};
  double trymove = 0;
  if (dmc) {
    wt.resize(W);
    fratio.resize(W);
    iage.resize(W);
    r.get(wt.data(), W);
    r.get(fratio.data(), W);
    r.get(iage.data(), W);
    r.get(pop, 4);
    r.get(ds.data(), 21);
    r.get(di, 10);
    trymove = r.get<double>();
    if (di[7] < 1 || di[7] > (1 << 20)) return fail(c, CW_ERR_ARG, "restore: bad nfprod");
    ff.resize((size_t)di[7]);
    r.get(ff.data(), ff.size());
  }
  // several states: cumulative and current-block sums of every state
  std::vector<double> st_cum, st_q;
  if (h.nstates > 1) {
    st_cum.assign((size_t)h.nstates * 5, 0.0);
    st_q.assign((size_t)W * h.nstates * 4, 0.0);
    r.get(st_cum.data(), st_cum.size());
    r.get(st_q.data(), st_q.size());
  }
  if (!r.ok || r.off != n) return fail(c, CW_ERR_ARG, "restore: truncated or oversized checkpoint buffer");
  BIND(c);
  int rc = dmc ? dmc_alloc(c, slots) : alloc_walkers(c, W);
  if (rc) return rc;
  c->W = W;
  c->st.W = W;
  CK(cudaMemcpyAsync(c->st.x, x.data(), sizeof(double) * x.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->st.rng, rng.data(), sizeof(uint64_t) * rng.size(), cudaMemcpyHostToDevice, c->stream));
  if (NQ > 0) CK(cudaMemcpyAsync(c->st.xq, xq.data(), sizeof(double) * xq.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->st.status, 0, sizeof(int) * slots, c->stream));
  // derived state: every table of the current configurations
  rc = run_hpsi(c, 0);
  if (rc) return rc;
  const long nt = (long)W * N;
  k_nearest<<<(unsigned)((nt + 127) / 128), 128, 0, c->stream>>>(c->h, c->st);
  LCHK("k_nearest");
  CK(cudaMemcpyAsync(c->st.sums, sums.data(), sizeof(double) * sums.size(), cudaMemcpyHostToDevice, c->stream));
  c->ecum = vg[0]; c->ecm2 = vg[1]; c->wcum = vg[2]; c->pecum = vg[3]; c->tpbcum = vg[4];
  c->pecm2 = vg[5]; c->tpbcm2 = vg[6]; c->acc = vg[7]; c->ecum1s = vg[8]; c->ecm21s = vg[9];
  c->iblk = vi[0];
  c->passes = vi[1];
  if (dmc) {
    DmcHost &d = c->dmc;
    DmcBuf &b = d.db;
    for (int w = 0; w < W; w++) {
      d.h_wt[w] = wt[w];
      d.h_iage[w] = iage[w];
    }
    CK(cudaMemcpyAsync(b.wt, d.h_wt, sizeof(double) * W, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(b.iage, d.h_iage, sizeof(int) * W, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(b.fratio, fratio.data(), sizeof(double) * W, cudaMemcpyHostToDevice, c->stream));
    d.pop.load(pop);
    d.tau = ds[0]; d.etrial = ds[1]; d.eest = ds[2]; d.eigv = ds[3]; d.wdsumo = ds[4]; d.fprod = ds[5];
    d.wsum1 = ds[6]; d.esum1 = ds[7]; d.pesum = ds[8]; d.tpbsum = ds[9]; d.tausum = ds[10]; d.wgsum = ds[11];
    d.egsum = ds[12]; d.wgcum = ds[13]; d.egcum = ds[14]; d.wgcm2 = ds[15]; d.egcm2 = ds[16]; d.taucum = ds[17];
    d.pecum = ds[18]; d.tpbcum = ds[19]; d.acc = ds[20];
    d.nconf = (int)di[0]; d.nfprod = (int)di[1]; d.ipass = di[2]; d.nacc = di[3]; d.nodecr = di[4];
    d.nbrnch = di[5]; d.iblk = di[6];
    d.trymove = trymove;
    d.ff = ff;
    d.on = true;
    if (di[8] != 0) {
      rc = cw_dmc_set_tmoves(c, (int)di[8]);
      if (rc) return rc;
    }
    d.nmove_casula = di[9];
  }
  if (h.nstates > 1) {
    c->st_cum = st_cum;
    CK(cudaMemcpyAsync(c->hb.sums_ms, st_q.data(), sizeof(double) * st_q.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return check_status(c);
}

}  // namespace

extern "C" long cw_checkpoint_bytes(cw_ctx *c) {
  if (!c) return -1;
  std::vector<uint8_t> b;
  if (ck_serialize(c, b)) return -1;
  return (long)b.size();
}

extern "C" int cw_checkpoint(cw_ctx *c, void *buf, long bytes) {
  if (!c || !buf) return fail(c, CW_ERR_ARG, "cw_checkpoint: bad arguments");
  std::vector<uint8_t> b;
  int rc = ck_serialize(c, b);
  if (rc) return rc;
  if ((long)b.size() > bytes) return fail(c, CW_ERR_ARG, "cw_checkpoint: buffer of %ld bytes, %zu needed", bytes, b.size());
  std::memcpy(buf, b.data(), b.size());
  return CW_OK;
}

extern "C" int cw_restore(cw_ctx *c, const void *buf, long bytes) {
  if (!c || !buf || bytes <= 0) return fail(c, CW_ERR_ARG, "cw_restore: bad arguments");
  return ck_restore(c, static_cast<const uint8_t *>(buf), (size_t)bytes);
}

extern "C" int cw_dmc_set_tmoves(cw_ctx *c, int icasula) {
  if (!c || !c->dmc.on) return fail(c, CW_ERR_STATE, "cw_dmc_set_tmoves: no DMC population");
  if (icasula != 0 && icasula != -1) return fail(c, CW_ERR_UNSUPPORTED, "T-moves: icasula %d (0 or -1 supported)", icasula);
  if (icasula != 0 && c->h.nloc == 0) return fail(c, CW_ERR_ARG, "T-moves need a pseudopotential (nloc > 0)");
  if (icasula != 0 && c->h.nstates > 1)
    return fail(c, CW_ERR_UNSUPPORTED, "T-moves of multi-state wave functions are not implemented");
  if (icasula != 0 && c->md_on && c->smem_md_tmove > 227 * 1024)
    return fail(c, CW_ERR_UNSUPPORTED, "multideterminant T-move stage exceeds shared memory");
  BIND(c);
  DmcHost &d = c->dmc;
  if (icasula != 0 && !c->hb.tvpsp) {
    const CSys &h = c->h;
    DALLOC(d.allocs, c->hb.tvpsp, (size_t)d.mwalk * h.N * h.nquad * h.M);
    if (c->md_on) DALLOC(d.allocs, c->hb.tvtrj, (size_t)d.mwalk * h.N * h.nquad * h.M);
  }
  d.icasula = icasula;
  return CW_OK;
}

extern "C" int cw_dmc_counts(cw_ctx *c, long *out) {
  if (!c || !out || !c->dmc.on) return fail(c, CW_ERR_STATE, "cw_dmc_counts: no DMC population");
  const DmcHost &d = c->dmc;
  out[0] = d.nacc;
  out[1] = d.nodecr;
  out[2] = d.nbrnch;
  out[3] = d.nmove_casula;
  return CW_OK;
}
