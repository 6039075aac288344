/*
 * champ_b200.h — C ABI of the B200 walker engine for CHAMP's VMC/DMC inner loop.
 *
 * Plain C: pointers, sizes and status codes only.  Every array is laid out
 * exactly like the corresponding CHAMP Fortran module array with the index
 * order reversed (Fortran a(i,j,k) column-major == C a[k][j][i] row-major),
 * so a Fortran caller passes its module arrays by reference through
 * iso_c_binding without copying.  Electron, orbital, centre and type indices
 * stored INSIDE arrays (iworbd, iwlbas, iwrwf) keep CHAMP's 1-based values;
 * iwctype is 0-based.
 *
 * Each entry point names the CHAMP routine (file:line, paths relative to the
 * CHAMP source tree) whose role it takes over.
 */
#ifndef CHAMP_B200_H
#define CHAMP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Fixed dimensions of CHAMP's parameter modules. */
#define CW_NCOEF    5    /* small-r polynomial, vmc_mod NCOEF (module/m_vmc.f90:96)      */
#define CW_MPS_L    4    /* max pseudopotential channels + local (pseudo_mod MPS_L)       */
#define CW_MGAUSS   16   /* max Gaussian terms per ECP channel                            */
#define CW_MPS_QUAD 86   /* max angular quadrature points (gesqua, vmc/rotqua.f90:3)      */

/* Status codes returned by every cw_* call. */
enum {
  CW_OK = 0,
  CW_ERR_ARG = 1,         /* invalid argument / unsupported size                      */
  CW_ERR_CUDA = 2,        /* CUDA runtime error (message in cw_last_error)            */
  CW_ERR_OOM = 3,         /* device allocation failed                                 */
  CW_ERR_SINGULAR = 4,    /* a Slater matrix was singular (matinv, vmc/matinv.f90:59) */
  CW_ERR_UNSUPPORTED = 5, /* input outside what the engine implements                 */
  CW_ERR_STATE = 6        /* call out of order (e.g. no walkers set)                  */
};

/* Arithmetic of the move/energy kernels. */
enum {
  CW_PREC_FP64 = 0,   /* plain FP64 everywhere (parity path)                           */
  CW_PREC_MIXED = 1   /* FP32/3xBF16 LCAO + FP32 Jastrow sums, FP64 Slater algebra     */
};

/*
 * Description of one molecular system, i.e. the contents of CHAMP's modules
 * after parser() (vmc/parser.f90) has read the input: geometry (system),
 * numerical basis (numbas, numbas1, numexp), LCAO (slater, dorb_m), Jastrow
 * type 4 (jastrow, bparm), Gaussian ECP (pseudo, gauss_ecp, qua) and the
 * Metropolis parameters (metropolis).  The engine copies everything it needs
 * at cw_create; the caller's arrays are borrowed for that call only.
 */
typedef struct cw_system_desc {
  /* --- system (module/m_system.f90) --- */
  int32_t nelec, nup;          /* ndn = nelec - nup                                  */
  int32_t ncent, nctype;
  const int32_t *iwctype;      /* [ncent], 0-based atom type of each centre          */
  const double *cent;          /* [ncent][3] bohr                                    */
  const double *znuc;          /* [nctype] (valence) charges                         */
  double pecent;               /* nuclear repulsion, pot_nn                          */

  /* --- numerical radial basis (read_bas_num, vmc/read_bas_num.f90:11) --- */
  int32_t mrwf;                /* leading dim: max radial functions per type         */
  int32_t mrwf_pts;            /* leading dim: max grid points                       */
  const int32_t *nrbas;        /* [nctype]                                           */
  const int32_t *igrid;        /* [nctype] 1, 2 or 3                                 */
  const int32_t *nr;           /* [nctype]                                           */
  const double *arg;           /* [nctype]                                           */
  const double *r0;            /* [nctype] after read_bas_num's igrid=3 rescaling    */
  const double *rwf;           /* [nctype][mrwf][mrwf_pts]                           */
  const double *d2rwf;         /* [nctype][mrwf][mrwf_pts] spline2 second derivs     */
  const double *ce;            /* [nctype][mrwf][CW_NCOEF] small-r polynomial        */
  const double *ae;            /* [nctype][mrwf][2] large-r exponential              */
  const double *rmaxwf;        /* [nctype][mrwf] cutoff radius                       */
  int32_t mbastyp;             /* leading dim of iwlbas/iwrwf                        */
  const int32_t *nbastyp;      /* [nctype] AOs on a centre of this type              */
  const int32_t *iwlbas;       /* [nctype][mbastyp] Slm index 1..35                  */
  const int32_t *iwrwf;        /* [nctype][mbastyp] radial function 1..nrbas         */

  /* --- orbitals and determinants (slater, dorb_m) --- */
  int32_t nbasis, norb;
  const double *coef;          /* [norb][nbasis] = Fortran coef(nbasis,norb)          */
  int32_t ndet;                /* determinants; kref = the first one                  */
  const int32_t *iworbd;       /* [ndet][nelec] 1-based orbital of each electron slot */
  const double *cdet;          /* [ndet] (excitations up to 4-fold per spin on the GPU) */

  /* --- Jastrow ijas=4 (jastrow, bparm; read_jastrow_file) --- */
  int32_t norda, nordb, nordc;
  int32_t isc;                 /* scaling type 2..5 (scale_dist.f90)                  */
  int32_t nspin2b, nocuspb;
  double scalek;
  const double *a4;            /* [nctype][norda+1]                                   */
  const double *b;             /* [nspin2b][nordb+1]                                  */
  const double *c;             /* [nctype][nterms4(nordc)]                            */

  /* --- Gaussian ECP (pseudo, gauss_ecp; readps_gauss) --- */
  int32_t nloc;                /* 0 all-electron, 4 Gaussian ECP                      */
  const int32_t *lpot;         /* [nctype] channels incl. local (local = index lpot)  */
  const int32_t *necp_term;    /* [nctype][CW_MPS_L]   (l index 0..lpot-1 = CHAMP 1..lpot) */
  const int32_t *necp_power;   /* [nctype][CW_MPS_L][CW_MGAUSS]                        */
  const double *ecp_exponent;  /* [nctype][CW_MPS_L][CW_MGAUSS]                        */
  const double *ecp_coef;      /* [nctype][CW_MPS_L][CW_MGAUSS]                        */
  int32_t nquad;
  const double *xq0, *yq0, *zq0, *wq;  /* [nquad] unrotated quadrature (gesqua)      */

  /* --- metropolis (parser.f90:398-404) --- */
  double deltar, deltat, fbias;

  /* --- several states sharing orbitals and Jastrow (csfs nstates,
   *     mstates_ctrl iguiding, mstates3 weights_g; vmc/determinante.f90:134-230,
   *     vmc/determinant_psig.f90:3).  nstates 0 or 1: one state; > 1 (VMC
   *     only, at most 8): cdet holds [nstates][ndet]; iguiding = 0: the walk
   *     samples |psi_1|^2 and state s is weighted by (psi_s/psi_1)^2;
   *     iguiding > 0: the walk samples psi2g |psi_1|^2 with
   *     psi2g = sum_i weights_g[i] (psi_i/psi_1)^2 (anormo = 1) and state s
   *     is weighted by (psi_s/psi_1)^2 / psi2g. --- */
  int32_t nstates;
  int32_t iguiding;
  const double *weights_g;     /* [nstates] guiding weights (read only when iguiding > 0) */
} cw_system_desc;

typedef struct cw_ctx cw_ctx;

/* ------------------------------------------------------------------------ */
/* Life cycle                                                               */
/* ------------------------------------------------------------------------ */

/* Upload one system and set up the engine on CUDA device `device`.
 * Replaces the module set-up CHAMP does after parser() (vmc/parser.f90:~150-700,
 * set_scale_dist vmc/scale_dist.f90:3). */
int cw_create(cw_ctx **ctx, const cw_system_desc *desc, int device, int precision);
void cw_destroy(cw_ctx *ctx);
const char *cw_last_error(const cw_ctx *ctx);
int cw_sync(cw_ctx *ctx);

/* Set the walker population: x [nwalk][nelec][3] (= CHAMP xold(3,nelec) per
 * walker) and xoshiro256** states rng [nwalk][4] (= the 8 int32 of setrn,
 * vmc/random.f90:27, reinterpreted as 4 uint64).  Replaces mc_configs_start
 * (vmc/mc_configs.f90:33) plus the per-rank jumprn (vmc/parser.f90:654-661).
 * Also runs the initial hpsi of zerest (vmc/acuest.f90:179) on every walker
 * with the unrotated quadrature, and zeroes the estimators. */
int cw_set_walkers(cw_ctx *ctx, int nwalk, const double *x, const uint64_t *rng);
int cw_get_walkers(cw_ctx *ctx, double *x, uint64_t *rng);

/* Per-walker status words of the population, status [nwalk]: bit 0 the
 * walker's Slater matrix was singular at its last full recompute (CHAMP
 * stops the run there, vmc/matinv.f90:59-63), bit 1 its local energy was not
 * finite, bit 2 a rejection loop of its proposal gave up.  A call that
 * returned CW_ERR_SINGULAR or CW_ERR_STATE leaves the population in place,
 * so the caller can find the walkers concerned (for example to draw new
 * start positions for them and call cw_set_walkers again). */
int cw_walker_status(cw_ctx *ctx, int32_t *status);

/* Device-clock stamps: cw_stamp enqueues, on the context's stream, a write of
 * the device's global nanosecond clock into the context's next stamp slot
 * (up to 16384 per context); cw_stamps waits for the stream, copies the first
 * min(n, count) stamps to ns and returns the count.  Stamps around blocks of
 * work of several contexts give the device-side timeline on which their
 * overlap is read (no CHAMP counterpart: a serving aid). */
int cw_stamp(cw_ctx *ctx);

/* Tile autotuner (no CHAMP counterpart): times each N tile (32, 48, 64, 80
 * orbitals) of the FP64 tensor-core LCAO contraction on this context's two
 * shapes (the move's 4 rows per walker, the all-electron chunk's 5 rows per
 * electron), reps launches each, and keeps the fastest; the choice changes
 * no result (every output sums its K slices in the same order).  Needs the
 * walkers (cw_set_walkers); choice [2] (nullable) receives the move and
 * all-electron tiles.  The mixed path's tensor-core kernel has one tile. */
int cw_autotune(cw_ctx *ctx, int reps, int32_t *choice);

/* Batches of contexts (no CHAMP counterpart; the batched configuration of
 * many systems).  A batch holds contexts of one device; cw_batch_vmc_steps
 * advances every one of them by nstep metrop6 sweeps through one CUDA graph
 * whose child nodes are the contexts' own captured sweep graphs (captured
 * here where needed), with no edges between them: one graph launch per sweep
 * for all systems, which the device runs side by side.  The batch's work is
 * ordered after each context's queued work and before its next, so
 * cw_end_block, cw_results etc. are used per context as after cw_vmc_steps;
 * each context's results are bitwise those of cw_vmc_steps on it alone.
 * cw_batch_last_ms: device time of the last call's sweeps.
 *
 * cw_batch_set_ragged(batch, bands) with bands >= 1 switches the batch to
 * one launch per move stage over the walkers of many systems (of different
 * electron, centre, basis and orbital counts): the systems, sorted by
 * electron count, are cut into `bands` runs of about equal work; in a band,
 * electron k of every system with more than k electrons moves in the same
 * six launches, each block working on one system's walkers, and the bands'
 * chains run side by side; after its last electron a system's hpsi runs on
 * its own stream inside the same graph.  bands = 0 returns to the child
 * graphs.  Each system takes the walk it takes alone:
 * the same random streams and decisions, bitwise in mixed precision, to
 * rounding (1e-10 relative over a few sweeps) in FP64.  Refused (CW_ERR_UNSUPPORTED, reason in cw_batch_last_error)
 * unless every system is a one-determinant VMC population with spins of at
 * most 128 electrons, the same precision and the same e-e-n order.
 * cw_batch_info: [bands asked for (0: not ragged), N tile of the grouped
 * FP64 LCAO (timed when the graph is built), ragged launches per sweep, the
 * systems' own hpsi launches per sweep, bands of the built graph]. */
typedef struct cw_batch cw_batch;
int cw_batch_create(cw_batch **batch, cw_ctx **ctxs, int nctx);
int cw_batch_vmc_steps(cw_batch *batch, int nstep);
float cw_batch_last_ms(const cw_batch *batch);
const char *cw_batch_last_error(const cw_batch *batch);
void cw_batch_destroy(cw_batch *batch);
int cw_batch_set_ragged(cw_batch *batch, int bands);
int cw_batch_info(const cw_batch *batch, int64_t *info);
int cw_stamps(cw_ctx *ctx, int64_t *ns, int n);

/* ------------------------------------------------------------------------ */
/* Batched drop-ins for CHAMP's per-walker routines                          */
/* ------------------------------------------------------------------------ */

/* `nstep` VMC steps for every walker: per step rotqua (vmc/rotqua.f90:357,
 * only if nloc>0) then metrop6 (vmc/metrop_mov1_slat.f90:3: one accelerated
 * Metropolis move per electron, hpsi at the end, weighted sums).  Same random
 * number consumption as CHAMP rank w with the walker's own stream.
 * Accumulates per-walker esum/wsum/pesum/tpbsum and acceptance. */
int cw_vmc_steps(cw_ctx *ctx, int nstep);

/* Close a block for every walker: acuest (vmc/acuest.f90:61) +
 * acuest_reduce (vmc/acuest_reduce.f90:3) with walkers in the role of ranks.
 * Writes, if non-NULL, block_energy = Σ esum / Σ wsum of the block. */
int cw_end_block(cw_ctx *ctx, double *block_energy);

/* Final estimates, finwrt (vmc/finwrt.f90:75-187): out[0]=E, out[1]=err,
 * out[2]=sigma, out[3]=Tcor, out[4]=acceptance, out[5]=PE, out[6]=KE,
 * out[7]=blocks so far (iblk). */
int cw_results(cw_ctx *ctx, double *out);

/* Results of state `istate` (0-based) of a multi-state wave function, from
 * the reweighted block sums of that state (acuest / finwrt per istate):
 * out[0] energy, out[1] its error, out[5] potential, out[6] kinetic energy,
 * out[7] blocks; out[2..4] are NaN (sigma, Tcorr and acceptance are those of
 * the sampled state, cw_results).  CW_ERR_ARG for istate outside [0, nstates). */
int cw_results_state(cw_ctx *ctx, int istate, double *out);

/* Wave-function optimisation: derivatives of ln psi with respect to the CI
 * coefficients (optci_deloc's ci_o, vmc/optci.f90:49-51, taken for the
 * coefficients as given in cw_system_desc, i.e. with the orbital-order sign
 * of multideterminants_define applied) and the stochastic-reconfiguration
 * sums of optwf_store (vmc/optwf_handle_wf.f90:1465) over the samples of
 * every VMC sweep: sum O_k, sum E_L O_k and, with with_overlap, the overlap
 * sum O_k O_l (one FP64 GEMM over the walkers).  Needs a multideterminant
 * expansion with one state; enable after cw_set_walkers (a new population
 * disables it).  cw_opt_ci_sums copies the sums (o, eo [ndet], oo
 * [ndet][ndet] or NULL, wsum = number of samples) and resets them;
 * cw_ci_o gives the per-walker derivatives of the last hpsi, [nwalk][ndet].
 * cw_opt_ci(ctx, e, ov) is cw_opt_setup(ctx, e, 0, NULL, ov) and
 * cw_opt_ci_sums is cw_opt_sums. */
int cw_opt_ci(cw_ctx *ctx, int enable, int with_overlap);
int cw_opt_ci_sums(cw_ctx *ctx, double *o, double *eo, double *oo, double *wsum);
int cw_ci_o(cw_ctx *ctx, double *out);

/* Jastrow and CI parameters together: the optimisation vector of a walker is
 * [njas Jastrow parameters | ndet CI coefficients when ci != 0], the layout
 * of optwf_store's sr_o (vmc/optwf_handle_wf.f90:1517-1521).  The Jastrow
 * part is deriv_jastrow4's gvalue (vmc/deriv_jastrow4.f90, d ln psi / d p of
 * the varied a, b, c parameters with the cusp-fixed e-e-n terms folded in by
 * checkdepend4's dependencies): the engine computes the raw derivative of J
 * with respect to every Jastrow coefficient -- cw_jas_nraw entries per
 * walker, [nctype][norda+1] a (1 = a(1), 2 = a(2), q >= 3 the r^(q-1)
 * coefficient), [nspin2b][nordb+1] b (the same for e-e), [nctype][nterms]
 * e-e-n terms -- and applies jas_map ([nraw][njas], row-major, built on the
 * host from the jasderiv selection) to it.  After every VMC sweep the sums
 * of cw_opt_sums run over the whole vector: o, eo [np], oo [np][np] (with
 * with_overlap), wsum; np = njas + (ci ? ndet : 0) + norbterm (cw_opt_orb).
 * ci = 0, njas = 0 and no orbital rotations disables.  Needs one state; Jastrow derivatives need norda, nordb >= 1.
 * cw_jas_raw gives the raw derivatives of the last hpsi [nwalk][nraw],
 * cw_jas_o the Jastrow part of the vector [nwalk][njas]. */
int cw_opt_setup(cw_ctx *ctx, int ci, int njas, const double *jas_map, int with_overlap);

/* Orbital rotations of the optimisation vector (ioptorb, optorb_define
 * vmc/optorb.f90:838-1030): ideriv [norbterm][2] holds 1-based orbital
 * indices (io, jo) of the variations phi_io -> phi_io + a phi_jo (orbitals
 * as rows of cw_system_desc.coef).  The next cw_opt_setup appends them to
 * the vector after the Jastrow and CI parts, in optwf_store's order
 * (vmc/optwf_handle_wf.f90:1517-1524); norbterm = 0 removes them.  The
 * derivative of a walker is optorb_deriv's orbprim (vmc/optorb.f90:5-95)
 * for one determinant: sum over the spins whose determinant holds io of
 * aa(irep, jo) = sum_i slmi(irep + (i-1) nel) orb(i, jo).  One determinant
 * and one state (CW_ERR_UNSUPPORTED otherwise: the multideterminant zmat
 * terms are not built).  cw_orb_o gives the per-walker derivatives of the
 * last hpsi, [nwalk][norbterm]. */
int cw_opt_orb(cw_ctx *ctx, int norbterm, const int32_t *ideriv);
int cw_orb_o(cw_ctx *ctx, double *out);
int cw_opt_sums(cw_ctx *ctx, double *o, double *eo, double *oo, double *wsum);
int cw_jas_nraw(cw_ctx *ctx, int *nraw);
int cw_jas_raw(cw_ctx *ctx, double *out);
int cw_jas_o(cw_ctx *ctx, double *out);

/* Per-walker local energies and psi_D of every state from the last hpsi:
 * energy, psid [nwalk][nstates]. */
int cw_state_energies(cw_ctx *ctx, double *energy, double *psid);

/* Local energy of every walker at its current configuration, hpsi
 * (vmc/hpsi.f90:3) with the quadrature grid (xq,yq,zq)[nquad] given (NULL:
 * the unrotated one).  Outputs per walker (any may be NULL): energy, psid,
 * psij, ekin. */
int cw_hpsi(cw_ctx *ctx, const double *xq, const double *yq, const double *zq,
            double *energy, double *psid, double *psij, double *ekin);

/* Orbitals of all electrons of every walker, orbitals (vmc/orbitals.f90:18):
 * orb [nwalk][norb][nelec] (= orb(nelec,norb)), dorb [nwalk][3][nelec][norb]
 * (= dorb(norb,nelec,3)), ddorb [nwalk][nelec][norb] (= ddorb(norb,nelec)). */
int cw_orbitals(cw_ctx *ctx, double *orb, double *dorb, double *ddorb);

/* Jastrow factor of every walker, jastrow_factor (vmc/jastrow.f90:3):
 * psij [nwalk], v [nwalk][nelec][3], d2j [nwalk]. */
int cw_jastrow(cw_ctx *ctx, double *psij, double *v, double *d2j);

/* Slater inverses and determinants after the full recompute of determinant
 * (vmc/determinant.f90:9): slmi [nwalk][2][nmax*nmax] with nmax=max(nup,ndn)
 * (spin iab: slmi(j+nel*(i-1)) of CHAMP), det [nwalk][2]. */
int cw_slater(cw_ctx *ctx, double *slmi, double *det);

/* ------------------------------------------------------------------------ */
/* Per-electron routines, for a driver that keeps metrop6's electron loop on */
/* the host (vmc/metrop_mov1_slat.f90:131-630), batched over the walkers of */
/* a VMC population (CW_ERR_STATE for a DMC population).  The caller makes */
/* the proposal and the accept/reject decision; the engine keeps the tables. */
/* Per electron iel (0-based): cw_grad(iel, 1), proposal, cw_psie(iel),      */
/* cw_grad(iel, 0), decision, cw_commit(iel), cw_update_ymat(iel); after the */
/* last electron, cw_hpsi.                                                  */
/* ------------------------------------------------------------------------ */

/* psie (vmc/hpsie.f90:3) of electron iel at the proposed point of every
 * walker, xnew [nwalk][3]: distances, jastrowe (jastrow4e), determinante
 * (orbitalse + the determinant ratio) and, with several determinants,
 * multideterminante + determinante_psit.  psid [nwalk] = psi_D at the point
 * (CHAMP's psid(1)), psij [nwalk] = the Jastrow exponent there (psij(1));
 * either may be NULL.  The walkers' own tables are not changed. */
int cw_psie(cw_ctx *ctx, int iel, const double *xnew, double *psid, double *psij);

/* compute_determinante_grad (vmc/determinante.f90:69) of electron iel:
 * vd [nwalk][3] = grad ln|psi_D| + grad J, iflag_move = 1 at the current
 * position, 0 at the point of the last cw_psie of the same electron
 * (CW_ERR_STATE without one). */
int cw_grad(cw_ctx *ctx, int iel, int iflag_move, double *vd);

/* The end of a move of electron iel (vmc/metrop_mov1_slat.f90:592-626):
 * walkers with accept[w] != 0 take the point of the last cw_psie as their
 * position, with jassav (vmc/jassav.f90:3) and detsav (vmc/detsav.f90:3:
 * the Sherman-Morrison update of the inverse, the new orbital row and
 * determinant); the other walkers keep their position and tables
 * (distancese_restore).  Needs the cw_psie of the same electron. */
int cw_commit(cw_ctx *ctx, int iel, const int32_t *accept);

/* update_ymat (vmc/multideterminant.f90:562) after the move of electron
 * iel: with several determinants the engine prepares the multideterminant
 * tables for the move of electron iel+1 (the spin-phase sums at the first
 * electron of a spin and the drift correction at its position); cw_grad and
 * cw_psie prepare them as well when this call is left out.  No-op for one
 * determinant. */
int cw_update_ymat(cw_ctx *ctx, int iel);

/* Per-walker sums since the last cw_end_block: out [nwalk][5] =
 * (wsum, esum, pesum, tpbsum, accepted moves). */
int cw_get_sums(cw_ctx *ctx, double *out);

/* Per-walker current values: eold, psido, psijo [nwalk] (any may be NULL). */
int cw_get_state(cw_ctx *ctx, double *eold, double *psido, double *psijo);

/* Device milliseconds of the last cw_vmc_steps call (CUDA events on the
 * engine stream). */
double cw_last_ms(const cw_ctx *ctx);

/* Kernel launches issued by the last cw_vmc_steps call. */
long cw_launches(const cw_ctx *ctx);

/* Device memory the context holds (bytes of its own allocations: system
 * tables, walker state, scratch).  A serving loop admits jobs against an HBM
 * budget with it; no reference counterpart (CHAMP runs one job per process). */
size_t cw_device_bytes(const cw_ctx *ctx);

/* Per-stage device timing.  enable=1 brackets every launch of the following
 * cw_vmc_steps calls with CUDA events on the engine stream (adds event
 * overhead; leave off for throughput runs).  cw_stage_times fills, for each
 * of the CW_NSTAGE stages below, the accumulated milliseconds and launch
 * counts since profiling was enabled. */
enum {
  CW_ST_ROTQUA = 0, CW_ST_PROPOSE, CW_ST_JASTROW_MOVE, CW_ST_BASIS_MOVE, CW_ST_LCAO_MOVE,
  CW_ST_ACCEPT, CW_ST_JASTROW_FULL, CW_ST_BASIS_ALL, CW_ST_LCAO_ALL, CW_ST_SCATTER,
  CW_ST_SLATER_INV, CW_ST_CTILDE, CW_ST_ECP, CW_ST_ENERGY, CW_ST_COMMIT, CW_ST_DMC_WEIGHTS,
  CW_ST_SPLITJ, CW_ST_MDET, CW_ST_TMOVE, CW_NSTAGE
};
int cw_profile(cw_ctx *ctx, int enable);
int cw_stage_times(cw_ctx *ctx, double *ms, long *launches);

/* Orbitals at points, allocating nothing.  No counterpart in CHAMP: this
 * entry point exists for callers that cannot call cudaMalloc while they run
 * (device memory owned by another allocator, or a step loop that cannot take
 * cudaMalloc's implicit device synchronisation).  xyz [npts][3] and out
 * [npts][5][norb] (value, d/dx, d/dy, d/dz, Laplacian of every orbital) are
 * DEVICE pointers on the context's device, provided by the caller.  Basis
 * values in between go to a fixed 16 MiB array that every GPU loading the
 * library reserves until exit, so npts*5*nbasis must not exceed 2^21
 * (CW_ERR_ARG otherwise).  The first call on a device looks up that array's
 * device address (make that first call before any stream capture).  The work
 * is queued on the context's stream: out is ready after cw_sync.  All calls
 * share the one array.  Each call's work waits on the device for the previous
 * call's (a per-device completion event, taken under a host lock), so calls
 * from any contexts and host threads do not overlap on the GPU; calls made
 * inside a stream capture are ordered by their graphs' launches only.  The
 * first-call address lookup is not locked; threads racing there store the
 * same address, which is harmless. */
int cw_orbitals_noalloc(cw_ctx *ctx, int npts, const double *xyz, double *out);

/* ------------------------------------------------------------------------ */
/* Diffusion Monte Carlo (idmc=2: dmc/dmc.f90:88-111); dmc_ps moves for      */
/* pseudopotential wave functions (nloc > 0), dmc_ae moves for all-electron  */
/* ones (nloc = 0, dmc/dmc_ae_mov1.f90:4)                                    */
/* ------------------------------------------------------------------------ */

/* Start a DMC population of nwalk walkers (capacity mwalk = CHAMP's MWALK)
 * from x [nwalk][nelec][3]: init (dmc/init.f90:60-150) — hpsi of every
 * walker with the unrotated quadrature, drift and fratio, wt=1, eest=eigv
 * start values, fprod=1.  rng [mwalk][4]: the move stream of every walker
 * slot (a slot keeps its stream through splitj copies); pop_rng [4]: the
 * population stream that rotqua and splitj draw from (CHAMP's per-rank
 * stream).  tau, etrial, nfprod as in the dmc input.  Replaces the walkers
 * of any earlier cw_set_walkers. */
int cw_dmc_init(cw_ctx *ctx, int nwalk, int mwalk, const double *x, const uint64_t *rng,
                const uint64_t *pop_rng, double tau, double etrial, int nfprod);

/* `nstep` DMC steps of the population, the body of dmc.f90's j loop:
 * rotqua (dmc.f90:94, one rotation for all walkers, only with a
 * pseudopotential), dmc_ps (dmc/dmc_ps_mov1.f90:4) or, for an all-electron
 * wave function, dmc_ae (dmc/dmc_ae_mov1.f90:4: the drift in the frame of
 * the nearest nucleus and a Gaussian / exponential diffusion mixture) --
 * per electron the drift-diffusion move with the Green-function
 * acceptance; hpsi; fratio and reweighting, dmc/branching.f90:27,111;
 * population factor fprod -- then splitj
 * (dmc/splitj.f90:3) and acues1 (dmc/acues1.f90:3).  The population size
 * changes; CW_ERR_STATE if it would exceed mwalk ("SPLITJ: MWALK exceeded"). */
int cw_dmc_steps(cw_ctx *ctx, int nstep);

/* Close a DMC block: the cumulative sums of acuest (dmc/acuest.f90). */
int cw_dmc_end_block(cw_ctx *ctx);

/* DMC estimates, finwrt (dmc/finwrt.f90): out[0]=egave (mixed estimator),
 * out[1]=its error (rn_eff of the block weights), out[2]=nwalk,
 * out[3]=eest, out[4]=acceptance, out[5]=taueff, out[6]=PE, out[7]=KE,
 * out[8]=blocks, out[9]=fprod, out[10]=eigv, out[11]=wdsumo. */
int cw_dmc_results(cw_ctx *ctx, double *out);

/* T-moves (Casula), icasula of the dmc input (dmc_ps :701-795,
 * dmc/nonloc_grid.f90:3): 0 off (default), -1 after each step's reweighting
 * one T-move per walker, chosen over every electron and quadrature point
 * from the negative nonlocal matrix elements of the step's hpsi and always
 * accepted.  Single-determinant wave functions with a pseudopotential. */
int cw_dmc_set_tmoves(cw_ctx *ctx, int icasula);

/* DMC move counts: out[0]=accepted drift-diffusion moves, out[1]=node
 * crossings, out[2]=branching events (nbrnch), out[3]=T-moves. */
int cw_dmc_counts(cw_ctx *ctx, long *out);

/* Current population: *nwalk, and (any may be NULL) x [nwalk][nelec][3],
 * wt [nwalk], eold [nwalk], rng [nwalk][4]; the arrays must hold mwalk. */
int cw_dmc_walkers(cw_ctx *ctx, int *nwalk, double *x, double *wt, double *eold, uint64_t *rng);

/* ------------------------------------------------------------------------ */
/* Checkpoint / restart (dumper / startr)                                     */
/* ------------------------------------------------------------------------ */

/* Checkpoint of the walker population and the accumulators, the content of
 * CHAMP's restart files (vmc/dumper.f90:51-106, dmc/dumper.f90:3,
 * dmc/restart.f90:3): configurations, random streams, the current
 * quadrature rotation, per-walker block sums and the global accumulators,
 * and for a DMC population its weights, ages, fratio, the population stream
 * and the branching scalars.  cw_checkpoint_bytes gives the size (-1 on
 * error); cw_checkpoint fills a host buffer of at least that size.
 * cw_restore loads a buffer made for the same system into a context
 * (replacing its walkers), rebuilds every table with hpsi (startr's hpsi
 * call) and continues the Markov chain exactly where it stopped. */
long cw_checkpoint_bytes(cw_ctx *ctx);
int cw_checkpoint(cw_ctx *ctx, void *buf, long bytes);
int cw_restore(cw_ctx *ctx, const void *buf, long bytes);

/* Diagnostics: measured FMA throughput of the CUDA cores of `device`
 * (fp64=1: FP64, else FP32), TFLOP/s — the roofline denominator of the
 * CUDA-core bound stages.  No counterpart in CHAMP. */
int cw_fma_peak(int device, int fp64, double *tflops);

/* ------------------------------------------------------------------------ */
/* Host-only helpers (no GPU needed)                                        */
/* ------------------------------------------------------------------------ */

/* Random streams of nwalk walkers: setrn(irn) (vmc/random.f90:27) followed
 * by w calls of jump() (vmc/xoroshiro256starstar.c:51) for walker w, as
 * CHAMP does for MPI rank w (vmc/parser.f90:651-661).  out [nwalk][4]. */
int cw_rng_states(const int32_t *irn8, int nwalk, uint64_t *out);

/* Initial electron positions of every walker: mc_configs_start's nsite rule
 * (vmc/mc_configs.f90:75-96) + sites (vmc/sites.f90:3), drawing from each
 * walker's stream (rng [nwalk][4] advanced in place).  x [nwalk][nelec][3]. */
int cw_sites(const cw_system_desc *desc, int nwalk, uint64_t *rng, double *x);

#ifdef __cplusplus
}
#endif
#endif /* CHAMP_B200_H */
