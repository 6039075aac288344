/*
 * oracle.h — CPU FP64 restatement of CHAMP's VMC hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA engine is
 * compared against (tests/, the smoke check and bench.py's CPU-baseline leg).
 * It is never linked into, loaded by, or called from the engine library.
 *
 * Every function restates the CHAMP routine it names (paths relative to the
 * CHAMP source tree) in plain C++ with the same loop order wherever that
 * order affects rounding.
 */
#ifndef CHAMP_ORACLE_H
#define CHAMP_ORACLE_H
#include <stdint.h>
#include "../include/champ_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

void *or_sys_create(const cw_system_desc *desc);
void or_sys_destroy(void *sys);
int or_nterms4(int nordc);
int or_jas_nraw(void *sys);
void or_jas_raw(void *sys, const double *x, double *out);

/* pot_nn: nuclear repulsion (module pot, used by zerest vmc/acuest.f90). */
double or_pot_nn(int ncent, const double *cent, const double *znuc, const int32_t *iwctype);
/* matinv (vmc/matinv.f90:22): in-place inverse of a(n,n) column-major, det. */
int or_matinv(double *a, int n, double *det);
/* xoshiro256** (vmc/xoroshiro256starstar.c): states of walker w = setrn(irn)
 * followed by w jump() calls (vmc/parser.f90:651-661). */
void or_rng_states(const int32_t *irn8, int nwalk, uint64_t *out);
/* draw n uniforms (next_uniform_double) from state (updated in place). */
void or_rng_uniform(uint64_t *state, int n, double *out);
/* gesqua (vmc/rotqua.f90:3): nq in/out, fills xq,yq,zq,wq. */
void or_gesqua(int *nq, double *xq, double *yq, double *zq, double *wq);
/* sites (vmc/sites.f90:3) with mc_configs_start's nsite rule
 * (vmc/mc_configs.f90:75-96); consumes draws from `state`. */
void or_sites(void *sys, uint64_t *state, double *x);

/* Single-configuration evaluations (x = xold(3,nelec)). */
void or_orbitals(void *sys, const double *x, double *orb, double *dorb, double *ddorb);
void or_jastrow(void *sys, const double *x, double *psij, double *v, double *d2j);
int or_slater(void *sys, const double *x, double *slmi, double *det);
/* hpsi (vmc/hpsi.f90:3); out[0..5] = energy, psid, psij, ekin, pe_local, vpsp */
int or_hpsi(void *sys, const double *x, const double *xq, const double *yq,
            const double *zq, double *out);

/* Walker populations (one walker == one CHAMP MPI rank in vmc_one_mpi). */
void *or_walkers_create(void *sys, int nwalk, const double *x, const uint64_t *rng);
void or_walkers_destroy(void *ws);
int or_vmc_steps(void *ws, int nstep, int nthreads);
/* zerest (vmc/acuest.f90:179): recompute hpsi, zero all estimators. */
int or_zerest(void *ws);
void or_end_block(void *ws, double *block_energy);
void or_results(void *ws, double *out);
int or_results_state(void *ws, int istate, double *out);
void or_opt_ci(void *ws, int enable);
void or_ci_o(void *ws, double *out);
void or_opt_ci_sums(void *ws, double *o, double *eo, double *oo, double *wsum);
void or_state_energies(void *ws, double *e, double *psid);
void or_get_walkers(void *ws, double *x, uint64_t *rng);
void or_get_sums(void *ws, double *out);
void or_get_state(void *ws, double *eold, double *psido, double *psijo);

/* DMC population (dmc_ps, branching, splitj, acues1/acuest), one CHAMP rank:
 * walker slot k owns move stream rng[k] (mwalk slots), pop_rng drives
 * rotqua and splitj. */
void *or_dmc_create(void *sys, int nwalk, const double *x, const uint64_t *rng, const uint64_t *pop_rng,
                    double tau, double etrial, int mwalk, int nfprod);
void or_dmc_destroy(void *dmc);
int or_dmc_steps(void *dmc, int nstep, int nthreads);
void or_dmc_end_block(void *dmc);
void or_dmc_results(void *dmc, double *out);
int or_dmc_walkers(void *dmc, double *x, double *wt, double *eold, uint64_t *rng);
int or_dmc_set_tmoves(void *dmc, int icasula);
long or_dmc_tmoves(void *dmc);

#ifdef __cplusplus
}
#endif
#endif
