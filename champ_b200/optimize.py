"""Stochastic-reconfiguration step for the CI coefficients from the engine's
SR sums (cw_opt_ci_sums), as optwf_sr does for the CI block of its parameter
vector (vmc/optwf_sr.f90: sr_hs builds <O>, <E O>, <O O>; the update solves
(S + adiag diag(S)) dp = -tau g).

* S_kl = <O_k O_l> - <O_k><O_l>, the overlap of the parameter derivatives;
* g_k = 2 (<E_L O_k> - <E_L><O_k>), the energy gradient.

psi is linear in the coefficients, so sum_k c_k O_k = 1 on every sample:
S c = 0 and g . c = 0 (a rescaling of all coefficients changes nothing).
Like CHAMP, which leaves one coefficient out of the optimised set to fix the
normalisation, the step holds one coefficient (`fixed`, the reference
determinant by default) and moves the others."""
from __future__ import annotations

import copy

import numpy as np


def sr_matrices(sums: dict, energy: float):
    """(S, g) from one set of SR sums; `energy` is the sampled <E_L> of the
    same samples."""
    w = sums["wsum"]
    if w <= 0:
        raise ValueError("no samples in the SR sums")
    o = sums["o"] / w
    eo = sums["eo"] / w
    S = sums["oo"] / w - np.outer(o, o)
    g = 2.0 * (eo - energy * o)
    return S, g


def sr_delta(sums: dict, energy: float, tau: float = 0.02, adiag: float = 0.01, fixed=None) -> np.ndarray:
    """Parameter change of one SR step of length tau over the whole
    optimisation vector (Jastrow parameters, then CI coefficients, as
    cw_opt_sums lays them out); the entry `fixed` (an index, or None) is
    held, as the one CI coefficient CHAMP leaves out of the varied set."""
    S, g = sr_matrices(sums, energy)
    n = len(g)
    keep = np.array([k for k in range(n) if k != fixed])
    Sr = S[np.ix_(keep, keep)].copy()
    Sr[np.diag_indices_from(Sr)] *= 1.0 + adiag
    dp = np.zeros(n)
    dp[keep] = np.linalg.solve(Sr, -tau * g[keep])
    return dp


def sr_step(sums: dict, cdet: np.ndarray, energy: float, tau: float = 0.02, adiag: float = 0.01,
            fixed: int = 0) -> np.ndarray:
    """New CI coefficients after one SR step of length tau (sums over the
    CI coefficients alone)."""
    return np.array(cdet, float) + sr_delta(sums, energy, tau, adiag, fixed)


def sr_optimize(system, jd=None, ci: bool = False, nwalk: int = 256, iters: int = 5, nblock: int = 4,
                nstep: int = 10, tau: float = 0.02, adiag: float = 0.01, precision: str = "fp64",
                seed_offset: int = 0, engine_factory=None, orb=None):
    """SR optimisation loop over Jastrow (jasderiv selection `jd`), with
    `ci` CI parameters, and with `orb` (orbital pairs [n][2], 1-based, from
    orbital_opt.orb_terms) orbital rotations, as CHAMP's optwf driver runs
    it with method sr_n:
    per iteration nblock VMC blocks of nstep sweeps on the engine with the
    derivative sums on, one SR step over the joint vector (the reference CI
    coefficient held), new parameters (cusp-fixed e-e-n terms recomputed),
    walkers carried over to the next iteration's engine.  Returns the final
    system and per-iteration (energy, error) of the sampled wave function."""
    from . import jastrow_opt
    from .engine import Engine, initial_configs, rng_states
    make = engine_factory or (lambda s: Engine(s, precision=precision))
    rng = rng_states(seed_offset + nwalk)[seed_offset:].copy()
    x = initial_configs(system, rng)
    history = []
    for _ in range(iters):
        eng = make(system)
        try:
            eng.set_walkers(x, rng)
            P = jastrow_opt.param_map(system, jd) if jd is not None and jd.nparmj else None
            if orb is not None and len(orb):
                eng.opt_orb(orb)
            eng.opt_setup(ci=ci, jas_map=P, overlap=True)
            for _ in range(nblock):
                eng.vmc_steps(nstep)
                eng.end_block()
            r = eng.results()
            sums = eng.opt_sums(overlap=True)
            x, rng = eng.walkers()
        finally:
            eng.close()
        history.append((float(r["energy"]), float(r["err"])))
        nj = 0 if P is None else P.shape[1]
        dp = sr_delta(sums, float(r["energy"]), tau, adiag, fixed=nj if ci else None)
        if nj:
            system = jastrow_opt.apply_step(system, jd, dp[:nj])
        nc = len(system.cdet) if ci else 0
        if ci:
            system = copy.copy(system)
            system.cdet = np.array(system.cdet, float) + dp[nj:nj + nc]
            system._keep = []
        if orb is not None and len(orb):
            from . import orbital_opt
            system = orbital_opt.apply_step(system, orb, dp[nj + nc:])
    return system, history
