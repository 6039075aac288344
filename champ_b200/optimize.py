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
