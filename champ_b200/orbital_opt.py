"""Orbital-rotation parameters of the wave-function optimisation (ioptorb).

CHAMP varies each occupied orbital by mixing in other orbitals:
phi_io -> phi_io + a phi_jo.  Which pairs (io, jo) are varied is decided by
``optorb_define`` (vmc/optorb.f90:838-1030) from the determinant list, the
orbital symmetry labels, ``ncore``, ``nadorb`` (external orbitals beyond the
determinants' highest one) and ``no_active``; ``orb_terms`` restates its
rules.  The engine returns, per walker, d ln psi / d a of every pair
(cw_opt_orb / cw_orb_o, after the Jastrow and CI parts of the SR vector as
optwf_store lays it out); ``apply_step`` applies a parameter change to the
LCAO coefficients to first order, phi_io += a phi_jo.
"""
from __future__ import annotations

import copy

import numpy as np


def orb_terms(system, ncore: int = 0, nadorb: int = 0, irrep=None, no_active: int = 0) -> np.ndarray:
    """Varied orbital pairs, [nterm][2] 1-based (io, jo), in optorb_define's
    order (io outer, jo inner).

    Rules of vmc/optorb.f90:904-1010: io runs over ncore+1..ndetorb and is
    skipped when no determinant holds it; jo runs over
    ncore+1..ndetorb+nadorb (nadorb capped at the orbitals left in the
    coefficient matrix); a pair is omitted when io == jo, when the orbitals'
    symmetry labels differ, when both are doubly occupied in every
    determinant, with no_active when io is partly occupied and jo is held by
    some determinant, and when no determinant of either spin holds io
    without jo.  irrep: per-orbital symmetry labels (None: all equal)."""
    iworbd = np.asarray(system.iworbd, int)
    ndet, nelec = iworbd.shape
    nup = system.nup
    norb = int(np.asarray(system.coef).shape[0])
    ndetorb = int(iworbd.max())
    nadorb = min(nadorb, norb - ndetorb)
    ntot = ndetorb + nadorb
    # iflag1: 0 when doubly occupied in every determinant; iflag2: held by some determinant
    iflag1 = np.ones(ntot + 1, int)
    iflag2 = np.zeros(ntot + 1, int)
    for i in range(1, ndetorb + 1):
        iflag1[i] = 0 if all(int(np.sum(iworbd[k] == i)) == 2 for k in range(ndet)) else 1
        iflag2[i] = 1 if np.any(iworbd == i) else 0
    lab = (lambda o: 0) if irrep is None else (lambda o: irrep[o - 1])
    spins = [(0, nup), (nup, nelec)]
    terms = []
    for io in range(ncore + 1, ndetorb + 1):
        if iflag2[io] == 0:
            continue
        for jo in range(ncore + 1, ntot + 1):
            if io == jo or lab(io) != lab(jo):
                continue
            if iflag1[io] == 0 and iflag1[jo] == 0:
                continue
            if no_active and iflag1[io] != 0 and iflag2[jo] != 0:
                continue
            m = 0
            for a, b in spins:
                for k in range(ndet):
                    occ = iworbd[k, a:b]
                    if np.any(occ == io) and not np.any(occ == jo):
                        m += 1
            if m:
                terms.append((io, jo))
    return np.array(terms, np.int32).reshape(-1, 2)


def apply_step(system, terms, da):
    """New system with phi_io += da_t phi_jo for every pair t (first order
    in the step, the coefficients of the pairs' orbitals taken before the
    step)."""
    s = copy.copy(system)
    coef = np.array(system.coef, float)
    new = coef.copy()
    for (io, jo), a in zip(np.asarray(terms, int), np.asarray(da, float)):
        new[io - 1] += a * coef[jo - 1]
    s.coef = new
    s._keep = []
    return s
