"""Jastrow parameters of the wave-function optimisation (CHAMP ijas = 4).

The engine returns, per walker, the derivative of J (= ln psi_J) with
respect to every Jastrow coefficient taken on its own (the "raw" vector:
a part [nctype][norda+1], b part [nspin2b][nordb+1], c part
[nctype][nterms]).  CHAMP optimises a selection of them, read from the
``jasderiv`` block (nparma/iwjasa, nparmb/iwjasb, nparmc/iwjasc), and keeps
the e-e-n coefficients fixed by the cusp conditions dependent on the varied
ones.  Its per-walker parameter derivatives (deriv_jastrow4's gvalue, the
first nparmj entries of the SR vector sr_o) are a linear map of the raw
vector; this module builds that map:

* a and b parameters: gvalue(npointa(it)+jparm) is the raw a entry
  q = iwjasa(jparm, it) of type it (likewise b per spin class);
  vmc/deriv_jastrow4.f90:181-234, 588-640;
* c parameters: gvalue(npoint(it)+jparm) is the raw term iwjasc(jparm, it)
  plus, for every cusp-fixed term iwc4(jj), cdep(jj, id, it) times that
  term's raw value for each varied parameter it depends on
  (vmc/deriv_jastrow4.f90:392-466, dependencies from checkdepend4 in
  vmc/cuspinit4.f90:72-149).

After an optimisation step the varied coefficients change and the
dependent ones are recomputed from the cusp conditions (cuspexact4).
"""
from __future__ import annotations

import copy
import dataclasses

import numpy as np

from .system import cuspexact4, cuspinit4, nterms4


@dataclasses.dataclass
class JasDeriv:
    """Varied Jastrow parameters (CHAMP's jasderiv block), 1-based indices
    as in the input: iwjasa[it] lists q values of type it (1 = a(1),
    2 = a(2), q >= 3 the r^(q-1) coefficient), iwjasb[isb] the same for b,
    iwjasc[it] e-e-n term numbers of type it."""
    iwjasa: list
    iwjasb: list
    iwjasc: list

    @property
    def nparma(self):
        return [len(v) for v in self.iwjasa]

    @property
    def nparmb(self):
        return [len(v) for v in self.iwjasb]

    @property
    def nparmc(self):
        return [len(v) for v in self.iwjasc]

    @property
    def nparmj(self) -> int:
        return sum(self.nparma) + sum(self.nparmb) + sum(self.nparmc)


def read_jasderiv(text: str, nctype: int, nspin2b: int = 1) -> JasDeriv:
    """Parse CHAMP's jastrow-derivative file (read_jasderiv_file in
    vmc/read_data_parser.f90:1555-1690): lines before ``jasderiv`` are
    skipped; then the counts nparma(1..nctype) nparmb(1..nspin2b)
    nparmc(1..nctype) nparmf(1..nctype), one list of iwjasa per type, of
    iwjasb per spin class, of iwjasc per type.  Each list is a Fortran
    list-directed read: it takes as many records as its values need, and an
    empty list still consumes one record."""
    lines = [ln.split("#")[0].strip() for ln in text.splitlines()]
    try:
        k = next(i for i, ln in enumerate(lines) if ln.split()[:1] == ["jasderiv"]) + 1
    except StopIteration:
        raise ValueError("no jasderiv line") from None

    def read(n):
        nonlocal k
        if n == 0:
            k += 1
            return []
        vals = []
        while len(vals) < n:
            if k >= len(lines):
                raise ValueError("jasderiv: file ends inside a list")
            vals += [int(v) for v in lines[k].split()]
            k += 1
        if len(vals) != n:
            raise ValueError(f"jasderiv: expected {n} values, got {vals}")
        return vals

    counts = read(3 * nctype + nspin2b)
    na = counts[:nctype]
    nb = counts[nctype:nctype + nspin2b]
    nc = counts[nctype + nspin2b:2 * nctype + nspin2b]
    nf = counts[2 * nctype + nspin2b:]
    if any(nf):
        raise ValueError("nparmf > 0: the f-type Jastrow terms are not part of ijas = 4")
    iwa = [read(n) for n in na]
    iwb = [read(n) for n in nb]
    iwc = [read(n) for n in nc]
    return JasDeriv(iwa, iwb, iwc)


def raw_layout(system) -> dict:
    """Offsets and sizes of the raw vector's parts for `system`."""
    NA, NB, NT = system.norda + 1, system.nordb + 1, nterms4(system.nordc) if system.nordc > 1 else 0
    nct, nsb = system.nctype, int(getattr(system, "nspin2b", 1))
    return dict(NA=NA, NB=NB, NT=NT, a=0, b=nct * NA, c=nct * NA + nsb * NB,
                nraw=nct * NA + nsb * NB + nct * NT)


def checkdepend4(nordc: int, iwjasc) -> tuple:
    """Dependence of the cusp-fixed e-e-n terms on the varied ones
    (checkdepend4, vmc/cuspinit4.f90:72-149).  Returns (iwc4, deps) with
    deps[it][jj] = list of (jparm 0-based, cdep) for equation jj (1-based),
    and refuses a varied term that the cusp conditions fix."""
    d, iwc4, nt = cuspinit4(nordc)
    neqs = 2 * (nordc - 1)
    deps = []
    for it, varied in enumerate(iwjasc):
        dj = {jj: [] for jj in range(1, neqs + 1)}
        # every equation but the 2nd-order e-n one: direct dependence
        for i in range(1, neqs + 1):
            if i == nordc:
                continue
            for j in range(1, nt + 1):
                if abs(d[i, j]) > 1e-10:
                    for l, t in enumerate(varied):
                        if j == t:
                            if j == iwc4[i]:
                                raise ValueError("do not vary dep. variable")
                            dj[i].append([l, -d[i, j] / d[i, iwc4[i]]])
        # the 2nd-order e-n term depends on all the others, hence on every
        # varied term
        cd = [0.0] * len(varied)
        for i in range(1, neqs + 1):
            if i == nordc:
                continue
            factor = -d[nordc, iwc4[i]] / d[nordc, iwc4[nordc]]
            for j in range(1, nt + 1):
                for l, t in enumerate(varied):
                    if j == t:
                        cd[l] -= factor * (d[i, j] / d[i, iwc4[i]])
        dj[nordc] = [[l, cd[l]] for l in range(len(varied))]
        deps.append(dj)
    return iwc4, deps


def param_map(system, jd: JasDeriv) -> np.ndarray:
    """[nraw, nparmj] map from the raw derivatives to CHAMP's gvalue."""
    lay = raw_layout(system)
    nct, nsb = system.nctype, int(getattr(system, "nspin2b", 1))
    if len(jd.iwjasa) != nct or len(jd.iwjasc) != nct or len(jd.iwjasb) != nsb:
        raise ValueError("jasderiv lists do not match the system's centre types / spin classes")
    P = np.zeros((lay["nraw"], jd.nparmj))
    ip = 0
    for it in range(nct):                     # npointa(it) + jparm
        for q in jd.iwjasa[it]:
            if not 1 <= q <= lay["NA"]:
                raise ValueError(f"iwjasa value {q} outside 1..norda+1")
            P[lay["a"] + it * lay["NA"] + q - 1, ip] = 1.0
            ip += 1
    for isb in range(nsb):                    # iparma + offset of isb + jparm
        for q in jd.iwjasb[isb]:
            if not 1 <= q <= lay["NB"]:
                raise ValueError(f"iwjasb value {q} outside 1..nordb+1")
            P[lay["b"] + isb * lay["NB"] + q - 1, ip] = 1.0
            ip += 1
    if any(jd.nparmc):
        if system.nordc <= 1:
            raise ValueError("e-e-n parameters need nordc > 1")
        for it in range(nct):
            v = list(jd.iwjasc[it])
            if v != sorted(v) or len(set(v)) != len(v):
                raise ValueError("iwjasc must be strictly increasing")
            if any(not 1 <= t <= lay["NT"] for t in v):
                raise ValueError("iwjasc value outside 1..nterms")
        iwc4, deps = checkdepend4(system.nordc, jd.iwjasc)
        for it in range(nct):
            base = lay["c"] + it * lay["NT"]
            for l, t in enumerate(jd.iwjasc[it]):
                P[base + t - 1, ip + l] += 1.0
            for jj, lst in deps[it].items():
                for l, cd in lst:
                    P[base + iwc4[jj] - 1, ip + l] += cd
            ip += len(jd.iwjasc[it])
    return P


def apply_step(system, jd: JasDeriv, dp) -> object:
    """A copy of `system` with the varied Jastrow parameters moved by dp
    (in gvalue order) and the cusp-fixed e-e-n terms recomputed
    (cuspexact4)."""
    dp = np.asarray(dp, float)
    if dp.shape != (jd.nparmj,):
        raise ValueError(f"dp has shape {dp.shape}, expected ({jd.nparmj},)")
    out = copy.copy(system)
    a4 = np.array(system.a4, float).copy()
    b = np.array(system.b, float).copy()
    c = np.array(system.c, float).copy()
    ip = 0
    for it, lst in enumerate(jd.iwjasa):
        for q in lst:
            a4[it, q - 1] += dp[ip]
            ip += 1
    for isb, lst in enumerate(jd.iwjasb):
        for q in lst:
            b[isb, q - 1] += dp[ip]
            ip += 1
    for it, lst in enumerate(jd.iwjasc):
        for t in lst:
            c[it, t - 1] += dp[ip]
            ip += 1
    if any(jd.nparmc):
        cuspexact4(c, system.nordc)
    out.a4, out.b, out.c = a4, b, c
    out._keep = []
    return out


def default_jasderiv(system) -> JasDeriv:
    """Every free parameter of the system, as CHAMP's input checks allow
    them (read_jasderiv_file, vmc/read_data_parser.f90:1622-1660): the
    polynomial a terms of each type, and a(2) too for all-electron systems
    (with pseudopotentials a(1) and a(2) stay fixed); b(2) and the
    polynomial b terms (b(1) is fixed by the e-e cusp); every e-e-n term the
    cusp conditions leave free."""
    lay = raw_layout(system)
    nct, nsb = system.nctype, int(getattr(system, "nspin2b", 1))
    a_first = 3 if int(getattr(system, "nloc", 0)) > 0 else 2
    iwa = [list(range(a_first, lay["NA"] + 1)) for _ in range(nct)]
    iwb = [list(range(2, lay["NB"] + 1)) for _ in range(nsb)]
    if system.nordc > 1:
        _, iwc4, nt = cuspinit4(system.nordc)
        fixed = set(iwc4[1:])
        free = [t for t in range(1, nt + 1) if t not in fixed]
    else:
        free = []
    return JasDeriv(iwa, iwb, [list(free) for _ in range(nct)])
