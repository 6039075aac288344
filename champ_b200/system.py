"""Molecular systems for the walker engine.

``System`` holds the contents of CHAMP's modules after ``parser()`` for one
molecule, laid out as in ``cw_system_desc`` (C order == Fortran order
reversed).  The set-up steps CHAMP performs while reading its input are
restated here because every engine input passes through them:

* ``prepare_radial``  — read_bas_num (vmc/read_bas_num.f90:11-247): small-r
  polynomial fit, cutoff radius, large-r exponential fit (fitting.f90
  exp_fit), cubic-spline second derivatives (vmc/spline2.f90:3);
* ``tabulate_gaussians`` — the numerical-grid tabulation of contracted
  Gaussians of CHAMP's converter (tools/trex_tools/trex2champ.py:560-760:
  grid type 3, 2000 points, arg 1.003, r0 20, gnorm normalisation);
* ``cuspexact4`` — e-e-n cusp conditions (vmc/cuspinit4.f90:3,
  vmc/cuspexact4.f90:3);
* ``gesqua`` — the angular quadrature (vmc/rotqua.f90:3);
* ``pot_nn`` — nuclear repulsion.

``make_synthetic`` builds the seeded synthetic molecules the benchmarks run
on (no public data set is involved).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .abi import CW_MGAUSS, CW_MPS_L, CW_NCOEF, CwSystemDesc, dptr, iptr

# ---------------------------------------------------------------------------
# CHAMP set-up restatements
# ---------------------------------------------------------------------------


def spline2(x, y, yp1, ypn):
    """spline2 (vmc/spline2.f90:3): second derivatives of the cubic spline."""
    n = len(x)
    y2 = np.zeros(n)
    work = np.zeros(n)
    if yp1 > 1e30:
        y2[0] = 0.0
        work[0] = 0.0
    else:
        y2[0] = -0.5
        work[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1)
    for i in range(1, n - 1):
        sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1])
        p = sig * y2[i - 1] + 2.0
        y2[i] = (sig - 1.0) / p
        work[i] = (6.0 * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1])
                          / (x[i] - x[i - 1])) / (x[i + 1] - x[i - 1]) - sig * work[i - 1]) / p
    if ypn > 1e30:
        qn = 0.0
        workn = 0.0
    else:
        qn = 0.5
        workn = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]))
    y2[n - 1] = (workn - qn * work[n - 2]) / (qn * y2[n - 2] + 1.0)
    for k in range(n - 2, -1, -1):
        y2[k] = y2[k] * y2[k + 1] + work[k]
    return y2


def exp_fit(x, y):
    """exp_fit (vmc/fitting.f90:11): least squares of log|y| = A - b x."""
    n = len(x)
    w = np.log(np.abs(y))
    x_sum = float(np.sum(x))
    w_sum = float(np.sum(w))
    xw_sum = float(np.sum(x * w))
    xx_sum = float(np.sum(x * x))
    x_mean, w_mean = x_sum / n, w_sum / n
    denom = xx_sum - n * x_mean * x_mean
    b = (n * x_mean * w_mean - xw_sum) / denom
    a = math.exp((w_mean * xx_sum - x_mean * xw_sum) / denom)
    return a, b


def prepare_radial(x, rwf_cols, igrid, arg, r0_in, znuc, nloc, lvals=None, icusp=0):
    """read_bas_num (vmc/read_bas_num.f90:11-247) for one atom type.

    x: grid as read from the basis file, rwf_cols: (nrbas, nr) values.
    Returns dict(arg, r0, rwf, d2rwf, ce, ae, rmaxwf).
    """
    nr = len(x)
    nrbas = rwf_cols.shape[0]
    if igrid == 2 and arg <= 1.0:
        arg = x[1] / x[0]
    r0 = r0_in
    if igrid == 3:
        r0 = r0_in / (arg ** (nr - 1) - 1.0)
    cutoff_rmax = 1.0e-12
    ce = np.zeros((nrbas, CW_NCOEF))
    ae = np.zeros((nrbas, 2))
    rmaxwf = np.zeros(nrbas)
    d2 = np.zeros((nrbas, nr))
    for irb in range(nrbas):
        y = rwf_cols[irb]
        if nloc == 0 and lvals is not None and lvals[irb] == 0 and icusp == 1:
            n1 = CW_NCOEF - 1
            A = np.zeros((n1, n1))
            A[:, 0] = 1.0 - znuc * x[:n1]
            for jj in range(2, CW_NCOEF):
                A[:, jj - 1] = x[:n1] ** jj
            sol = np.linalg.solve(A, y[:n1].copy())
            ce[irb, 0] = sol[0]
            ce[irb, 1] = -znuc * sol[0]
            ce[irb, 2:5] = sol[1:4]
        else:
            A = np.array([[x[ii] ** jj for jj in range(CW_NCOEF)] for ii in range(CW_NCOEF)])
            ce[irb] = np.linalg.solve(A, y[:CW_NCOEF].copy())
        dwf1 = 0.0
        for icoef in range(2, CW_NCOEF + 1):
            dwf1 += (icoef - 1) * ce[irb, icoef - 1] * (x[0] ** (icoef - 2))
        rmax = x[nr - 1]
        for ir in range(nr - 1, -1, -1):
            if abs(y[ir]) > cutoff_rmax:
                rmax = x[ir]
                break
        if abs(rmax - x[nr - 1]) < 1.0e-10:
            a, b = exp_fit(x[nr - 10:], y[nr - 10:])
            if b < 0:
                raise ValueError("BASIS_READ_NUM: ak<0")
            ae[irb] = (a, b)
            rmax = -math.log(cutoff_rmax / abs(a)) / b
            dwfn = -b * a * math.exp(-b * x[nr - 1])
        else:
            dwfn = 0.0
        rmaxwf[irb] = rmax
        d2[irb] = spline2(x, y, dwf1, dwfn)
    return dict(arg=arg, r0=r0, rwf=rwf_cols.copy(), d2rwf=d2, ce=ce, ae=ae, rmaxwf=rmaxwf)


def gnorm(alp, l):
    """Normalisation of a primitive Gaussian (trex2champ.py write_champ_file_basis_grid)."""
    if l == 0:
        return (2.0 * alp) ** (3.0 / 4.0) * 2.0 * (1.0 / (np.pi ** (1.0 / 4.0)))
    if l == 1:
        return (2.0 * alp) ** (5.0 / 4.0) * np.sqrt(8.0 / 3.0) * (1.0 / (np.pi ** (1.0 / 4.0)))
    if l == 2:
        return (2.0 * alp) ** (7.0 / 4.0) * np.sqrt(16.0 / 15.0) * (1.0 / (np.pi ** (1.0 / 4.0)))
    if l == 3:
        return (2.0 * alp) ** (9.0 / 4.0) * np.sqrt(32.0 / 105.0) * (1.0 / (np.pi ** (1.0 / 4.0)))
    if l == 4:
        return (2.0 * alp) ** (11.0 / 4.0) * np.sqrt(64.0 / 945.0) * (1.0 / (np.pi ** (1.0 / 4.0)))
    return 1.0


GRID_TYPE, GRID_POINTS, GRID_ARG, GRID_R0 = 3, 2000, 1.003, 20.0


def _round12(a):
    # the converter writes ' %.12e'; CHAMP reads those rounded values back
    return np.array([float(f"{v:.12e}") for v in np.ravel(a)]).reshape(np.shape(a))


def tabulate_gaussians(shells):
    """Radial grid file contents for one atom type.

    shells: list of (l, exponents, coefficients).  Returns (x, rwf[nshell, nr])
    rounded as the converter writes them.
    """
    r0 = GRID_R0 / (GRID_ARG ** (GRID_POINTS - 1) - 1)
    i = np.arange(GRID_POINTS)
    x = r0 * GRID_ARG ** i - r0
    r2 = x * x
    rwf = np.zeros((len(shells), GRID_POINTS))
    for s, (l, ex, co) in enumerate(shells):
        v = np.zeros(GRID_POINTS)
        for e, c in zip(ex, co):
            v += gnorm(e, l) * c * np.exp(-e * r2)
        rwf[s] = v
    return _round12(x), _round12(rwf)


def nterms4(nord):
    i = 0
    for n in range(2, nord + 1):
        for k in range(n - 1, -1, -1):
            l_hi = n - k - 2 if k == 0 else n - k
            for l in range(l_hi, -1, -1):
                m = (n - k - l) // 2
                if 2 * m == n - k - l:
                    i += 1
    return i


def cuspinit4(nordc):
    """cuspinit4 (vmc/cuspinit4.f90:3): constraint matrix d and fixed terms iwc4."""
    nt = nterms4(nordc)
    neq = 2 * (nordc - 1)
    d = np.zeros((neq + 1, nt + 1))  # 1-based
    iwc4 = [0] * (neq + 1)
    i = 0
    for n in range(2, nordc + 1):
        for k in range(n - 1, -1, -1):
            l_hi = n - k - 2 if k == 0 else n - k
            for l in range(l_hi, -1, -1):
                m = (n - k - l) // 2
                if 2 * m == n - k - l:
                    i += 1
                    if k == 1 and iwc4[n - 1] == 0:
                        iwc4[n - 1] = i
                    if k == 0 and iwc4[n + nordc - 2] == 0:
                        iwc4[n + nordc - 2] = i
                    iord = l + 2 * m
                    d[iord, i] -= 2 * k
                    if l + m > 0:
                        d[nordc - 1 + k + m, i] -= (l + m)
                    if m > 0:
                        d[nordc - 1 + k + l + m, i] -= m
    return d, iwc4, nt


def cuspexact4(c, nordc):
    """cuspexact4 (vmc/cuspexact4.f90:3) applied to c[nctype, nterms] in place."""
    if nordc <= 1:
        return c
    d, iwc4, nt = cuspinit4(nordc)
    cc = np.zeros(nt + 1)
    order = list(range(1, nordc)) + list(range(nordc + 1, 2 * (nordc - 1) + 1)) + [nordc]
    for it in range(c.shape[0]):
        cc[1:] = c[it]
        for i in order:
            s = 0.0
            for j in range(1, nt + 1):
                if j != iwc4[i]:
                    s += d[i, j] * cc[j]
            cc[iwc4[i]] = -s / d[i, iwc4[i]]
        c[it] = cc[1:]
    return c


def gesqua(nq):
    """gesqua (vmc/rotqua.f90:3) for the tetrahedron (4) and octahedron (6) rules."""
    if nq == 4:
        q = 1.0 / math.sqrt(3.0)
        xq = np.array([q, q, -q, -q])
        yq = np.array([q, -q, q, -q])
        zq = np.array([q, -q, -q, q])
        return xq, yq, zq, np.full(4, 0.25)
    if nq != 6:
        raise ValueError("only nquad 4 or 6 are generated here")
    xq = np.array([1.0, -1.0, 0, 0, 0, 0])
    yq = np.array([0, 0, 1.0, -1.0, 0, 0])
    zq = np.array([0, 0, 0, 0, 1.0, -1.0])
    return xq, yq, zq, np.full(6, 1.0 / 6.0)


def pot_nn(cent, znuc, iwctype):
    pe = 0.0
    for i in range(1, len(cent)):
        for j in range(i):
            r = math.sqrt(sum((cent[i][k] - cent[j][k]) ** 2 for k in range(3)))
            pe += znuc[iwctype[i]] * znuc[iwctype[j]] / r
    return pe


# ---------------------------------------------------------------------------
# System container
# ---------------------------------------------------------------------------

# Slm index sets per shell type (vmc/slm.f90 table)
SLM_OF_L = {0: [1], 1: [2, 3, 4], 2: [5, 6, 7, 8, 9, 10], 3: list(range(11, 21)), 4: list(range(21, 36))}


@dataclass
class System:
    name: str
    nelec: int
    nup: int
    iwctype: np.ndarray
    cent: np.ndarray
    znuc: np.ndarray
    # numerical basis per type
    nrbas: np.ndarray
    igrid: np.ndarray
    nr: np.ndarray
    arg: np.ndarray
    r0: np.ndarray
    rwf: np.ndarray
    d2rwf: np.ndarray
    ce: np.ndarray
    ae: np.ndarray
    rmaxwf: np.ndarray
    nbastyp: np.ndarray
    iwlbas: np.ndarray
    iwrwf: np.ndarray
    coef: np.ndarray      # [norb, nbasis]
    iworbd: np.ndarray    # [ndet, nelec]
    cdet: np.ndarray
    norda: int
    nordb: int
    nordc: int
    scalek: float
    a4: np.ndarray
    b: np.ndarray
    c: np.ndarray
    isc: int = 2
    nspin2b: int = 1
    nocuspb: int = 0
    nloc: int = 0
    lpot: np.ndarray | None = None
    necp_term: np.ndarray | None = None
    necp_power: np.ndarray | None = None
    ecp_exponent: np.ndarray | None = None
    ecp_coef: np.ndarray | None = None
    nquad: int = 0
    xq0: np.ndarray | None = None
    yq0: np.ndarray | None = None
    zq0: np.ndarray | None = None
    wq: np.ndarray | None = None
    deltar: float = 5.0
    deltat: float = 1.0
    fbias: float = 1.0
    # several states sharing orbitals and Jastrow: [nstates][ndet] CI vectors
    # (row 0 = cdet), guiding flag and weights
    cdet_states: np.ndarray | None = None
    iguiding: int = 0
    weights_g: np.ndarray | None = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def nstates(self):
        return 1 if self.cdet_states is None else int(np.asarray(self.cdet_states).shape[0])

    @property
    def ncent(self):
        return len(self.iwctype)

    @property
    def nctype(self):
        return len(self.znuc)

    @property
    def ndn(self):
        return self.nelec - self.nup

    @property
    def nbasis(self):
        return self.coef.shape[1]

    @property
    def norb(self):
        return self.coef.shape[0]

    @property
    def pecent(self):
        return pot_nn(self.cent, self.znuc, self.iwctype)

    def desc(self) -> CwSystemDesc:
        """ctypes cw_system_desc pointing at this object's arrays."""
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        keep = []

        def D(a):
            a = f64(a)
            keep.append(a)
            return dptr(a)

        def I(a):
            a = i32(a)
            keep.append(a)
            return iptr(a)

        d = CwSystemDesc()
        d.nelec, d.nup, d.ncent, d.nctype = self.nelec, self.nup, self.ncent, self.nctype
        d.iwctype, d.cent, d.znuc = I(self.iwctype), D(self.cent), D(self.znuc)
        d.pecent = self.pecent
        d.mrwf, d.mrwf_pts = self.rwf.shape[1], self.rwf.shape[2]
        d.nrbas, d.igrid, d.nr = I(self.nrbas), I(self.igrid), I(self.nr)
        d.arg, d.r0 = D(self.arg), D(self.r0)
        d.rwf, d.d2rwf, d.ce, d.ae, d.rmaxwf = (D(self.rwf), D(self.d2rwf), D(self.ce), D(self.ae),
                                               D(self.rmaxwf))
        d.mbastyp = self.iwlbas.shape[1]
        d.nbastyp, d.iwlbas, d.iwrwf = I(self.nbastyp), I(self.iwlbas), I(self.iwrwf)
        d.nbasis, d.norb = self.nbasis, self.norb
        d.coef = D(self.coef)
        d.ndet = len(self.cdet)
        d.iworbd = I(self.iworbd)
        cst = getattr(self, "cdet_states", None)
        if cst is not None and len(cst) > 1:
            cst = np.asarray(cst, float)
            if cst.shape[1] != d.ndet or not np.array_equal(cst[0], np.asarray(self.cdet, float)):
                raise ValueError("cdet_states must be [nstates][ndet] with state 1 equal to cdet")
            d.cdet, d.nstates = D(cst), cst.shape[0]
            d.iguiding = int(getattr(self, "iguiding", 0))
            wg = getattr(self, "weights_g", None)
            d.weights_g = D(wg if wg is not None else np.ones(cst.shape[0]))
        else:
            d.cdet, d.nstates = D(self.cdet), 1
        d.norda, d.nordb, d.nordc = self.norda, self.nordb, self.nordc
        d.isc, d.nspin2b, d.nocuspb = self.isc, self.nspin2b, self.nocuspb
        d.scalek = self.scalek
        d.a4, d.b = D(self.a4), D(self.b)
        d.c = D(self.c if self.c.size else np.zeros(1))
        d.nloc = self.nloc
        if self.nloc > 0:
            d.lpot, d.necp_term, d.necp_power = I(self.lpot), I(self.necp_term), I(self.necp_power)
            d.ecp_exponent, d.ecp_coef = D(self.ecp_exponent), D(self.ecp_coef)
            d.nquad = self.nquad
            d.xq0, d.yq0, d.zq0, d.wq = D(self.xq0), D(self.yq0), D(self.zq0), D(self.wq)
        else:
            d.nquad = 0
        d.deltar, d.deltat, d.fbias = self.deltar, self.deltat, self.fbias
        self._keep = keep
        return d


def assemble_basis(types):
    """Pack per-type radial tables into the padded arrays of cw_system_desc.

    types: list of dicts with keys x, rwf (nrbas, nr), shells_l (per radial
    function, its l), aos: list of (slm, irb) and prepared radial data.
    """
    nct = len(types)
    mrwf = max(t["prep"]["rwf"].shape[0] for t in types)
    mpts = max(t["prep"]["rwf"].shape[1] for t in types)
    mbas = max(len(t["aos"]) for t in types)
    rwf = np.zeros((nct, mrwf, mpts))
    d2 = np.zeros((nct, mrwf, mpts))
    ce = np.zeros((nct, mrwf, CW_NCOEF))
    ae = np.zeros((nct, mrwf, 2))
    rmax = np.zeros((nct, mrwf))
    iwl = np.zeros((nct, mbas), np.int32)
    iwr = np.zeros((nct, mbas), np.int32)
    for it, t in enumerate(types):
        p = t["prep"]
        n, npt = p["rwf"].shape
        rwf[it, :n, :npt] = p["rwf"]
        d2[it, :n, :npt] = p["d2rwf"]
        ce[it, :n] = p["ce"]
        ae[it, :n] = p["ae"]
        rmax[it, :n] = p["rmaxwf"]
        for ib, (slm, irb) in enumerate(t["aos"]):
            iwl[it, ib] = slm
            iwr[it, ib] = irb
    return dict(
        nrbas=np.array([t["prep"]["rwf"].shape[0] for t in types], np.int32),
        igrid=np.array([t["igrid"] for t in types], np.int32),
        nr=np.array([t["prep"]["rwf"].shape[1] for t in types], np.int32),
        arg=np.array([t["prep"]["arg"] for t in types]),
        r0=np.array([t["prep"]["r0"] for t in types]),
        rwf=rwf, d2rwf=d2, ce=ce, ae=ae, rmaxwf=rmax,
        nbastyp=np.array([len(t["aos"]) for t in types], np.int32), iwlbas=iwl, iwrwf=iwr)


# ---------------------------------------------------------------------------
# Seeded synthetic systems
# ---------------------------------------------------------------------------

def _random_shells(rng, spec, ranges=None):
    """spec: list of (l, count); 3 primitives per shell, exponents log-uniform
    in [0.1, 20], or in ranges[l] = (lo, hi) when given."""
    shells = []
    for l, cnt in spec:
        lo, hi = ranges[l] if ranges else (0.1, 20.0)
        for _ in range(cnt):
            ex = np.exp(rng.uniform(np.log(lo), np.log(hi), size=3))
            co = rng.uniform(0.2, 1.0, size=3)
            shells.append((l, ex, co))
    return shells


def _type_from_shells(shells, znuc, nloc):
    x, rwf = tabulate_gaussians(shells)
    prep = prepare_radial(x, rwf, GRID_TYPE, GRID_ARG, GRID_R0, znuc, nloc)
    aos = []
    for irb, (l, _, _) in enumerate(shells):
        for slm in SLM_OF_L[l]:
            aos.append((slm, irb + 1))
    return dict(prep=prep, aos=aos, igrid=GRID_TYPE, shells=shells)


def _bfd_like_ecp(rng, zval, lpot):
    """Seeded BFD-form semilocal ECP: local channel removes the -Z/r singularity."""
    nterm = np.zeros(CW_MPS_L, np.int32)
    power = np.zeros((CW_MPS_L, CW_MGAUSS), np.int32)
    expo = np.zeros((CW_MPS_L, CW_MGAUSS))
    coef = np.zeros((CW_MPS_L, CW_MGAUSS))
    if lpot == 1:  # zero-coefficient local term (bare Coulomb atom)
        nterm[0] = 1
        power[0, 0] = 2
        expo[0, 0] = 1.0
        coef[0, 0] = 0.0
        return nterm, power, expo, coef
    f = lambda v: v * rng.uniform(0.8, 1.2)
    # local channel stored at index lpot-1 (CHAMP idx=lpot)
    a1 = f(8.36)
    loc = lpot - 1
    nterm[loc] = 3
    power[loc, :3] = (1, 3, 2)
    expo[loc, :3] = (a1, f(4.48), f(3.94))
    coef[loc, :3] = (zval, zval * a1, -f(19.2))
    # nonlocal channels l = 0 .. lpot-2 stored at index l
    for l in range(lpot - 1):
        nterm[l] = 1
        power[l, 0] = 2
        expo[l, 0] = f(5.03)
        coef[l, 0] = f(22.6)
    return nterm, power, expo, coef


def _jastrow(rng, nctype, cusp_a1, nord=5):
    a4 = rng.normal(0.0, 0.05, size=(nctype, nord + 1))
    a4[:, 0] = cusp_a1
    b = rng.normal(0.0, 0.05, size=(1, nord + 1))
    b[0, 0] = 0.5
    nt = nterms4(nord)
    c = rng.normal(0.0, 0.05, size=(nctype, nt))
    cuspexact4(c, nord)
    return a4, b, c


def _orthonormal(rng, k, o):
    q, _ = np.linalg.qr(rng.normal(size=(k, o)))
    return np.ascontiguousarray(q.T)  # [norb, nbasis]


# Exponent (bohr^-2) of the Gaussian model density that screens a nucleus in
# the model Hamiltonian of the trial orbitals (trial.py), unless a type sets
# its own ("screen"): a valence cloud of mean radius about 1.3 bohr.
SCREEN_ALPHA = 0.75


def model_hamiltonian_orbitals(cent, types_of_centre, type_defs, norb, ecp=None):
    """Lowest `norb` orbitals of the seeded molecule's model one-electron
    Hamiltonian (champ_b200.trial): kinetic energy, screened nuclear
    attraction and pseudopotential, in the molecule's Gaussian basis."""
    from . import trial
    shells = [td["basis"]["shells"] for td in type_defs]
    aos = [td["basis"]["aos"] for td in type_defs]
    prim, basis = trial.primitives(np.asarray(cent, float), types_of_centre, shells, aos, gnorm)
    S, T = trial.overlap_kinetic(prim, len(basis["ao_cent"]))
    znuc = np.array([td["z"] for td in type_defs], float)
    V = trial.potential_matrix(basis, np.asarray(cent, float), types_of_centre, znuc, ecp,
                               [td.get("screen", SCREEN_ALPHA) for td in type_defs])
    coef, _ = trial.model_orbitals(S, T + V, norb)
    return coef, basis


def determinant_scale(system, basis, nconf=8, seed=12345):
    """A constant c for the LCAO coefficients of `system` such that the
    Slater determinants at its start configurations are of order one.

    psi_D is defined up to a constant factor, and every determinant of an
    expansion holds the same number of electrons of each spin, so scaling
    every orbital by c scales psi_D by c^nelec and leaves ratios, drifts,
    local energies and the walk unchanged.  Unscaled, the determinants of
    large molecules (100 electrons of a spin) fall below the smallest FP64
    number and psi_D underflows to zero.  c is exp(-median(ln|det|)/n) over
    nconf start configurations of CHAMP's sites rule (cw_sites, a host-side
    routine of the engine library) drawn from a private stream."""
    from . import trial
    from .engine import initial_configs, rng_states
    coef = np.asarray(system.coef, float)
    rng = rng_states(nconf, cseed=str(seed).rjust(32, "1"))
    x = initial_configs(system, rng)
    logs = []
    for k in range(nconf):
        for n, e0 in ((system.nup, 0), (system.ndn, system.nup)):
            if n == 0:
                continue
            A = trial.ao_values(basis, np.arange(coef.shape[1]), x[k, e0:e0 + n]) @ coef[np.asarray(system.iworbd[0][e0:e0 + n]) - 1].T
            sgn, lg = np.linalg.slogdet(A)
            if sgn != 0:
                logs.append(lg / n)
    return float(np.exp(-np.median(logs))) if logs else 1.0


def _assemble(name, rng, cent, types_of_centre, type_defs, nelec, nup, norb, nocc_up, nocc_dn,
              nloc=4, nquad=6, orbitals="random"):
    nct = len(type_defs)
    basis = assemble_basis([td["basis"] for td in type_defs])
    nbasis = int(sum(len(type_defs[t]["basis"]["aos"]) for t in types_of_centre))
    znuc = np.array([td["z"] for td in type_defs], float)
    coef = _orthonormal(rng, nbasis, norb)   # drawn in every case: the seeded stream stays the same
    iworbd = np.array([list(range(1, nocc_up + 1)) + list(range(1, nocc_dn + 1))], np.int32)
    a4, b, c = _jastrow(rng, nct, np.array([td["a1"] for td in type_defs]))
    sysd = dict(name=name, nelec=nelec, nup=nup, iwctype=np.array(types_of_centre, np.int32),
                cent=np.asarray(cent, float), znuc=znuc, coef=coef, iworbd=iworbd,
                cdet=np.array([1.0]), norda=5, nordb=5, nordc=5, scalek=0.6, a4=a4, b=b, c=c,
                **basis)
    if nloc:
        lpot = np.array([td["lpot"] for td in type_defs], np.int32)
        nterm = np.zeros((nct, CW_MPS_L), np.int32)
        power = np.zeros((nct, CW_MPS_L, CW_MGAUSS), np.int32)
        expo = np.zeros((nct, CW_MPS_L, CW_MGAUSS))
        ecoef = np.zeros((nct, CW_MPS_L, CW_MGAUSS))
        for it, td in enumerate(type_defs):
            nterm[it], power[it], expo[it], ecoef[it] = _bfd_like_ecp(rng, td["z"], td["lpot"])
        xq, yq, zq, wq = gesqua(nquad)
        sysd.update(nloc=nloc, lpot=lpot, necp_term=nterm, necp_power=power, ecp_exponent=expo,
                    ecp_coef=ecoef, nquad=nquad, xq0=xq, yq0=yq, zq0=zq, wq=wq)
    if orbitals == "model":
        ecp = None
        if nloc:
            ecp = [(lpot[it], nterm[it], power[it], expo[it], ecoef[it]) for it in range(nct)]
        coef, basis_desc = model_hamiltonian_orbitals(cent, types_of_centre, type_defs, norb, ecp)
        sysd["coef"] = coef
        sysm = System(**sysd)
        sysm.coef = coef * determinant_scale(sysm, basis_desc)
        return sysm
    return System(**sysd)


_MADE = {}


def _memo(key, make):
    """Generated molecules are deterministic: build each once per process and
    hand out copies (callers may modify theirs)."""
    import copy
    if key not in _MADE:
        _MADE[key] = make()
    return copy.deepcopy(_MADE[key])


def make_synthetic(config: str, seed: int = 20261203, orbitals: str = "model") -> System:
    """Seeded synthetic molecule of one benchmark configuration (built once
    per process, a copy returned).

    c0: 3 nuclei in a 4 bohr box (Z 6/1/1, ECP on the heavy atom, l_max=1,
        6-point quadrature), 8 electrons (4/4), 60 Gaussians (s/p/d,
        exponents log-uniform 0.1-20), 4 orbitals, order-5 Jastrow.
    c1: 30 nuclei on a zig-zag chain alternating Cl-like (Z=7, ECP with s
        and p channels) and H-like (Z=1) centres, neutral: 120 electrons
        (60/60), 540 Gaussians (valence exponent ranges), 60 orbitals.
    tiny: 2 nuclei, 6 electrons, small basis (fast parity cases).
    c2: 12 nuclei, 40 electrons, 300 Gaussians, 80 orbitals, 10^4
        determinants (multideterminant DMC).
    he: He atom through the ECP path (DMC reaches the exact energy).

    c1, c2: orbitals of the molecule's model one-electron Hamiltonian
    (orbitals="model", trial.py); orbitals="random" gives a seeded random
    orthonormal coefficient matrix instead (c0 and tiny always use that).
    """
    return _memo(("synthetic", config, seed, orbitals), lambda: _make_synthetic(config, seed, orbitals))


def _make_synthetic(config, seed, orbitals):
    rng = np.random.default_rng(seed)
    if config == "c0":
        while True:
            cent = rng.uniform(-2.0, 2.0, size=(3, 3))
            dmin = min(np.linalg.norm(cent[i] - cent[j]) for i in range(3) for j in range(i))
            if dmin > 1.2:
                break
        heavy = dict(z=6.0, lpot=2, a1=0.0,
                     basis=_type_from_shells(_random_shells(rng, [(0, 4), (1, 4), (2, 2)]), 6.0, 4))
        hyd = dict(z=1.0, lpot=1, a1=-1.0,
                   basis=_type_from_shells(_random_shells(rng, [(0, 4), (1, 4)]), 1.0, 4))
        return _assemble("c0", rng, cent, [0, 1, 1], [heavy, hyd], 8, 4, 4, 4, 4)
    if config == "c1":
        return _chain_molecule(rng, "c1", 30, 120, orbitals)
    if config == "tiny":
        cent = np.array([[0.0, 0.0, -0.7], [0.3, 0.2, 0.8]])
        heavy = dict(z=4.0, lpot=2, a1=0.0,
                     basis=_type_from_shells(_random_shells(rng, [(0, 3), (1, 2), (2, 1)]), 4.0, 4))
        hyd = dict(z=1.0, lpot=1, a1=-1.0,
                   basis=_type_from_shells(_random_shells(rng, [(0, 2), (1, 1)]), 1.0, 4))
        return _assemble("tiny", rng, cent, [0, 1], [heavy, hyd], 5, 3, 4, 3, 2)
    if config == "he":
        return _helium()
    if config == "c2":
        return _c2(rng, orbitals)
    raise ValueError(f"unknown synthetic config {config!r}")


# Exponent ranges (bohr^-2) of the chain molecules' valence basis: s and p
# down to diffuse 0.08, up to 6 (s) and 4 (p); one d shell between 0.3 and
# 1.5 -- the span of pseudopotential valence basis sets, without the steep
# core-like functions that a pseudopotential makes unnecessary.
VALENCE_RANGES = {0: (0.08, 6.0), 1: (0.08, 4.0), 2: (0.3, 1.5)}


def _chain_molecule(rng, name, nat, nelec, orbitals):
    """Zig-zag chain of nat centres alternating Cl-like heavy atoms (valence
    charge 7, BFD-form pseudopotential with a local, an s and a p channel,
    s4 p4 d1 basis = 22 Cartesian AOs) and H-like atoms (charge 1, s2 p4 =
    14 AOs), valence basis exponents (VALENCE_RANGES), 2.0 bohr apart along x
    and 1.2 bohr across, nelec electrons (ceil/floor halves), one occupied
    orbital per up electron.  With nelec = 4 nat the molecule is neutral (a
    chain of HCl-like units)."""
    cent = np.zeros((nat, 3))
    for i in range(nat):
        cent[i] = (2.0 * i + rng.normal(0, 0.05), 1.2 * (i % 2) + rng.normal(0, 0.05), rng.normal(0, 0.05))
    heavy = dict(z=7.0, lpot=3, a1=0.0, screen=0.5,
                 basis=_type_from_shells(_random_shells(rng, [(0, 4), (1, 4), (2, 1)], VALENCE_RANGES), 7.0, 4))
    hyd = dict(z=1.0, lpot=1, a1=-1.0, screen=0.5,
               basis=_type_from_shells(_random_shells(rng, [(0, 2), (1, 4)], VALENCE_RANGES), 1.0, 4))
    types = [0 if i % 2 == 0 else 1 for i in range(nat)]
    nup, ndn = (nelec + 1) // 2, nelec // 2
    return _assemble(name, rng, cent, types, [heavy, hyd], nelec, nup, nup, nup, ndn, orbitals=orbitals)


def make_chain(nelec: int, seed: int, orbitals: str = "model") -> System:
    """Seeded chain molecule of the batched / serving job distribution:
    about nelec/4 centres of the c1 chain's two atom types (so about
    neutral), nelec electrons, basis about 4.5 x nelec Gaussians."""
    if nelec < 2:
        raise ValueError("a chain job needs at least 2 electrons")
    return _memo(("chain", nelec, seed, orbitals), lambda: _chain_molecule(
        np.random.default_rng(seed), f"chain{nelec}", max(2, int(round(nelec / 4))), nelec, orbitals))


def ci_expansion(rng, nup, ndn, norb, ndet, pools=(150, 500, 300, 120), nact_occ=8, nact_virt=30,
                 level_p=(0.1, 0.45, 0.3, 0.15)):
    """Seeded CI expansion of single to quadruple excitations of the aufbau
    reference (orbitals 1..nup / 1..ndn).

    Spin strings come from per-level pools (excitations from the top
    nact_occ occupied slots into the lowest nact_virt virtual orbitals), as
    selected-CI expansions reuse spin strings; each determinant pairs an up
    and a down string whose levels add up to 1..4.  Coefficients decay as
    |c_k| = k**-1.5 with random signs, c_1 = 1 for the reference.
    Returns (iworbd [ndet][nup+ndn] 1-based, cdet [ndet]).
    """
    def pool(nel, lev, size):
        out, seen = [], set()
        occ_slots = list(range(max(0, nel - nact_occ), nel))
        virt = list(range(nel + 1, min(norb, nel + nact_virt) + 1))
        tries = 0
        while len(out) < size and tries < 50 * size:
            tries += 1
            slots = tuple(sorted(rng.choice(occ_slots, size=lev, replace=False)))
            orbs = tuple(rng.choice(virt, size=lev, replace=False))
            key = (slots, tuple(sorted(orbs)))
            if key in seen:
                continue
            seen.add(key)
            occ = list(range(1, nel + 1))
            for sl, o in zip(slots, orbs):
                occ[sl] = int(o)
            out.append(tuple(occ))
        return out
    ref = (tuple(range(1, nup + 1)), tuple(range(1, ndn + 1)))
    pu = {lev: pool(nup, lev, sz) for lev, sz in zip((1, 2, 3, 4), pools)}
    pd = {lev: pool(ndn, lev, sz) for lev, sz in zip((1, 2, 3, 4), pools)}
    dets, seen = [ref], {ref}
    while len(dets) < ndet:
        L = int(rng.choice([1, 2, 3, 4], p=list(level_p)))
        lu = int(rng.integers(0, L + 1))
        ld = L - lu
        up = ref[0] if lu == 0 else pu[lu][int(rng.integers(len(pu[lu])))]
        dn = ref[1] if ld == 0 else pd[ld][int(rng.integers(len(pd[ld])))]
        if (up, dn) in seen:
            continue
        seen.add((up, dn))
        dets.append((up, dn))
    iworbd = np.array([list(u) + list(d) for u, d in dets], np.int32)
    k = np.arange(1, ndet + 1, dtype=float)
    cdet = k ** -1.5 * np.where(rng.random(ndet) < 0.5, -1.0, 1.0)
    cdet[0] = 1.0
    return iworbd, cdet


def _c2(rng, orbitals="model") -> System:
    """Config 2: 12 centres (9 C-like Z=4 with BFD-form ECP, 3 H-like), 40
    electrons (20/20; the valence charges add up to 39, so one extra
    electron), 300 Gaussians (C-like s4p5d1, H-like s4p7), 80 orbitals,
    order-5 Jastrow, 10^4 determinants (ci_expansion)."""
    nat = 12
    types = [0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1]
    cent = np.zeros((nat, 3))
    for i in range(nat):
        cent[i] = (1.35 * i + rng.normal(0, 0.05), 0.8 * (i % 2) + rng.normal(0, 0.05), 0.4 * ((i // 2) % 2) +
                   rng.normal(0, 0.05))
    heavy = dict(z=4.0, lpot=2, a1=0.0,
                 basis=_type_from_shells(_random_shells(rng, [(0, 4), (1, 5), (2, 1)]), 4.0, 4))
    hyd = dict(z=1.0, lpot=1, a1=-1.0,
               basis=_type_from_shells(_random_shells(rng, [(0, 4), (1, 7)]), 1.0, 4))
    s = _assemble("c2", rng, cent, types, [heavy, hyd], 40, 20, 80, 20, 20, orbitals=orbitals)
    s.iworbd, s.cdet = ci_expansion(rng, 20, 20, 80, 10000)
    return s


HE_EXACT = -2.903724377  # non-relativistic ground state of He, Hartree


def _helium() -> System:
    """He atom through the ECP code path (a bare-Coulomb local channel, no
    nonlocal channel), one 1s orbital for both spins: a nodeless trial
    function, so DMC converges to the exact ground-state energy HE_EXACT.

    The orbital is a non-negative combination of six s Gaussians fitted to
    exp(-zeta r) / exp(J_en(r)) so that orbital times the electron-nucleus
    Jastrow factor (a1 = -2: the nuclear cusp) is close to the hydrogenic
    1s with zeta = 27/16; the electron-electron term carries the 1/2 cusp.
    """
    from scipy.optimize import nnls
    kappa, zeta = 0.6, 27.0 / 16.0
    ex = np.array([0.08, 0.25, 0.8, 2.5, 8.0, 25.0])
    r = np.linspace(0.0, 8.0, 801)
    target = np.exp(-zeta * r + 2.0 * (1.0 - np.exp(-kappa * r)) / kappa)
    A = np.stack([gnorm(e, 0) * np.exp(-e * r * r) for e in ex], axis=1)
    wts = (r + 0.05)
    co, _ = nnls(A * wts[:, None], target * wts)
    keep = co > 0
    shells = [(0, ex[keep], co[keep])]
    he = dict(z=2.0, lpot=1, a1=-2.0, basis=_type_from_shells(shells, 2.0, 4))
    basis = assemble_basis([he["basis"]])
    rng = np.random.default_rng(7)
    a4 = np.zeros((1, 6))
    a4[0, 0] = -2.0
    b = np.zeros((1, 6))
    b[0, 0] = 0.5
    c = np.zeros((1, nterms4(5)))
    nterm, power, expo, ecoef = _bfd_like_ecp(rng, 2.0, 1)
    xq, yq, zq, wq = gesqua(6)
    return System(name="he", nelec=2, nup=1, iwctype=np.array([0], np.int32), cent=np.zeros((1, 3)),
                  znuc=np.array([2.0]), coef=np.ones((1, 1)), iworbd=np.array([[1, 1]], np.int32),
                  cdet=np.array([1.0]), norda=5, nordb=5, nordc=5, scalek=kappa, a4=a4, b=b, c=c,
                  nloc=4, lpot=np.array([1], np.int32), necp_term=nterm[None], necp_power=power[None],
                  ecp_exponent=expo[None], ecp_coef=ecoef[None], nquad=6, xq0=xq, yq0=yq, zq0=zq, wq=wq,
                  **basis)


def rotation_expansion(s: System, rots, extra_orbitals: int = 0, seed: int = 11, permute: bool = True):
    """Multideterminant system built from orbital rotations, and its single-
    determinant twin.

    Each rotation (spin, slot, orbital, t) replaces the reference orbital of
    that electron slot by phi_ref + t * phi_orbital (0-based orbital, a
    virtual one).  The product over rotations of (reference + t * excitation)
    is a multideterminant expansion with 2**len(rots) determinants whose
    value equals the single determinant of the rotated orbitals; the twin
    holds those rotated orbitals as extra LCAO rows.  With permute=True some
    determinants list their orbitals in a swapped order with the sign folded
    into cdet, as CHAMP inputs may.  Returns (multidet system, twin).
    """
    import dataclasses
    import itertools
    rng = np.random.default_rng(seed)
    coef = np.asarray(s.coef, float)
    if extra_orbitals:
        extra = rng.normal(size=(extra_orbitals, coef.shape[1])) * 0.3
        coef = np.vstack([coef, extra])
    ref = np.asarray(s.iworbd[0], np.int32)
    slots = [(sp, sl) for sp, sl, _, _ in rots]
    if len(set(slots)) != len(slots):
        raise ValueError("one rotation per electron slot")
    dets, cdets = [], []
    for mask in itertools.product([0, 1], repeat=len(rots)):
        occ = ref.copy()
        c = 1.0
        for (sp, sl, orb, t), m in zip(rots, mask):
            if m:
                occ[sl + (0 if sp == 0 else s.nup)] = orb + 1
                c *= t
        if permute and len(dets) % 3 == 1 and s.nup >= 2:
            occ[0], occ[1] = occ[1], occ[0]
            c = -c
        dets.append(occ)
        cdets.append(c)
    md = dataclasses.replace(s, name=s.name + "_md", coef=coef, iworbd=np.array(dets, np.int32),
                             cdet=np.array(cdets, float), _keep=[])
    # twin: rotated orbitals appended as new rows, the up and down slots point at them
    rows = [coef]
    occ1 = ref.copy()
    nextra = coef.shape[0]
    for sp, sl, orb, t in rots:
        e = sl + (0 if sp == 0 else s.nup)
        o = occ1[e] - 1
        rows.append((coef[o] + t * coef[orb])[None, :])
        occ1[e] = nextra + 1
        nextra += 1
    twin = dataclasses.replace(s, name=s.name + "_twin", coef=np.vstack(rows), iworbd=occ1[None, :].astype(np.int32),
                               cdet=np.array([1.0]), _keep=[])
    return md, twin
