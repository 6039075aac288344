"""Trial orbitals of the synthetic molecules from a model one-electron Hamiltonian.

The synthetic molecules need a trial wave function whose local energy has a
finite, modest variance, so that the efficiency 1/(sigma^2 t) of a run means
something.  Orbitals here are the lowest eigenvectors of

    H0 = -1/2 nabla^2 + sum_A [ -Z_A erfc(sqrt(alpha_A) r_A) / r_A
                                + v_loc,A(r_A) + sum_l v_l,A(r_A) P_l,A ]

in the molecule's own basis: the kinetic energy, the attraction of each
nucleus screened by a Gaussian model density of its Z_A valence electrons
(a superposition of neutral-atom potentials, short-ranged for every atom),
and the atom's pseudopotential (local channel and the semilocal projectors,
the same BFD-form Gaussian sums the engine evaluates, vmc/readps_gauss.f90:57).
The overlap and kinetic matrices are analytic integrals over the contracted
Cartesian Gaussians the basis tables were tabulated from (Obara-Saika
recurrences); the potential matrix is a sum of atom-centred quadratures, one
per atom (its potential is short-ranged, so no partition of space is
needed).  The generalised eigenproblem H0 C = S C e is solved in the
canonically orthogonalised basis, so the orbitals are orthonormal in the
overlap metric and occupied by aufbau.

No counterpart in CHAMP: CHAMP reads its orbitals from an .lcao file made by
a quantum-chemistry code.  This module only makes the inputs of the
synthetic benchmarks.
"""
from __future__ import annotations

import math

import numpy as np

# Slm of vmc/slm.f90 as Cartesian monomials x^a y^b z^c times a constant
# (1-based index 1..20 used here: s, p, d, f)
_SLM_K = (0.28209479177387814, 0.48860251190291992, 0.630783130505040, 1.092548430592079)
SLM_MONO = {
    1: (0, 0, 0, _SLM_K[0]),
    2: (1, 0, 0, _SLM_K[1]), 3: (0, 1, 0, _SLM_K[1]), 4: (0, 0, 1, _SLM_K[1]),
    5: (2, 0, 0, _SLM_K[2]), 6: (1, 1, 0, _SLM_K[3]), 7: (1, 0, 1, _SLM_K[3]),
    8: (0, 2, 0, _SLM_K[2]), 9: (0, 1, 1, _SLM_K[3]), 10: (0, 0, 2, _SLM_K[2]),
}


def primitives(cent, types_of_centre, type_shells, type_aos, gnorm):
    """The molecule's basis in the engine's AO order (centre by centre, the
    AOs of a centre in the order of its type's list).

    Returns (prim, basis).  prim: arrays over primitive Gaussians -- centre
    coordinates A [P,3], exponents alpha [P], monomial powers lmn [P,3],
    coefficient [P] (Slm constant x gnorm x contraction coefficient), owning
    AO [P].  basis: per shell its centre, exponents and gnorm-weighted
    contraction coefficients; per AO its shell, monomial powers, Slm
    constant and centre."""
    A, al, lmn, co, ao = [], [], [], [], []
    sh_cent, sh_ex, sh_co = [], [], []
    ao_shell, ao_mono, ao_k, ao_cent = [], [], [], []
    k = 0
    for ic, it in enumerate(types_of_centre):
        shells = type_shells[it]
        first = len(sh_cent)
        for l, ex, cc in shells:
            sh_cent.append(ic)
            sh_ex.append(np.asarray(ex, float))
            sh_co.append(np.array([gnorm(e, l) * w for e, w in zip(ex, cc)]))
        for slm, irb in type_aos[it]:
            l, ex, cc = shells[irb - 1]
            a, b, c, kk = SLM_MONO[slm]
            for e, w in zip(ex, cc):
                A.append(cent[ic])
                al.append(e)
                lmn.append((a, b, c))
                co.append(kk * gnorm(e, l) * w)
                ao.append(k)
            ao_shell.append(first + irb - 1)
            ao_mono.append((a, b, c))
            ao_k.append(kk)
            ao_cent.append(ic)
            k += 1
    prim = dict(A=np.array(A, float), alpha=np.array(al, float), lmn=np.array(lmn, int),
                coef=np.array(co, float), ao=np.array(ao, int))
    basis = dict(cent=np.asarray(cent, float), sh_cent=np.array(sh_cent, int), sh_ex=sh_ex, sh_co=sh_co,
                 ao_shell=np.array(ao_shell, int), ao_mono=np.array(ao_mono, int), ao_k=np.array(ao_k, float),
                 ao_cent=np.array(ao_cent, int))
    return prim, basis


def _os_1d(XA, XB, p, imax, jmax):
    """Obara-Saika overlap recurrences in one dimension for all primitive
    pairs: S[i][j] (without the common exp/sqrt prefactor), i <= imax, j <= jmax."""
    S = [[None] * (jmax + 1) for _ in range(imax + 1)]
    one = np.ones_like(XA)
    S[0][0] = one
    h = 0.5 / p
    for i in range(imax + 1):
        for j in range(jmax + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                v = XA * S[i - 1][j]
                if i > 1:
                    v = v + (i - 1) * h * S[i - 2][j]
                if j > 0:
                    v = v + j * h * S[i - 1][j - 1]
            else:
                v = XB * S[i][j - 1]
                if j > 1:
                    v = v + (j - 1) * h * S[i][j - 2]
            S[i][j] = v
    return S


def overlap_kinetic(prim, nbasis, chunk=1 << 17):
    """Analytic overlap S and kinetic T = -1/2 <mu|nabla^2|nu> of the AOs,
    accumulated over chunks of primitive pairs."""
    A, al, lmn, co, ao = prim["A"], prim["alpha"], prim["lmn"], prim["coef"], prim["ao"]
    P = len(al)
    IA, IB = np.triu_indices(P)
    lmax = int(lmn.max())
    S = np.zeros(nbasis * nbasis)
    T = np.zeros(nbasis * nbasis)
    for c0 in range(0, len(IA), chunk):
        ia, ib = IA[c0:c0 + chunk], IB[c0:c0 + chunk]
        a, b = al[ia], al[ib]
        p = a + b
        mu = a * b / p
        Pc = (a[:, None] * A[ia] + b[:, None] * A[ib]) / p[:, None]
        AB2 = np.sum((A[ia] - A[ib]) ** 2, axis=1)
        pref = (math.pi / p) ** 1.5 * np.exp(-mu * AB2)
        s1, t1 = [], []
        for d in range(3):
            tab = _os_1d(Pc[:, d] - A[ia, d], Pc[:, d] - A[ib, d], p, lmax, lmax + 2)
            i = lmn[ia, d]
            j = lmn[ib, d]
            sd = np.zeros(len(ia))
            td = np.zeros(len(ia))
            for ii in range(lmax + 1):
                for jj in range(lmax + 1):
                    m = (i == ii) & (j == jj)
                    if not m.any():
                        continue
                    sv = tab[ii][jj][m]
                    # d^2/dx^2 of x^j e^{-b x^2} = j(j-1) x^{j-2} - 2b(2j+1) x^j + 4b^2 x^{j+2}
                    lap = -2.0 * b[m] * (2 * jj + 1) * sv + 4.0 * b[m] ** 2 * tab[ii][jj + 2][m]
                    if jj >= 2:
                        lap = lap + jj * (jj - 1) * tab[ii][jj - 2][m]
                    sd[m] = sv
                    td[m] = -0.5 * lap
            s1.append(sd)
            t1.append(td)
        w = co[ia] * co[ib] * pref
        sp = w * s1[0] * s1[1] * s1[2]
        tp = w * (t1[0] * s1[1] * s1[2] + s1[0] * t1[1] * s1[2] + s1[0] * s1[1] * t1[2])
        off = ia != ib
        idx = np.concatenate([ao[ia] * nbasis + ao[ib], (ao[ib] * nbasis + ao[ia])[off]])
        S += np.bincount(idx, np.concatenate([sp, sp[off]]), minlength=nbasis * nbasis)
        T += np.bincount(idx, np.concatenate([tp, tp[off]]), minlength=nbasis * nbasis)
    return S.reshape(nbasis, nbasis), T.reshape(nbasis, nbasis)


def ao_values(basis, aos, pts):
    """Values of the AOs `aos` (indices into the basis) at points [npts,3]
    -> [npts, len(aos)]: each shell's radial sum once, times the monomials."""
    out = np.empty((len(pts), len(aos)))
    rad = {}
    for j, m in enumerate(aos):
        sh = basis["ao_shell"][m]
        d = pts - basis["cent"][basis["sh_cent"][sh]]
        if sh not in rad:
            r2 = np.einsum("ij,ij->i", d, d)
            v = np.zeros(len(pts))
            for e, w in zip(basis["sh_ex"][sh], basis["sh_co"][sh]):
                v += w * np.exp(-e * r2)
            rad[sh] = v
        v = basis["ao_k"][m] * rad[sh]
        a, b, c = basis["ao_mono"][m]
        if a:
            v = v * d[:, 0] ** a
        if b:
            v = v * d[:, 1] ** b
        if c:
            v = v * d[:, 2] ** c
        out[:, j] = v
    return out


def atom_grid(nrad=40, ntheta=12, nphi=24, rm=1.0, rcut=8.0):
    """Atom-centred quadrature: Gauss-Chebyshev (second kind) radial points
    mapped by r = rm (1+x)/(1-x) (points beyond rcut dropped), times a
    Gauss-Legendre (cos theta) x uniform (phi) sphere.  Returns radial
    r [nr], radial weights (including r^2) [nr], unit vectors [nang,3],
    angular weights [nang] (summing to 4 pi)."""
    i = np.arange(1, nrad + 1)
    x = np.cos(i * np.pi / (nrad + 1))
    wx = np.pi / (nrad + 1) * np.sin(i * np.pi / (nrad + 1)) ** 2 / np.sqrt(1 - x * x)
    r = rm * (1 + x) / (1 - x)
    dr = rm * 2.0 / (1 - x) ** 2
    wr = wx * dr * r * r
    keep = r <= rcut
    r, wr = r[keep], wr[keep]
    ct, wt = np.polynomial.legendre.leggauss(ntheta)
    ph = (np.arange(nphi) + 0.5) * 2 * np.pi / nphi
    st = np.sqrt(1 - ct * ct)
    u = np.stack([np.outer(st, np.cos(ph)).ravel(), np.outer(st, np.sin(ph)).ravel(),
                  np.repeat(ct, nphi)], axis=1)
    wa = np.repeat(wt, nphi) * (2 * np.pi / nphi)
    return r, wr, u, wa


def gauss_sum(r, nterm, power, expo, coef):
    """BFD Gaussian sum v(r) = sum_k coef_k r^(power_k - 2) exp(-expo_k r^2)
    (gauss_pot, vmc/readps_gauss.f90:57)."""
    v = np.zeros_like(r)
    for k in range(int(nterm)):
        v += coef[k] * r ** (power[k] - 2) * np.exp(-expo[k] * r * r)
    return v


def potential_matrix(basis, cent, types_of_centre, znuc, ecp, screen_alpha, reach=14.0):
    """Sum over atoms of the atom-centred quadrature of the screened nuclear
    attraction, the local pseudopotential channel and the semilocal
    projectors.  ecp: None or per type (lpot, nterm[4], power[4,16],
    expo[4,16], coef[4,16]) with the local channel at index lpot-1 and the
    nonlocal channel l at index l.  AOs of centres farther than `reach`
    bohr from the atom are left out of its quadrature."""
    from scipy.special import erfc
    ao_cent = basis["ao_cent"]
    nbasis = len(ao_cent)
    V = np.zeros((nbasis, nbasis))
    for iat, it in enumerate(types_of_centre):
        Z = float(znuc[it])
        al = screen_alpha[it]
        r, wr, u, wa = atom_grid(rcut=6.0 / math.sqrt(al))
        near = np.nonzero(np.sum((cent[ao_cent] - cent[iat]) ** 2, axis=1) <= reach * reach)[0]
        pts = (cent[iat] + r[:, None, None] * u[None, :, :]).reshape(-1, 3)
        phi = ao_values(basis, near, pts)
        vloc = -Z * erfc(math.sqrt(al) * r) / r
        lp = 0
        if ecp is not None and ecp[it] is not None:
            lpot, nterm, power, expo, coef = ecp[it]
            lp = int(lpot)
            vloc = vloc + gauss_sum(r, nterm[lp - 1], power[lp - 1], expo[lp - 1], coef[lp - 1])
        w = ((wr * vloc)[:, None] * wa[None, :]).ravel()
        Vs = (phi * w[:, None]).T @ phi
        # semilocal projectors: sum_m <mu|Y_lm> v_l <Y_lm|nu> on each radial shell
        ph3 = phi.reshape(len(r), len(u), len(near))
        for l in range(max(0, lp - 1)):
            vl = gauss_sum(r, nterm[l], power[l], expo[l], coef[l])
            for Y in _real_ylm(l, u):
                f = np.einsum("ram,a->rm", ph3, wa * Y)
                Vs += (f * (wr * vl)[:, None]).T @ f
        V[np.ix_(near, near)] += Vs
    return 0.5 * (V + V.T)


def _real_ylm(l, u):
    x, y, z = u[:, 0], u[:, 1], u[:, 2]
    if l == 0:
        return [np.full(len(u), 0.28209479177387814)]
    if l == 1:
        c = 0.48860251190291992
        return [c * x, c * y, c * z]
    if l == 2:
        c1, c2, c3 = 1.0925484305920792, 0.31539156525252005, 0.5462742152960396
        return [c1 * x * y, c1 * y * z, c2 * (3 * z * z - 1), c1 * x * z, c3 * (x * x - y * y)]
    raise ValueError("projectors up to l=2")


def model_orbitals(S, H, norb, lindep=1e-8):
    """Lowest `norb` eigenvectors of H C = S C e by canonical orthogonalisation
    (overlap eigenvectors with eigenvalues below lindep x the largest are
    dropped).  Returns (coef [norb, nbasis], orbital energies [norb])."""
    s, U = np.linalg.eigh(S)
    keep = s > lindep * s[-1]
    X = U[:, keep] / np.sqrt(s[keep])
    e, C = np.linalg.eigh(X.T @ H @ X)
    if C.shape[1] < norb:
        raise ValueError(f"basis keeps {C.shape[1]} independent functions, {norb} orbitals asked")
    coef = (X @ C[:, :norb]).T
    # fixed sign convention: largest coefficient of each orbital positive
    for i in range(norb):
        if coef[i, np.argmax(np.abs(coef[i]))] < 0:
            coef[i] = -coef[i]
    return np.ascontiguousarray(coef), e[:norb]
