"""The oracle's multideterminant wave function (multideterminants_define,
multideterminante, compute_ymat, multideterminante_grad,
multideterminant_hpsi) against two independent checks:

* exact equivalence: a product of orbital rotations expands into 2**n
  determinants whose sum equals one determinant of rotated orbitals, so ψ,
  E_L (kinetic and ECP parts), the drift and whole VMC/DMC trajectories on
  identical streams must match the single-determinant path;
* brute force: ψ of a non-factorizable expansion (random CI coefficients,
  single to triple excitations, permuted orbital lists) against numpy
  determinants of the oracle's own orbital values."""
import numpy as np
import pytest

ROTS = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]


def _systems():
    from champ_b200.system import make_synthetic, rotation_expansion
    return rotation_expansion(make_synthetic("tiny"), ROTS, extra_orbitals=4)


def _configs(oracle_mod, o, W):
    st = oracle_mod.rng_states(W)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    return np.array(xs), st


def test_rotation_equivalence_hpsi(oracle_mod):
    md, twin = _systems()
    assert md.iworbd.shape[0] == 32
    om, ot = oracle_mod.OracleSystem(md), oracle_mod.OracleSystem(twin)
    xs, _ = _configs(oracle_mod, om, 6)
    for x in xs:
        a, b = om.hpsi(x), ot.hpsi(x)
        assert abs(a["psid"] - b["psid"]) <= 1e-11 * abs(b["psid"])
        for k in ("energy", "ekin", "psij"):
            assert abs(a[k] - b[k]) <= 1e-9 * max(1.0, abs(b[k])), (k, a[k], b[k])


def test_bruteforce_psi(oracle_mod):
    from champ_b200.system import make_synthetic, rotation_expansion
    md, _ = rotation_expansion(make_synthetic("tiny"), ROTS, extra_orbitals=4)
    rng = np.random.default_rng(3)
    md.cdet = rng.normal(size=md.cdet.shape)          # no longer a product: a genuine CI vector
    om = oracle_mod.OracleSystem(md)
    xs, _ = _configs(oracle_mod, om, 5)
    nup = md.nup
    for x in xs:
        orb, _, _ = om.orbitals(x)                    # [norb][nelec]
        psi = 0.0
        for occ, c in zip(md.iworbd, md.cdet):
            up = orb[np.asarray(occ[:nup]) - 1][:, :nup].T
            dn = orb[np.asarray(occ[nup:]) - 1][:, nup:].T
            psi += c * np.linalg.det(up) * np.linalg.det(dn)
        r = om.hpsi(x)
        assert abs(r["psid"] - psi) <= 1e-10 * abs(psi)


def test_rotation_equivalence_vmc(oracle_mod):
    md, twin = _systems()
    om, ot = oracle_mod.OracleSystem(md), oracle_mod.OracleSystem(twin)
    xs, st = _configs(oracle_mod, om, 8)
    wm = oracle_mod.OracleWalkers(om, xs, st)
    wt = oracle_mod.OracleWalkers(ot, xs, st)
    for _ in range(3):
        wm.steps(1)
        wt.steps(1)
        xm, rm = wm.walkers()
        xt, rt = wt.walkers()
        assert np.array_equal(rm, rt)
        assert np.max(np.abs(xm - xt)) < 1e-9
        assert np.array_equal(wm.sums()[:, 4], wt.sums()[:, 4])
    em, _, _ = wm.state()
    et, _, _ = wt.state()
    assert np.max(np.abs(em - et) / np.maximum(1, np.abs(et))) < 1e-8


def test_rotation_equivalence_dmc(oracle_mod):
    md, twin = _systems()
    om, ot = oracle_mod.OracleSystem(md), oracle_mod.OracleSystem(twin)
    W = 12
    xs, st = _configs(oracle_mod, om, 4 * W + 1)
    x, rng, pop = xs[:W], st[:4 * W], st[4 * W]
    e0 = om.hpsi(x[0])["energy"]
    dm = oracle_mod.OracleDmc(om, x, rng, pop, tau=0.01, etrial=e0, mwalk=4 * W)
    dt = oracle_mod.OracleDmc(ot, x, rng, pop, tau=0.01, etrial=e0, mwalk=4 * W)
    for _ in range(3):
        dm.steps(1)
        dt.steps(1)
        a, b = dm.walkers(), dt.walkers()
        assert len(a[1]) == len(b[1])
        assert np.array_equal(a[3], b[3])
        assert np.max(np.abs(a[0] - b[0])) < 1e-9
        assert np.max(np.abs(a[1] - b[1]) / np.abs(b[1])) < 1e-9
