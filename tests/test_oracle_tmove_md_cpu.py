"""T-move matrix elements of multideterminant wave functions in the oracle
(dmc/multideterminant_tmove.f90:3 after nonloc.f90:296-301).

psi_D is linear in the orbital row of the electron a T-move displaces, so
CHAMP's correction of the reference-determinant element by the Y matrix,
detratio * sum ymat(jrep,irep) gmat(irep,jrep), makes every element exactly
term_radial_jas * psi_D(x_q) / psi_D(x), x_q the configuration with the
electron on the quadrature point.  The test checks that identity point by
point against full hpsi evaluations at x_q, on a 32-determinant expansion
with permuted orbitals and on the 40-electron, 10^4-determinant molecule,
and on a single determinant (where the correction vanishes)."""
import numpy as np
import pytest


def _systems(name):
    from champ_b200.system import make_synthetic, rotation_expansion
    if name == "md32":
        rots = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]
        md, _ = rotation_expansion(make_synthetic("tiny"), rots, extra_orbitals=4)
        md.cdet = np.random.default_rng(3).normal(size=md.cdet.shape) * 0.3
        md.cdet[0] = 1.0
        return md
    return make_synthetic(name)


@pytest.mark.parametrize("name,npoint", [("md32", 400), ("c2", 60), ("tiny", 200)])
def test_tmove_elements_exact_ratio(oracle_mod, name, npoint):
    from champ_b200.engine import initial_configs, rng_states
    s = _systems(name)
    o = oracle_mod.OracleSystem(s)
    rng = rng_states(2)
    x0 = initial_configs(s, rng)
    ow = oracle_mod.OracleWalkers(o, x0, rng)
    ow.steps(4, 2)
    x, _ = ow.walkers()
    cent = np.asarray(s.cent, float).reshape(-1, 3)
    xq, yq, zq = (np.asarray(a, float) for a in (s.xq0, s.yq0, s.zq0))
    checked = 0
    worst = 0.0
    for w in range(x.shape[0]):
        rows, psid = o.tmove_elements(x[w])
        assert len(rows) > 0
        for iel, ic, iq, trj, tv in rows[:npoint]:
            iel, ic, iq = int(iel), int(ic), int(iq)
            r = np.linalg.norm(x[w, iel] - cent[ic])
            xn = x[w].copy()
            xn[iel] = r * np.array([xq[iq], yq[iq], zq[iq]]) + cent[ic]
            exact = trj * o.hpsi(xn)["psid"] / psid
            err = abs(tv - exact) / max(abs(exact), 1e-3 * abs(trj))
            worst = max(worst, err)
            checked += 1
    print(f"{name}: {checked} quadrature points, worst relative difference {worst:.2e}")
    assert worst < 1e-8


def test_oracle_dmc_tmoves_multideterminant(oracle_mod):
    """The oracle's DMC with T-moves runs on a multideterminant expansion:
    T-moves are made, and two runs from the same streams agree bitwise."""
    from champ_b200.engine import initial_configs, rng_states
    s = _systems("md32")
    o = oracle_mod.OracleSystem(s)
    W = 16
    st = oracle_mod.rng_states(4 * W + 2)
    x = initial_configs(s, rng_states(W))
    vw = oracle_mod.OracleWalkers(o, x, st[:W])
    vw.steps(6, 2)
    vw.end_block()
    x, r = vw.walkers()
    e0 = vw.results()["energy"]
    runs = []
    for _ in range(2):
        do = oracle_mod.OracleDmc(o, x, np.concatenate([r, st[W:4 * W]]), st[4 * W], tau=0.02, etrial=e0,
                                  mwalk=4 * W)
        do.set_tmoves(-1)
        do.steps(4, 2)
        runs.append((do.tmoves(), do.walkers()[0]))
    assert runs[0][0] == runs[1][0] > 0
    assert np.array_equal(runs[0][1], runs[1][1])
