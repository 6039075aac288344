"""Several states sharing orbitals and Jastrow (CHAMP nstates > 1,
iguiding = 0) in the oracle, pinned by identities:

* the local energy and psi_D of state s at a configuration equal those of the
  single-state wave function with state s's CI vector;
* a state whose CI vector is a multiple of state 1's has state 1's energies
  exactly (its weight (psi_s/psi_1)^2 is a constant);
* the per-state block estimators are the (psi_s/psi_1)^2-weighted averages of
  the per-walker local energies of every sweep (acuest per istate)."""
import copy

import numpy as np
import pytest

ROTS = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]


def _multistate(alpha=None):
    from champ_b200.system import make_synthetic, rotation_expansion
    md, _ = rotation_expansion(make_synthetic("tiny"), ROTS, extra_orbitals=4)
    rng = np.random.default_rng(5)
    c1 = rng.normal(size=md.cdet.shape)
    c2 = alpha * c1 if alpha is not None else rng.normal(size=md.cdet.shape)
    c3 = rng.normal(size=md.cdet.shape)
    md.cdet = c1
    md.cdet_states = np.stack([c1, c2, c3])
    return md


def _single(md, s):
    one = copy.copy(md)
    one.cdet = np.array(md.cdet_states[s])
    one.cdet_states = None
    one._keep = []
    return one


def _walkers(oracle_mod, system, W):
    o = oracle_mod.OracleSystem(system)
    st = oracle_mod.rng_states(W)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    return o, np.array(xs), st


def test_state_energies_match_single_state(oracle_mod):
    md = _multistate()
    o, xs, st = _walkers(oracle_mod, md, 5)
    ws = oracle_mod.OracleWalkers(o, xs, st.copy())
    e, p = ws.state_energies(3)
    for s in range(3):
        osingle = oracle_mod.OracleSystem(_single(md, s))
        for k, x in enumerate(xs):
            r = osingle.hpsi(x)
            assert abs(p[k, s] - r["psid"]) <= 1e-11 * abs(r["psid"])
            assert abs(e[k, s] - r["energy"]) <= 1e-9 * max(1.0, abs(r["energy"])), (s, k)


def test_proportional_state_has_state1_energies(oracle_mod):
    md = _multistate(alpha=-2.5)
    o, xs, st = _walkers(oracle_mod, md, 4)
    ws = oracle_mod.OracleWalkers(o, xs, st.copy())
    for _ in range(3):
        ws.steps(2, 1)
        ws.end_block()
    r1, r2 = ws.results_state(0), ws.results_state(1)
    assert r2["energy"] == pytest.approx(r1["energy"], rel=1e-12, abs=1e-12)
    assert r2["err"] == pytest.approx(r1["err"], rel=1e-9, abs=1e-12)
    assert ws.results()["energy"] == pytest.approx(r1["energy"], rel=1e-12)


def test_block_estimators_are_reweighted_averages(oracle_mod):
    md = _multistate()
    o, xs, st = _walkers(oracle_mod, md, 4)
    ws = oracle_mod.OracleWalkers(o, xs, st.copy())
    W, ns, nblk, nstep = 4, 3, 3, 2
    wsum = np.zeros(ns)
    esum = np.zeros(ns)
    ecm2 = np.zeros(ns)
    wcum = np.zeros(ns)
    for _ in range(nblk):
        bw = np.zeros((W, ns))
        be = np.zeros((W, ns))
        for _ in range(nstep):
            ws.steps(1, 1)
            e, p = ws.state_energies(ns)
            wt = (p / p[:, :1]) ** 2
            bw += wt
            be += wt * e
        ws.end_block()
        for k in range(W):                      # acuest per walker (rank) then the reduction
            en = be[k] / bw[k]
            wcum += bw[k]
            esum += be[k]
            ecm2 += be[k] * en
        wsum += bw.sum(0)
    for s in range(ns):
        r = ws.results_state(s)
        ef = esum[s] / wcum[s]
        err = np.sqrt(abs(ecm2[s] / wcum[s] - ef * ef) / (W * nblk))
        assert r["energy"] == pytest.approx(ef, rel=1e-11)
        assert r["err"] == pytest.approx(err, rel=1e-8)
    assert ws.results_state(0)["energy"] == pytest.approx(ws.results()["energy"], rel=1e-12)
    with pytest.raises(ValueError):
        ws.results_state(3)


def _guided(md, weights):
    g = copy.copy(md)
    g.iguiding = 1
    g.weights_g = np.asarray(weights, float)
    g._keep = []
    return g


def test_guiding_with_zero_weights_is_state1_walk(oracle_mod):
    """weights (1, 0, 0): psi2g = 1 exactly, so the guided walk is the walk of
    state 1, bitwise."""
    md = _multistate()
    o, xs, st = _walkers(oracle_mod, md, 4)
    a = oracle_mod.OracleWalkers(o, xs, st.copy())
    og = oracle_mod.OracleSystem(_guided(md, [1.0, 0.0, 0.0]))
    b = oracle_mod.OracleWalkers(og, xs, st.copy())
    for _ in range(2):
        a.steps(2, 1)
        b.steps(2, 1)
        a.end_block()
        b.end_block()
    xa, ra = a.walkers()
    xb, rb = b.walkers()
    assert np.array_equal(ra, rb) and np.array_equal(xa, xb)
    for s in range(3):
        assert a.results_state(s) == b.results_state(s)


def test_guiding_with_proportional_states_follows_state1(oracle_mod):
    """States proportional to state 1 leave psi_g proportional to psi_1: the
    guided walk is state 1's walk (to rounding) and every weight is 1/psi2g."""
    from champ_b200.system import make_synthetic, rotation_expansion
    md, _ = rotation_expansion(make_synthetic("tiny"), ROTS, extra_orbitals=4)
    c1 = np.random.default_rng(5).normal(size=md.cdet.shape)
    md.cdet = c1
    md.cdet_states = np.stack([c1, 2.0 * c1, -0.5 * c1])
    o, xs, st = _walkers(oracle_mod, md, 4)
    a = oracle_mod.OracleWalkers(o, xs, st.copy())
    b = oracle_mod.OracleWalkers(oracle_mod.OracleSystem(_guided(md, [1.0, 0.5, 2.0])), xs, st.copy())
    for _ in range(2):
        a.steps(2, 1)
        b.steps(2, 1)
    xa, ra = a.walkers()
    xb, rb = b.walkers()
    assert np.array_equal(ra, rb)
    assert np.max(np.abs(xa - xb)) < 1e-10
    a.end_block()
    b.end_block()
    for s in range(3):
        assert b.results_state(s)["energy"] == pytest.approx(a.results_state(0)["energy"], rel=1e-10)
