"""The oracle's DMC (dmc_ps + branching + splitj + acues1/acuest) on the CPU.

The reference's own DMC CI cases cannot be rerun here (their initial walker
files and several orbital files are not in the source tree, and there is no
Fortran compiler), so the DMC restatement is pinned by physics instead: He
through the ECP move path with a nodeless trial function, where DMC must
reach the exact ground-state energy while VMC stays above it."""
import numpy as np
import pytest


def _he_population(oracle_mod, W, nvmc_blocks=10):
    from champ_b200.system import make_synthetic
    s = make_synthetic("he")
    o = oracle_mod.OracleSystem(s)
    st = oracle_mod.rng_states(3 * W + 2)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    vw = oracle_mod.OracleWalkers(o, np.array(xs), st[:W])
    vw.steps(50, 8)
    vw.end_block()
    vw.zerest()
    for _ in range(nvmc_blocks):
        vw.steps(20, 8)
        vw.end_block()
    x, r = vw.walkers()
    rng = np.concatenate([r, st[W:3 * W]])
    return s, o, vw.results(), x, rng, st[3 * W], st[3 * W + 1]


def test_dmc_helium_exact(oracle_mod):
    from champ_b200.system import HE_EXACT
    W, tau = 400, 0.01
    s, o, vmc, x, rng, pop0, pop1 = _he_population(oracle_mod, W)
    eq = oracle_mod.OracleDmc(o, x, rng, pop0, tau=tau, etrial=vmc["energy"], mwalk=3 * W)
    for _ in range(20):
        eq.steps(100, 8)
        eq.end_block()
    xe = eq.walkers()[0]
    d = oracle_mod.OracleDmc(o, xe, rng, pop1, tau=tau, etrial=eq.results()["eest"], mwalk=3 * W)
    for _ in range(20):
        d.steps(100, 8)
        d.end_block()
    r = d.results()
    # DMC projects out the exact energy (tau=0.01 time-step bias << 1 mHa for He)
    assert abs(r["energy"] - HE_EXACT) <= 3 * r["err"] + 1e-3, r
    # while VMC with the same trial function stays clearly above it
    assert vmc["energy"] - HE_EXACT > 5 * vmc["err"], vmc
    assert r["energy"] < vmc["energy"] - 3 * np.hypot(r["err"], vmc["err"])
    assert 0.98 < r["accept"] < 1.0
    assert abs(r["taueff"] - tau) < 0.01 * tau
    assert W // 2 < r["nwalk"] < 2 * W


def test_dmc_threads_and_determinism(oracle_mod):
    """Walkers move independently on their own streams: the thread count
    does not change the result, and reruns are bit-identical."""
    W = 24
    s, o, vmc, x, rng, pop0, _ = _he_population(oracle_mod, W, nvmc_blocks=1)
    runs = []
    for nth in (1, 4, 4):
        d = oracle_mod.OracleDmc(o, x, rng, pop0, tau=0.02, etrial=vmc["energy"], mwalk=3 * W)
        for _ in range(3):
            d.steps(10, nth)
            d.end_block()
        runs.append((d.walkers(), d.results()))
    (w0, r0) = runs[0]
    for (w1, r1) in runs[1:]:
        for a, b in zip(w0, w1):
            assert np.array_equal(a, b)
        assert r0 == r1


def test_dmc_branching_population(oracle_mod):
    """A poor trial function (random orbitals) branches heavily: the
    population changes size, stays inside mwalk, and keeps finite,
    non-negative weights."""
    from champ_b200.system import make_synthetic
    s = make_synthetic("tiny")
    o = oracle_mod.OracleSystem(s)
    W = 32
    st = oracle_mod.rng_states(4 * W + 1)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    vw = oracle_mod.OracleWalkers(o, np.array(xs), st[:W])
    vw.steps(20, 4)
    vw.end_block()
    x, r = vw.walkers()
    rng = np.concatenate([r, st[W:4 * W]])
    d = oracle_mod.OracleDmc(o, x, rng, st[4 * W], tau=0.01, etrial=vw.results()["energy"], mwalk=4 * W)
    sizes = []
    for _ in range(6):
        d.steps(1, 4)
        xw, wt, eo, rw = d.walkers()
        sizes.append(len(wt))
        assert 0 < len(wt) <= 4 * W
        assert np.all(wt >= 0) and np.all(np.isfinite(eo))
    assert len(set(sizes)) > 1, "population never changed: branching not exercised"


def test_tmoves_oracle(oracle_mod):
    """T-moves move electrons when the pseudopotential has negative matrix
    elements, reproducibly, and are refused where unsupported."""
    from champ_b200.system import make_synthetic, rotation_expansion
    s = make_synthetic("c0")
    o = oracle_mod.OracleSystem(s)
    W = 16
    st = oracle_mod.rng_states(4 * W + 1)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    e0 = float(np.median([o.hpsi(x)["energy"] for x in xs]))
    runs = []
    for _ in range(2):
        d = oracle_mod.OracleDmc(o, np.array(xs), st[:4 * W], st[4 * W], tau=0.02, etrial=e0, mwalk=4 * W)
        d.set_tmoves(-1)
        d.steps(4, 4)
        runs.append((d.tmoves(), d.walkers()[0]))
    assert runs[0][0] == runs[1][0] > 0
    assert np.array_equal(runs[0][1], runs[1][1])
    # multideterminant expansions take T-moves too (test_oracle_tmove_md_cpu)
    md, _ = rotation_expansion(make_synthetic("tiny"), [(0, 2, 3, 0.3)], extra_orbitals=2)
    om = oracle_mod.OracleSystem(md)
    dm = oracle_mod.OracleDmc(om, np.array([om.sites(st[0])[0]]), st[:4], st[4], tau=0.01, etrial=0.0, mwalk=4)
    dm.set_tmoves(-1)


def _he_all_electron():
    import copy
    from champ_b200.system import make_synthetic
    s = copy.deepcopy(make_synthetic("he"))
    s.nloc, s.nquad = 0, 0
    s.lpot = s.necp_term = s.necp_power = s.ecp_exponent = s.ecp_coef = None
    s.xq0 = s.yq0 = s.zq0 = s.wq = None
    s._keep = []
    return s


def test_dmc_all_electron_helium_exact(oracle_mod):
    """dmc_ae (dmc/dmc_ae_mov1.f90:4) on all-electron He with a nodeless
    trial function reaches the exact energy: the move's drift in the
    nucleus frame, its Gaussian / exponential mixture and the reverse
    density, and dmc_eloc_cutoff's all-electron branch are then unbiased."""
    from champ_b200.system import HE_EXACT
    s = _he_all_electron()
    o = oracle_mod.OracleSystem(s)
    W = 400
    st = oracle_mod.rng_states(3 * W + 1)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    vw = oracle_mod.OracleWalkers(o, np.array(xs), st[:W])
    vw.steps(200, 8)
    vw.end_block()
    x, r = vw.walkers()
    rng = np.concatenate([r, st[W:3 * W]])
    d = oracle_mod.OracleDmc(o, x, rng, st[3 * W], tau=0.02, etrial=vw.results()["energy"], mwalk=3 * W)
    d.steps(200, 8)
    d.end_block()
    for _ in range(20):
        d.steps(100, 8)
        d.end_block()
    res = d.results()
    assert abs(res["energy"] - HE_EXACT) <= 3 * res["err"] + 1e-3, res
    assert res["accept"] > 0.98
