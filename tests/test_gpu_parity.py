"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle on
identical configurations and identical random streams.  FP64 plain path:
1e-10 relative (relative to the largest entry of each compared array)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _setup(oracle_mod, config, W, seed_steps=0):
    from champ_b200.engine import Engine, initial_configs, rng_states
    from champ_b200.system import make_synthetic
    s = make_synthetic(config)
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    o = oracle_mod.OracleSystem(s)
    return s, eng, o, x, rng


@pytest.fixture(scope="module", params=["tiny", "c0"])
def pop(request, oracle_mod):
    return _setup(oracle_mod, request.param, 8)


def test_orbitals(pop):
    s, eng, o, x, _ = pop
    orb, dorb, ddorb = eng.orbitals()
    for w in range(x.shape[0]):
        ro, rd, rdd = o.orbitals(x[w])
        assert rel_err(orb[w], ro) < TOL
        assert rel_err(dorb[w], rd) < TOL
        assert rel_err(ddorb[w], rdd) < TOL


def test_jastrow(pop):
    s, eng, o, x, _ = pop
    psij, v, d2 = eng.jastrow()
    for w in range(x.shape[0]):
        rj, rv, rd = o.jastrow(x[w])
        assert abs(psij[w] - rj) <= TOL * max(1.0, abs(rj))
        assert rel_err(v[w], rv) < TOL
        assert abs(d2[w] - rd) <= TOL * max(1.0, abs(rd))


def test_slater(pop):
    s, eng, o, x, _ = pop
    slmi, det = eng.slater()
    nmax = max(s.nup, s.ndn)
    for w in range(x.shape[0]):
        rs, rdet = o.slater(x[w])
        for iab, nel in enumerate((s.nup, s.ndn)):
            assert rel_err(slmi[w, iab, :nel * nel], rs[iab, :nel * nel]) < TOL
            assert abs(det[w, iab] - rdet[iab]) <= TOL * abs(rdet[iab])


@pytest.mark.parametrize("rotated", [False, True])
def test_hpsi(pop, rotated):
    s, eng, o, x, _ = pop
    quad = None
    if rotated and s.nloc:
        th = 0.7
        R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1.0]])
        q = R @ np.vstack([s.xq0, s.yq0, s.zq0])
        quad = (q[0].copy(), q[1].copy(), q[2].copy())
    h = eng.hpsi(quad)
    for w in range(x.shape[0]):
        r = o.hpsi(x[w], quad)
        assert abs(h["energy"][w] - r["energy"]) <= TOL * max(1.0, abs(r["energy"]))
        assert abs(h["psid"][w] - r["psid"]) <= TOL * abs(r["psid"])
        assert abs(h["psij"][w] - r["psij"]) <= TOL * max(1.0, abs(r["psij"]))
        assert abs(h["ekin"][w] - r["ekin"]) <= TOL * max(1.0, abs(r["ekin"]))


def test_vmc_stream_parity(oracle_mod):
    """Same streams => same accept/reject decisions, same walkers, same sums."""
    for config in ("tiny", "c0"):
        s, eng, o, x, rng = _setup(oracle_mod, config, 16)
        ow = oracle_mod.OracleWalkers(o, x, rng)
        for step in range(3):
            eng.vmc_steps(1)
            ow.steps(1)
            xg, rg = eng.walkers()
            xo, ro = ow.walkers()
            assert np.array_equal(rg, ro), f"{config}: random streams diverged at step {step}"
            assert rel_err(xg, xo) < 1e-9
            sg, so = eng.sums(), ow.sums()
            assert np.array_equal(sg[:, 4], so[:, 4]), "acceptance counts differ"
            assert rel_err(sg[:, :4], so[:, :4]) < 1e-9
        eg, _, _ = eng.state()
        eo, _, _ = ow.state()
        assert rel_err(eg, eo) < 1e-9


def test_block_statistics(oracle_mod):
    s, eng, o, x, rng = _setup(oracle_mod, "tiny", 16)
    ow = oracle_mod.OracleWalkers(o, x, rng)
    for _ in range(2):
        eng.vmc_steps(2)
        ow.steps(2)
        eb = eng.end_block()
        ob = ow.end_block()
        assert abs(eb - ob) <= 1e-9 * abs(ob)
    rg, ro = eng.results(), ow.results()
    for k in ("energy", "err", "sigma", "accept", "pe", "ke"):
        assert abs(rg[k] - ro[k]) <= 1e-8 * max(1.0, abs(ro[k])), k


def test_determinism(oracle_mod):
    from champ_b200.engine import Engine
    s, eng, o, x, rng = _setup(oracle_mod, "c0", 32)
    eng.vmc_steps(2)
    xa, ra = eng.walkers()
    ea, _, _ = eng.state()
    eng2 = Engine(s)
    eng2.set_walkers(x, rng)
    eng2.vmc_steps(2)
    xb, rb = eng2.walkers()
    eb, _, _ = eng2.state()
    assert np.array_equal(xa, xb) and np.array_equal(ra, rb) and np.array_equal(ea, eb)


def test_c1_hpsi(oracle_mod):
    """The 120-electron, 30-centre, 540-AO benchmark molecule: per-walker E_L
    at configurations equilibrated by 10 oracle sweeps (a sites start can put
    more same-spin electrons near an atom than its occupied orbitals hold,
    where the Slater matrix is nearly singular and E_L ill-conditioned)."""
    from champ_b200.engine import Engine
    s, eng, o, x, rng = _setup(oracle_mod, "c1", 2)
    ow = oracle_mod.OracleWalkers(o, x, rng)
    ow.steps(10, 2)
    x, rng = ow.walkers()
    eng.set_walkers(x, rng)
    h = eng.hpsi()
    for w in range(2):
        r = o.hpsi(x[w])
        assert abs(h["energy"][w] - r["energy"]) <= TOL * max(1.0, abs(r["energy"]))
        assert abs(h["psid"][w] - r["psid"]) <= 1e-9 * abs(r["psid"])
        assert abs(h["psij"][w] - r["psij"]) <= TOL * max(1.0, abs(r["psij"]))


def test_two_systems_interleaved(oracle_mod):
    """Two contexts of different molecules in one process, calls interleaved:
    each keeps computing its own system."""
    s1, e1, o1, x1, r1 = _setup(oracle_mod, "tiny", 8)
    s2, e2, o2, x2, r2 = _setup(oracle_mod, "c0", 8)
    w1 = oracle_mod.OracleWalkers(o1, x1, r1)
    w2 = oracle_mod.OracleWalkers(o2, x2, r2)
    for _ in range(2):
        h1 = e1.hpsi()
        h2 = e2.hpsi()
        xa, _ = e1.walkers()
        xb, _ = e2.walkers()
        for w in range(8):
            assert abs(h1["energy"][w] - o1.hpsi(xa[w])["energy"]) <= TOL * max(1.0, abs(h1["energy"][w]))
            assert abs(h2["energy"][w] - o2.hpsi(xb[w])["energy"]) <= TOL * max(1.0, abs(h2["energy"][w]))
        e1.vmc_steps(1)
        e2.vmc_steps(1)
        w1.steps(1)
        w2.steps(1)
        assert rel_err(e1.walkers()[0], w1.walkers()[0]) < 1e-9
        assert rel_err(e2.walkers()[0], w2.walkers()[0]) < 1e-9
