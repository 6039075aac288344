"""GPU parity of multi-state wave functions (three CI vectors over one
32-determinant expansion sharing orbitals and Jastrow, the walk sampling
state 1) against the oracle: per-walker local energies and psi_D of every
state, VMC on identical streams, the reweighted per-state block estimators,
a checkpoint/restore in the middle of a run, and VMC sampling the guiding
function of the states."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
ROTS = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]


def _system():
    from champ_b200.system import make_synthetic, rotation_expansion
    md, _ = rotation_expansion(make_synthetic("tiny"), ROTS, extra_orbitals=4)
    rng = np.random.default_rng(9)
    cs = rng.normal(size=(3,) + md.cdet.shape) * 0.3
    cs[:, 0] = 1.0
    md.cdet = cs[0].copy()
    md.cdet_states = cs
    return md


def _setup(oracle_mod, W):
    from champ_b200.engine import Engine, initial_configs, rng_states
    s = _system()
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    o = oracle_mod.OracleSystem(s)
    return s, eng, o, oracle_mod.OracleWalkers(o, x, rng), x


def test_state_energies_hpsi(oracle_mod):
    s, eng, o, ow, x = _setup(oracle_mod, 8)
    eg, pg = eng.state_energies()
    eo, po = ow.state_energies(3)
    assert eg.shape == (8, 3)
    assert rel_err(pg, po) < 1e-10
    assert np.max(np.abs(eg - eo)) < 1e-10 * max(1.0, np.max(np.abs(eo)))
    h = eng.hpsi()                                   # state 1 is the sampled one
    assert np.max(np.abs(h["energy"] - eg[:, 0])) < 1e-12 * max(1.0, np.max(np.abs(eo)))


def test_multistate_vmc_and_estimators(oracle_mod):
    s, eng, o, ow, x = _setup(oracle_mod, 16)
    for blk in range(3):
        eng.vmc_steps(2)
        ow.steps(2)
        xg, rg = eng.walkers()
        xo, ro = ow.walkers()
        assert np.array_equal(rg, ro), f"streams diverged in block {blk}"
        eg, _ = eng.state_energies()
        eo, _ = ow.state_energies(3)
        assert np.max(np.abs(eg - eo)) < 1e-9 * max(1.0, np.max(np.abs(eo)))
        eng.end_block()
        ow.end_block()
    for st in range(3):
        a, b = eng.results_state(st), ow.results_state(st)
        assert abs(a["energy"] - b["energy"]) < 1e-9 * max(1.0, abs(b["energy"])), st
        assert abs(a["err"] - b["err"]) < 1e-7 * max(1e-3, b["err"]), st
        assert a["nblocks"] == b["nblocks"]
    assert eng.results_state(0)["energy"] == pytest.approx(eng.results()["energy"], rel=1e-12)


def test_multistate_checkpoint_continues():
    from champ_b200.engine import Engine, initial_configs, rng_states
    s = _system()
    rng = rng_states(8)
    x = initial_configs(s, rng)
    a = Engine(s)
    a.set_walkers(x, rng)
    a.vmc_steps(2)
    a.end_block()
    a.vmc_steps(1)
    blob = a.checkpoint()
    b = Engine(s)
    b.restore(blob)
    for e in (a, b):
        e.vmc_steps(1)
        e.end_block()
    # the pseudopotential B matrix of a multideterminant expansion is summed
    # with atomics across warps (order not fixed), so the continuation agrees
    # to rounding rather than bitwise
    for st in range(3):
        ra, rb = a.results_state(st), b.results_state(st)
        for k in ra:
            assert rb[k] == pytest.approx(ra[k], rel=1e-12, abs=1e-14), (st, k)


def test_guiding_vmc_parity(oracle_mod):
    """Sampling the guiding function sum_i w_i |psi_i|^2: drift, acceptance and
    the per-state weights (psi_s/psi_1)^2 / psi2g on identical streams."""
    from champ_b200.engine import Engine, initial_configs, rng_states
    s = _system()
    s.iguiding = 1
    s.weights_g = np.array([1.0, 0.6, 0.3])
    W = 16
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    ow = oracle_mod.OracleWalkers(oracle_mod.OracleSystem(s), x, rng)
    for blk in range(3):
        eng.vmc_steps(2)
        ow.steps(2)
        xg, rg = eng.walkers()
        xo, ro = ow.walkers()
        assert np.array_equal(rg, ro), f"streams diverged in block {blk}"
        assert rel_err(xg, xo) < 1e-9
        sg, so = eng.sums(), ow.sums()
        assert np.array_equal(sg[:, 4], so[:, 4])               # identical accepted moves
        assert rel_err(sg[:, :4], so[:, :4]) < 1e-9             # state-1 sums weighted by 1/psi2g
        eng.end_block()
        ow.end_block()
    for st in range(3):
        a, b = eng.results_state(st), ow.results_state(st)
        assert abs(a["energy"] - b["energy"]) < 1e-9 * max(1.0, abs(b["energy"])), st
        assert abs(a["err"] - b["err"]) < 1e-7 * max(1e-3, b["err"]), st


def test_multistate_refusals():
    from champ_b200.engine import Dmc, Engine, EngineError, initial_configs, rng_states
    s = _system()
    s.iguiding = 1
    s.weights_g = np.array([0.0, 1.0, 1.0])      # state 1 must carry weight
    with pytest.raises(EngineError):
        Engine(s)
    s.weights_g = np.array([1.0, 1.0, 1.0])      # DMC does not sample a guiding function
    rng = rng_states(9)
    x = initial_configs(s, rng[:4].copy())
    with pytest.raises(EngineError, match="guiding"):
        Dmc(Engine(s), x, rng[:8], rng[8], tau=0.01, etrial=-1.0, mwalk=8)


def test_multistate_dmc_is_state_one(oracle_mod):
    """dmc_ps propagates and estimates state 1 alone (psidn(1), enew(1)):
    DMC of the three-state wave function takes the same steps as DMC of its
    first CI vector on its own (same populations, walkers, weights and
    energies), and the oracle agrees."""
    import copy
    from champ_b200.engine import Dmc, Engine
    s3 = _system()
    s1 = copy.deepcopy(s3)
    s1.cdet_states = None
    W, mw = 16, 64
    o = oracle_mod.OracleSystem(s1)
    st = oracle_mod.rng_states(mw + 2)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    vw = oracle_mod.OracleWalkers(o, np.array(xs), st[:W])
    vw.steps(8, 4)
    vw.end_block()
    x, r = vw.walkers()
    rng = np.concatenate([r, st[W:mw]])
    e0 = vw.results()["energy"]
    runs = {}
    for name, s in (("three", s3), ("one", s1)):
        d = Dmc(Engine(s), x, rng, st[mw], tau=0.01, etrial=e0, mwalk=mw)
        d.steps(5)
        runs[name] = d.walkers()
    do = oracle_mod.OracleDmc(o, x, rng, st[mw], tau=0.01, etrial=e0, mwalk=mw)
    do.steps(5, 4)
    ref = do.walkers()
    for name in ("three", "one"):
        xg, wg, eg, rg = runs[name]
        assert len(wg) == len(ref[1])
        assert np.array_equal(rg, ref[3])
        assert rel_err(xg, ref[0]) < 1e-9 and rel_err(wg, ref[1]) < 1e-9 and rel_err(eg, ref[2]) < 1e-9
    assert np.array_equal(runs["three"][3], runs["one"][3])
    assert rel_err(runs["three"][2], runs["one"][2]) < 1e-12
