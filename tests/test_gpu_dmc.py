"""GPU parity of the DMC step (dmc_ps + reweighting + splitj + acues1): the
CUDA engine through the C ABI against the oracle, with the same per-slot
move streams and the same population stream, so both take the same
accept/reject, branching and copy decisions."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _vmc_start(oracle_mod, config, W, nslot, vmc_steps):
    from champ_b200.system import make_synthetic
    s = make_synthetic(config)
    o = oracle_mod.OracleSystem(s)
    st = oracle_mod.rng_states(nslot + 2)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    vw = oracle_mod.OracleWalkers(o, np.array(xs), st[:W])
    vw.steps(vmc_steps, 8)
    vw.end_block()
    x, r = vw.walkers()
    rng = np.concatenate([r, st[W:nslot]])
    return s, o, vw.results()["energy"], x, rng, st[nslot]


def _compare(dg, do, tol=1e-9):
    xg, wg, eg, rg = dg.walkers()
    xo, wo, eo, ro = do.walkers()
    assert len(wg) == len(wo), "population sizes differ"
    assert np.array_equal(rg, ro), "move streams diverged"
    assert rel_err(xg, xo) < tol
    assert rel_err(wg, wo) < tol
    assert rel_err(eg, eo) < tol


@pytest.mark.parametrize("config,W,tau", [("tiny", 32, 0.01), ("he", 64, 0.02), ("c0", 16, 0.005)])
def test_dmc_step_parity(oracle_mod, config, W, tau):
    from champ_b200.engine import Dmc, Engine
    mw = 4 * W
    s, o, e0, x, rng, pop = _vmc_start(oracle_mod, config, W, mw, 20)
    eng = Engine(s)
    dg = Dmc(eng, x, rng, pop, tau=tau, etrial=e0, mwalk=mw)
    do = oracle_mod.OracleDmc(o, x, rng, pop, tau=tau, etrial=e0, mwalk=mw)
    _compare(dg, do)
    for step in range(5):
        dg.steps(1)
        do.steps(1, 8)
        _compare(dg, do)
    dg.end_block()
    do.end_block()
    rg, ro = dg.results(), do.results()
    for k in ("energy", "nwalk", "eest", "accept", "taueff", "pe", "ke", "fprod", "eigv", "wdsumo"):
        assert abs(rg[k] - ro[k]) <= 1e-9 * max(1.0, abs(ro[k])), k


def test_dmc_helium_exact_gpu(oracle_mod):
    """The engine's DMC reaches the exact He energy, and over 4000 steps of
    400 walkers follows the oracle's trajectory to the same estimates."""
    from champ_b200.engine import Dmc, Engine
    from champ_b200.system import HE_EXACT
    W, tau = 400, 0.01
    s, o, e0, x, rng, pop = _vmc_start(oracle_mod, "he", W, 3 * W, 200)
    eng = Engine(s)
    dg = Dmc(eng, x, rng, pop, tau=tau, etrial=e0, mwalk=3 * W)
    do = oracle_mod.OracleDmc(o, x, rng, pop, tau=tau, etrial=e0, mwalk=3 * W)
    for _ in range(40):
        dg.steps(100)
        dg.end_block()
        do.steps(100, 16)
        do.end_block()
    rg, ro = dg.results(), do.results()
    assert abs(rg["energy"] - HE_EXACT) <= 3 * rg["err"] + 2e-3, rg
    for k in ("energy", "err", "nwalk", "accept", "taueff"):
        assert abs(rg[k] - ro[k]) <= 1e-8 * max(1.0, abs(ro[k])), (k, rg[k], ro[k])


def test_dmc_mwalk_exceeded(oracle_mod):
    """A capacity too small for the branching is reported, not overrun."""
    from champ_b200.engine import Dmc, Engine, EngineError
    s, o, e0, x, rng, pop = _vmc_start(oracle_mod, "tiny", 32, 33, 20)
    eng = Engine(s)
    dg = Dmc(eng, x, rng, pop, tau=0.05, etrial=e0 + 50.0, mwalk=33)
    with pytest.raises(EngineError, match="MWALK"):
        dg.steps(20)


@pytest.mark.parametrize("config,W", [("tiny", 32), ("c0", 24)])
def test_dmc_tmove_parity(oracle_mod, config, W):
    """T-moves (icasula = -1): same choices, same moved electrons, same
    populations as the oracle."""
    from champ_b200.engine import Dmc, Engine
    mw = 4 * W
    s, o, e0, x, rng, pop = _vmc_start(oracle_mod, config, W, mw, 10)
    eng = Engine(s)
    dg = Dmc(eng, x, rng, pop, tau=0.02, etrial=e0, mwalk=mw)
    dg.set_tmoves(-1)
    do = oracle_mod.OracleDmc(o, x, rng, pop, tau=0.02, etrial=e0, mwalk=mw)
    do.set_tmoves(-1)
    for step in range(5):
        dg.steps(1)
        do.steps(1, 8)
        _compare(dg, do)
    assert dg.counts()["tmoves"] == do.tmoves() > 0
