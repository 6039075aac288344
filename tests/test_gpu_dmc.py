"""GPU parity of the DMC step (dmc_ps + reweighting + splitj + acues1): the
CUDA engine through the C ABI against the oracle, with the same per-slot
move streams and the same population stream, so both take the same
accept/reject, branching and copy decisions."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _md32():
    from champ_b200.system import make_synthetic, rotation_expansion
    rots = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]
    md, _ = rotation_expansion(make_synthetic("tiny"), rots, extra_orbitals=4)
    md.cdet = np.random.default_rng(3).normal(size=md.cdet.shape) * 0.3
    md.cdet[0] = 1.0
    return md


def _vmc_start(oracle_mod, config, W, nslot, vmc_steps):
    from champ_b200.system import make_synthetic
    s = _md32() if config == "md32" else make_synthetic(config)
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


@pytest.mark.parametrize("config,W,nstep", [("md32", 32, 5), ("c2", 6, 2)])
def test_dmc_tmove_md_parity(oracle_mod, config, W, nstep):
    """T-moves of multideterminant wave functions (multideterminant_tmove):
    the elements gain the excitations' part from hpsi's Y, the chosen
    electron's move is priced with the expansion's psi_D; same choices,
    moved electrons and populations as the oracle, on a 32-determinant
    expansion with permuted orbitals and on the 10^4-determinant molecule."""
    from champ_b200.engine import Dmc, Engine
    mw = 4 * W
    s, o, e0, x, rng, pop = _vmc_start(oracle_mod, config, W, mw, 6)
    dg = Dmc(Engine(s), x, rng, pop, tau=0.02, etrial=e0, mwalk=mw)
    dg.set_tmoves(-1)
    do = oracle_mod.OracleDmc(o, x, rng, pop, tau=0.02, etrial=e0, mwalk=mw)
    do.set_tmoves(-1)
    for step in range(nstep):
        dg.steps(1)
        do.steps(1, 8)
        _compare(dg, do)
    assert dg.counts()["tmoves"] == do.tmoves() > 0


def _all_electron(name):
    import copy
    import os
    from champ_b200.system import make_synthetic
    if name == "he":
        s = copy.deepcopy(make_synthetic("he"))
        s.nloc, s.nquad = 0, 0
        s.lpot = s.necp_term = s.necp_power = s.ecp_exponent = s.ecp_coef = None
        s.xq0 = s.yq0 = s.zq0 = s.wq = None
        s._keep = []
        return s
    from champ_b200.champ_io import load_npz
    from conftest import GOLDEN
    return load_npz(os.path.join(GOLDEN, "vmc_h2_system.npz"))


@pytest.mark.parametrize("name,W,tau", [("he", 32, 0.02), ("h2", 32, 0.01)])
def test_dmc_all_electron_parity(oracle_mod, name, W, tau):
    """dmc_ae moves (dmc/dmc_ae_mov1.f90:4) of all-electron wave functions:
    identical populations, streams, weights, positions and energies."""
    from champ_b200.engine import Dmc, Engine
    s = _all_electron(name)
    o = oracle_mod.OracleSystem(s)
    mw = 4 * W
    st = oracle_mod.rng_states(mw + 2)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    vw = oracle_mod.OracleWalkers(o, np.array(xs), st[:W])
    vw.steps(20, 8)
    vw.end_block()
    x, r = vw.walkers()
    rng = np.concatenate([r, st[W:mw]])
    e0 = vw.results()["energy"]
    dg = Dmc(Engine(s), x, rng, st[mw], tau=tau, etrial=e0, mwalk=mw)
    do = oracle_mod.OracleDmc(o, x, rng, st[mw], tau=tau, etrial=e0, mwalk=mw)
    _compare(dg, do)
    for step in range(5):
        dg.steps(1)
        do.steps(1, 8)
        _compare(dg, do)
    dg.end_block()
    do.end_block()
    rg, ro = dg.results(), do.results()
    for k in ("energy", "nwalk", "eest", "accept", "taueff", "fprod", "eigv"):
        assert abs(rg[k] - ro[k]) <= 1e-9 * max(1.0, abs(ro[k])), k


def test_dmc_all_electron_helium_exact_gpu(oracle_mod):
    """All-electron He (nodeless trial function) through the engine's dmc_ae
    moves reaches the exact energy."""
    from champ_b200.engine import Dmc, Engine, initial_configs, rng_states
    from champ_b200.system import HE_EXACT
    s = _all_electron("he")
    W = 1024
    st = rng_states(3 * W + 1)
    x = initial_configs(s, st[:W].copy())
    eng = Engine(s)
    eng.set_walkers(x, st[:W].copy())
    eng.vmc_steps(100)
    xv, _ = eng.walkers()
    e0 = float(np.mean(eng.state()[0]))
    d = Dmc(eng, xv, st[:3 * W], st[3 * W], tau=0.02, etrial=e0, mwalk=3 * W)
    d.steps(200)
    d.end_block()
    for _ in range(10):
        d.steps(100)
        d.end_block()
    r = d.results()
    print(f"all-electron He DMC {r['energy']:.5f} +- {r['err']:.5f} (exact {HE_EXACT}), accept {r['accept']:.4f}")
    assert abs(r["energy"] - HE_EXACT) <= 3 * r["err"] + 1e-3, r
