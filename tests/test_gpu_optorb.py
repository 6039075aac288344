"""GPU parity of the orbital-rotation derivatives (optorb_deriv,
vmc/optorb.f90:5-95, for one determinant and for expansions) against the
oracle, and of the SR sums
over the joint [Jastrow | orbital] vector (optwf_store's sr_o layout,
vmc/optwf_handle_wf.f90:1517-1524)."""
import copy

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _with_virtuals(s, n, seed=5):
    rng = np.random.default_rng(seed)
    t = copy.deepcopy(s)
    t.coef = np.vstack([np.asarray(s.coef, float), rng.normal(size=(n, s.coef.shape[1])) * 0.3])
    t._keep = []
    return t


@pytest.mark.parametrize("config,W", [("tiny", 16), ("chain37", 8)])
def test_orb_derivatives_and_sr_sums(oracle_mod, config, W):
    from champ_b200.engine import Engine, initial_configs, rng_states
    from champ_b200.jastrow_opt import default_jasderiv, param_map
    from champ_b200.orbital_opt import orb_terms
    from champ_b200.system import make_chain, make_synthetic
    base = make_synthetic("tiny") if config == "tiny" else make_chain(37, 4037)
    s = _with_virtuals(base, 4)
    terms = orb_terms(s, nadorb=4)
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    o = oracle_mod.OracleSystem(s)
    P = param_map(s, default_jasderiv(s))
    eng.opt_orb(terms)
    eng.opt_setup(jas_map=P, overlap=True)
    nj = P.shape[1]
    # derivatives at the start configurations
    g = eng.orb_o()
    ref = np.array([o.orb_o(x[w], terms) for w in range(W)])
    assert rel_err(g, ref) < 1e-10
    # the SR sums over three sweeps against the per-sweep vectors
    so, seo, soo = 0, 0, 0
    for _ in range(3):
        eng.vmc_steps(1)
        xw, _ = eng.walkers()
        g = eng.orb_o()
        ref = np.array([o.orb_o(xw[w], terms) for w in range(W)])
        assert rel_err(g, ref) < 1e-10
        vec = np.hstack([eng.jas_o(), g])
        e = eng.state()[0]
        so = so + vec.sum(0)
        seo = seo + (e[:, None] * vec).sum(0)
        soo = soo + vec.T @ vec
    sums = eng.opt_sums(overlap=True)
    assert sums["wsum"] == 3 * W
    assert rel_err(sums["o"][nj:], so[nj:]) < 1e-10
    assert rel_err(sums["eo"], seo) < 1e-10
    assert rel_err(sums["oo"], soo) < 1e-10


def test_opt_orb_refusals():
    from champ_b200.engine import Engine, EngineError, initial_configs, rng_states
    from champ_b200.system import make_synthetic, rotation_expansion
    s = _with_virtuals(make_synthetic("tiny"), 2)
    e = Engine(s)
    with pytest.raises(EngineError, match="outside"):
        e.opt_orb([[1, 9]])
    with pytest.raises(EngineError, match="outside"):
        e.opt_orb([[2, 2]])
    rng = rng_states(4)
    e.set_walkers(initial_configs(s, rng), rng)
    with pytest.raises(EngineError, match="not enabled"):
        e.orb_o()


def _md32():
    from champ_b200.system import make_synthetic, rotation_expansion
    rots = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]
    md, _ = rotation_expansion(make_synthetic("tiny"), rots, extra_orbitals=4)
    md.cdet = np.random.default_rng(3).normal(size=md.cdet.shape) * 0.3
    md.cdet[0] = 1.0
    return _with_virtuals(md, 2, seed=8)


@pytest.mark.parametrize("config,W", [("md32", 16), ("c2", 4)])
def test_orb_derivatives_multideterminant(oracle_mod, config, W):
    """Expansions: the reference part plus detratio times the zmat / aaz
    terms of every varied pair, against the oracle at the start and after
    each of two sweeps, on a 32-determinant expansion with permuted
    orbitals and on the 10^4-determinant molecule."""
    from champ_b200.engine import Engine, initial_configs, rng_states
    from champ_b200.orbital_opt import orb_terms
    from champ_b200.system import make_synthetic
    s = _md32() if config == "md32" else make_synthetic("c2")
    terms = orb_terms(s, nadorb=2) if config == "md32" else orb_terms(s)[:200]
    assert len(terms) > 0
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    o = oracle_mod.OracleSystem(s)
    eng.opt_orb(terms)
    eng.opt_setup()
    for sweep in range(3):
        if sweep:
            eng.vmc_steps(1)
        xw, _ = eng.walkers()
        g = eng.orb_o()
        ref = np.array([o.orb_o(xw[w], terms) for w in range(W)])
        err = rel_err(g, ref)
        print(f"{config}: {len(terms)} pairs, sweep {sweep}: relative difference {err:.1e}")
        assert err < 1e-9
