"""GPU parity of the Jastrow parameter derivatives (deriv_jastrow4's gvalue)
and of the SR sums over the optimisation vector [Jastrow | CI] against the
oracle on identical streams: raw derivatives and mapped parameters at every
walker, then the sums of three VMC sweeps (sum O, sum E_L O, sum O O^T)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
ROTS = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]


def _engine(s, W):
    from champ_b200.engine import Engine, initial_configs, rng_states
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    return eng, x, rng


@pytest.mark.parametrize("config,W,nspin2b", [("tiny", 16, 1), ("c0", 8, 1), ("tiny", 16, 2)])
def test_jastrow_derivatives(oracle_mod, config, W, nspin2b):
    from champ_b200 import jastrow_opt as jo
    from champ_b200.system import make_synthetic
    s = make_synthetic(config)
    if nspin2b == 2:                                  # like / unlike spin e-e functions
        s.nspin2b = 2
        b = np.array(s.b, float)
        s.b = np.vstack([b[:1], b[:1] * 0.8 + 0.01])
        s.b[1, 0] = 0.25
    eng, x, _ = _engine(s, W)
    jd = jo.default_jasderiv(s)
    P = jo.param_map(s, jd)
    eng.opt_setup(ci=False, jas_map=P, overlap=True)
    o = oracle_mod.OracleSystem(s)
    xg, _ = eng.walkers()
    raw_o = np.array([o.jas_raw(xg[w]) for w in range(W)])
    raw_g = eng.jas_raw()
    assert raw_g.shape == raw_o.shape
    assert rel_err(raw_g, raw_o) < 1e-11
    assert rel_err(eng.jas_o(), raw_o @ P) < 1e-11


def test_sr_sums_jastrow_and_ci(oracle_mod):
    from champ_b200 import jastrow_opt as jo
    from champ_b200.system import make_synthetic, rotation_expansion
    s, _ = rotation_expansion(make_synthetic("tiny"), ROTS, extra_orbitals=4)
    s.cdet = np.random.default_rng(17).normal(size=s.cdet.shape)
    W = 16
    eng, x, rng = _engine(s, W)
    jd = jo.default_jasderiv(s)
    P = jo.param_map(s, jd)
    eng.opt_setup(ci=True, jas_map=P, overlap=True)
    osys = oracle_mod.OracleSystem(s)
    ow = oracle_mod.OracleWalkers(osys, x, rng)
    ow.opt_ci(True)
    assert rel_err(eng.ci_o(), ow.ci_o()) < 1e-10
    nj, nd = jd.nparmj, s.cdet.shape[0]
    so, seo, soo = np.zeros(nj + nd), np.zeros(nj + nd), np.zeros((nj + nd, nj + nd))
    for _ in range(3):
        eng.vmc_steps(1)
        ow.steps(1)
        xo, _ = ow.walkers()
        e, _, _ = ow.state()
        ojas = np.array([osys.jas_raw(xo[w]) for w in range(W)]) @ P
        O = np.hstack([ojas, ow.ci_o()])
        so += O.sum(0)
        seo += (e[:, None] * O).sum(0)
        soo += O.T @ O
    a = eng.opt_sums(overlap=True)
    assert a["wsum"] == 3 * W
    assert rel_err(a["o"], so) < 1e-9
    assert rel_err(a["eo"], seo) < 1e-9
    assert rel_err(a["oo"], soo) < 1e-9
    # the CI block agrees with the oracle's own CI sums
    b = ow.opt_ci_sums()
    assert rel_err(a["o"][nj:], b["o"]) < 1e-9
    assert rel_err(a["oo"][nj:, nj:], b["oo"]) < 1e-9


def test_opt_setup_refusals():
    from champ_b200 import jastrow_opt as jo
    from champ_b200.engine import EngineError
    from champ_b200.system import make_synthetic
    s = make_synthetic("tiny")
    eng, _, _ = _engine(s, 4)
    with pytest.raises(EngineError):
        eng.opt_setup(ci=True)                   # one determinant: no CI parameters
    with pytest.raises(ValueError):
        eng.opt_setup(jas_map=np.zeros((3, 2)))  # map rows must match the raw vector
    P = jo.param_map(s, jo.default_jasderiv(s))
    eng.opt_setup(jas_map=P)
    eng.opt_setup()                              # disable
    with pytest.raises(EngineError):
        eng.jas_o()


def test_sr_optimize_loop():
    """The optwf loop on the GPU: parameters move, the cusp conditions hold
    after every step, energies stay finite."""
    from champ_b200 import jastrow_opt as jo
    from champ_b200 import optimize
    from champ_b200.system import cuspinit4, make_synthetic
    s = make_synthetic("tiny")
    jd = jo.default_jasderiv(s)
    t, hist = optimize.sr_optimize(s, jd, nwalk=128, iters=3, nblock=2, nstep=5, tau=0.02)
    assert len(hist) == 3 and all(np.isfinite(e) and np.isfinite(err) for e, err in hist)
    assert not np.array_equal(t.c, s.c)
    d, _, _ = cuspinit4(s.nordc)
    assert np.max(np.abs(d[1:, 1:] @ t.c.T)) < 1e-12
