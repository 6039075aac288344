"""GPU parity of the CI-coefficient derivatives and stochastic-reconfiguration
sums (optci_deloc's ci_o, optwf_store) against the oracle on identical
streams; the overlap sum is one FP64 GEMM over the walkers per sweep."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
ROTS = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]


def _system():
    from champ_b200.system import make_synthetic, rotation_expansion
    md, _ = rotation_expansion(make_synthetic("tiny"), ROTS, extra_orbitals=4)
    md.cdet = np.random.default_rng(17).normal(size=md.cdet.shape)
    return md


def test_ci_derivatives_and_sr_sums(oracle_mod):
    from champ_b200.engine import Engine, initial_configs, rng_states
    s = _system()
    W = 16
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    ow = oracle_mod.OracleWalkers(oracle_mod.OracleSystem(s), x, rng)
    eng.opt_ci(True, overlap=True)
    ow.opt_ci(True)
    cg, co = eng.ci_o(), ow.ci_o()
    assert rel_err(cg, co) < 1e-10
    assert np.allclose(cg @ s.cdet, 1.0, atol=1e-11)          # psi is linear in the coefficients
    for _ in range(3):
        eng.vmc_steps(1)
        ow.steps(1)
    a, b = eng.opt_ci_sums(), ow.opt_ci_sums()
    assert a["wsum"] == b["wsum"] == 3 * W
    for k in ("o", "eo", "oo"):
        assert rel_err(a[k], b[k]) < 1e-9, k
    assert np.allclose(a["oo"], a["oo"].T, rtol=1e-12, atol=1e-12)
    z = eng.opt_ci_sums()                                     # read and reset
    assert z["wsum"] == 0 and not z["o"].any()


def test_opt_ci_refusals():
    from champ_b200.engine import Engine, EngineError, initial_configs, rng_states
    from champ_b200.system import make_synthetic
    s = make_synthetic("tiny")                                # one determinant
    rng = rng_states(4)
    e = Engine(s)
    e.set_walkers(initial_configs(s, rng), rng)
    with pytest.raises(EngineError):
        e.opt_ci(True)
