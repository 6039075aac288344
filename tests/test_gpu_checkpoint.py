"""Checkpoint / restart (the role of CHAMP's dumper / startr): a run that is
checkpointed, restored into a fresh context and continued is identical to
the uninterrupted run — walkers, streams, estimators, DMC population."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_vmc_restart_bitwise():
    from champ_b200.engine import Engine, initial_configs, rng_states
    from champ_b200.system import make_synthetic
    s = make_synthetic("c0")
    rng = rng_states(32)
    x = initial_configs(s, rng)
    a = Engine(s)
    a.set_walkers(x, rng)
    a.vmc_steps(2)
    a.end_block()
    a.vmc_steps(1)
    ck = a.checkpoint()
    a.vmc_steps(2)
    a.end_block()
    b = Engine(s)
    b.restore(ck)
    b.vmc_steps(2)
    b.end_block()
    xa, ra = a.walkers()
    xb, rb = b.walkers()
    assert np.array_equal(xa, xb) and np.array_equal(ra, rb)
    assert a.results() == b.results()


def test_dmc_restart_bitwise():
    from champ_b200.engine import Dmc, Engine, initial_configs, rng_states
    from champ_b200.system import make_synthetic
    s = make_synthetic("tiny")
    W, mw = 32, 128
    rng = rng_states(mw + 1)
    x = initial_configs(s, rng[:W].copy())
    a = Engine(s)
    da = Dmc(a, x, rng[:mw], rng[mw], tau=0.01, etrial=50.0, mwalk=mw)
    da.steps(3)
    da.end_block()
    da.steps(1)
    ck = a.checkpoint()
    da.steps(3)
    da.end_block()
    b = Engine(s)
    b.restore(ck)
    db = Dmc.attach(b, mw)
    db.steps(3)
    db.end_block()
    wa, wb = da.walkers(), db.walkers()
    for u, v in zip(wa, wb):
        assert np.array_equal(u, v)
    assert da.results() == db.results()


def test_restore_rejects_other_system():
    from champ_b200.engine import Engine, EngineError, initial_configs, rng_states
    from champ_b200.system import make_synthetic
    s, t = make_synthetic("c0"), make_synthetic("tiny")
    rng = rng_states(4)
    a = Engine(s)
    a.set_walkers(initial_configs(s, rng), rng)
    ck = a.checkpoint()
    b = Engine(t)
    with pytest.raises(EngineError, match="different system"):
        b.restore(ck)
    with pytest.raises(EngineError, match="not a checkpoint"):
        b.restore(b"x" * 64)
