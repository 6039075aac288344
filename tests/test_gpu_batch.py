"""Batches of contexts (cw_batch_vmc_steps): the sweeps of several systems
as one CUDA graph of the contexts' own sweep graphs.  Every system's walk is
bitwise the one it takes alone, the contexts keep working on their own
afterwards, and a population change re-captures the batch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems():
    from champ_b200.system import make_chain, make_synthetic
    return [make_chain(16, 61), make_chain(21, 62), make_synthetic("tiny")]


def _engines(walkers):
    from champ_b200.engine import Engine, initial_configs, rng_states
    out = []
    off = 0
    for s, w in zip(_systems(), walkers):
        rng = rng_states(off + w)[off:].copy()
        off += w
        e = Engine(s)
        e.set_walkers(initial_configs(s, rng), rng)
        out.append(e)
    return out


def test_batch_matches_alone():
    from champ_b200.engine import Batch
    walkers = (64, 48, 32)
    alone = []
    for e in _engines(walkers):
        e.vmc_steps(3)
        e.end_block()
        e.vmc_steps(2)
        alone.append((e.walkers(), e.sums(), e.results()))
        e.close()
    engines = _engines(walkers)
    b = Batch(engines)
    b.vmc_steps(3)
    assert b.last_ms() > 0
    for e in engines:
        e.end_block()
    b.vmc_steps(1)
    for e in engines:
        e.vmc_steps(1)          # a context continues on its own after the batch
    for e, (wa, sa, ra) in zip(engines, alone):
        wb = e.walkers()
        assert np.array_equal(wb[0], wa[0]) and np.array_equal(wb[1], wa[1])
        assert np.array_equal(e.sums(), sa)
        assert e.results()["energy"] == ra["energy"]
    # a new population in one context: the batch re-captures it
    x, r = engines[2].walkers()
    engines[2].set_walkers(x[:16], r[:16])
    b.vmc_steps(1)
    b.close()
    for e in engines:
        e.close()
