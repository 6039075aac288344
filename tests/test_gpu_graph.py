"""The captured CUDA graph of a VMC sweep replays exactly the launches of the
direct path: walkers, streams and sums are bitwise identical whether the
sweeps run as one graph launch each or launch by launch (the profiled path),
and a new population or enabling the optimisation sums re-captures."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine(cfg="c0", W=64):
    from champ_b200.engine import Engine, initial_configs, rng_states
    from champ_b200.system import make_synthetic
    s = make_synthetic(cfg)
    rng = rng_states(W)
    x = initial_configs(s, rng)
    e = Engine(s)
    e.set_walkers(x, rng)
    return e, x, rng


@pytest.mark.parametrize("cfg", ["c0", "tiny"])
def test_graph_replay_matches_direct_launches(cfg):
    a, x, rng = _engine(cfg)
    b, _, _ = _engine(cfg)
    a.profile(True)                      # launch by launch
    for _ in range(2):
        a.vmc_steps(2)
        b.vmc_steps(2)                   # captured once, replayed
    xa, ra = a.walkers()
    xb, rb = b.walkers()
    assert np.array_equal(ra, rb) and np.array_equal(xa, xb)
    assert np.array_equal(a.sums(), b.sums())
    assert a.launches() == b.launches() > 0
    b.set_walkers(x, rng)                # new population: re-capture
    a.set_walkers(x, rng)
    a.vmc_steps(1)
    b.vmc_steps(1)
    assert np.array_equal(a.walkers()[0], b.walkers()[0])
