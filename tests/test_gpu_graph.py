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


def test_walkers_round_trip_through_caller_buffers():
    """cw_set_walkers / cw_get_walkers move positions in the caller's
    [W][N][3] layout (reordered on the device): the positions come back
    exactly, into new arrays or into the caller's (pinned) buffers."""
    import torch
    e, x, rng = _engine("c0", W=37)
    x0, r0 = e.walkers()
    assert np.array_equal(x0, x) and np.array_equal(r0, rng)
    xp = torch.empty(x.shape, dtype=torch.float64, pin_memory=True).numpy()
    rp = torch.empty(rng.shape, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    e.vmc_steps(1)
    out = e.walkers(xp, rp)
    assert out[0] is xp and out[1] is rp
    x1, r1 = e.walkers()
    assert np.array_equal(xp, x1) and np.array_equal(rp, r1)
    e.set_walkers(xp, rp)                # from pinned buffers: the same walkers back
    assert np.array_equal(e.walkers()[0], x1)
    with pytest.raises(ValueError):
        e.walkers(np.zeros((36, x.shape[1], 3)), rp)
    e.close()
