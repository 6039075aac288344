"""Tile autotuner (cw_autotune): each context times the N tiles of its FP64
tensor-core LCAO contraction on its own shapes and keeps the fastest.  The
choice changes no result: walks of a tuned and an untuned context from the
same walkers and streams stay bitwise identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TILES = {32, 48, 64, 80}


@pytest.mark.parametrize("name,W", [("chain37", 256), ("c2sd", 128)])
def test_autotune_keeps_results(name, W):
    from champ_b200.engine import Engine, initial_configs, rng_states
    from champ_b200.system import make_chain, make_synthetic
    if name == "chain37":
        s = make_chain(37, 4037)
    else:
        s = make_synthetic("c2")
        s.iworbd, s.cdet = s.iworbd[:1].copy(), s.cdet[:1].copy()
    rng = rng_states(W)
    x = initial_configs(s, rng)
    out = {}
    for tuned in (False, True):
        e = Engine(s)
        e.set_walkers(x, rng)
        if tuned:
            choice = e.autotune(3)
            print(f"{name}: tiles {choice} for {s.norb} orbitals")
            assert choice["lcao_move_tile"] in TILES and choice["lcao_all_tile"] in TILES
        e.vmc_steps(2)
        out[tuned] = (e.walkers(), e.sums(), e.state()[0])
        e.close()
    (xa, ra), sa, ea = out[False]
    (xb, rb), sb, eb = out[True]
    assert np.array_equal(ra, rb) and np.array_equal(xa, xb)
    assert np.array_equal(sa, sb) and np.array_equal(ea, eb)
