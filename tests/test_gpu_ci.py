"""The engine on CHAMP's VMC-C4H6-ci1010_pVTZ-00500-dets CI case (BFD
pseudopotentials, 500 determinants, f functions; the oracle is pinned on
it in test_oracle_ci_cpu.py): local energies against the oracle at 1e-10,
identical streams and decisions over sweeps, and a population of walkers
reaching CHAMP's reference energy within tools/compare_value.py's rule."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu


def _c4h6():
    from champ_b200.champ_io import load_npz
    return load_npz(os.path.join(GOLDEN, "vmc_c4h6_500_system.npz"))


def _equilibrated(oracle_mod, s, W, sweeps=20):
    o = oracle_mod.OracleSystem(s)
    rng = oracle_mod.rng_states(W)
    xs = []
    for w in range(W):
        x, rng[w] = o.sites(rng[w])
        xs.append(x)
    ow = oracle_mod.OracleWalkers(o, np.array(xs), rng)
    ow.steps(sweeps, 8)
    x, rng = ow.walkers()
    return o, x, rng


def test_c4h6_hpsi_and_streams(oracle_mod):
    from champ_b200.engine import Engine
    s = _c4h6()
    o, x, rng = _equilibrated(oracle_mod, s, 8)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    h = eng.hpsi()
    for w in range(8):
        r = o.hpsi(x[w])
        assert abs(h["energy"][w] - r["energy"]) <= 1e-10 * max(1.0, abs(r["energy"]))
        assert abs(h["psid"][w] - r["psid"]) <= 1e-10 * abs(r["psid"])
    eng.set_walkers(x, rng)
    ow = oracle_mod.OracleWalkers(o, x, rng)
    for step in range(3):
        eng.vmc_steps(1)
        ow.steps(1, 8)
        xg, rg = eng.walkers()
        xo, ro = ow.walkers()
        assert np.array_equal(rg, ro), f"streams diverged at step {step}"
        assert np.array_equal(eng.sums()[:, 4], ow.sums()[:, 4])
        assert rel_err(xg, xo) < 1e-9
        eg, _, _ = eng.state()
        eo, _, _ = ow.state()
        assert np.max(np.abs(eg - eo) / np.maximum(1.0, np.abs(eo))) < 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c4h6_energy_against_champ(precision):
    """2048 walkers from the sites start with CHAMP's default seed: 1
    equilibration block, 10 blocks of 20 steps.  The energy must agree with
    CHAMP's one-rank reference by compare_value.py's 2-sigma rule."""
    from champ_b200.engine import Engine, rng_states, start_population
    s = _c4h6()
    W = 2048
    eng = Engine(s, precision=precision)
    start_population(eng, s, rng_states(W))
    eng.vmc_steps(20)                       # equilibration block, discarded:
    x, rng = eng.walkers()
    eng.set_walkers(x, rng)                 # new population, estimators zeroed (zerest)
    for _ in range(10):
        eng.vmc_steps(20)
        eng.end_block()
    r = eng.results()
    e_ref, err_ref = -26.1993642, 0.0233401
    print(f"{precision}: engine {r['energy']:.5f} +- {r['err']:.5f} (sigma {r['sigma']:.3f}, "
          f"accept {r['accept']:.3f}), CHAMP {e_ref} +- {err_ref}")
    assert abs(r["energy"] - e_ref) <= 2.0 * np.sqrt(r["err"] ** 2 + err_ref ** 2)
