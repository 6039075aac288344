"""GPU parity of multideterminant wave functions (compact excitation
tables, Y matrix, drift and energy corrections) against the oracle: a
32-determinant expansion with single to triple excitations in both spins,
random (non-factorizable) CI coefficients and permuted orbital lists, on
the ECP molecule; E_L, psi_D, the kinetic energy, VMC and DMC steps on
identical streams."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10
ROTS = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]


def _system(base="tiny", seed=3):
    from champ_b200.system import make_synthetic, rotation_expansion
    md, _ = rotation_expansion(make_synthetic(base), ROTS, extra_orbitals=4)
    md.cdet = np.random.default_rng(seed).normal(size=md.cdet.shape) * 0.3
    md.cdet[0] = 1.0
    return md


def _setup(oracle_mod, W):
    from champ_b200.engine import Engine, initial_configs, rng_states
    s = _system()
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    return s, eng, oracle_mod.OracleSystem(s), x, rng


def test_mdet_hpsi(oracle_mod):
    s, eng, o, x, _ = _setup(oracle_mod, 8)
    h = eng.hpsi()
    for w in range(x.shape[0]):
        r = o.hpsi(x[w])
        assert abs(h["psid"][w] - r["psid"]) <= TOL * abs(r["psid"])
        assert abs(h["energy"][w] - r["energy"]) <= TOL * max(1.0, abs(r["energy"])), (w, h["energy"][w], r["energy"])
        assert abs(h["ekin"][w] - r["ekin"]) <= TOL * max(1.0, abs(r["ekin"]))


def test_mdet_vmc_stream_parity(oracle_mod):
    s, eng, o, x, rng = _setup(oracle_mod, 16)
    ow = oracle_mod.OracleWalkers(o, x, rng)
    for step in range(3):
        eng.vmc_steps(1)
        ow.steps(1)
        xg, rg = eng.walkers()
        xo, ro = ow.walkers()
        assert np.array_equal(rg, ro), f"streams diverged at step {step}"
        assert rel_err(xg, xo) < 1e-9
        sg, so = eng.sums(), ow.sums()
        assert np.array_equal(sg[:, 4], so[:, 4])
        assert rel_err(sg[:, :4], so[:, :4]) < 1e-9


def test_mdet_dmc_parity(oracle_mod):
    from champ_b200.engine import Dmc, Engine, initial_configs, rng_states
    s = _system()
    W = 16
    o = oracle_mod.OracleSystem(s)
    st = rng_states(4 * W + 1)
    x = initial_configs(s, st[:W].copy())
    e0 = o.hpsi(x[0])["energy"]
    eng = Engine(s)
    dg = Dmc(eng, x, st[:4 * W], st[4 * W], tau=0.01, etrial=e0, mwalk=4 * W)
    do = oracle_mod.OracleDmc(o, x, st[:4 * W], st[4 * W], tau=0.01, etrial=e0, mwalk=4 * W)
    for step in range(4):
        dg.steps(1)
        do.steps(1)
        a, b = dg.walkers(), do.walkers()
        assert len(a[1]) == len(b[1]), step
        assert np.array_equal(a[3], b[3])
        assert rel_err(a[0], b[0]) < 1e-9
        assert rel_err(a[1], b[1]) < 1e-9
        assert rel_err(a[2], b[2]) < 1e-9


def test_c2_hpsi(oracle_mod):
    """The 10^4-determinant, 40-electron, 300-Gaussian, 80-orbital molecule."""
    from champ_b200.engine import Engine, initial_configs, rng_states
    from champ_b200.system import make_synthetic
    s = make_synthetic("c2")
    rng = rng_states(2)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    h = eng.hpsi()
    o = oracle_mod.OracleSystem(s)
    for w in range(2):
        r = o.hpsi(x[w])
        assert abs(h["psid"][w] - r["psid"]) <= 1e-9 * abs(r["psid"])
        assert abs(h["energy"][w] - r["energy"]) <= TOL * max(1.0, abs(r["energy"]))
