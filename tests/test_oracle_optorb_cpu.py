"""Orbital-rotation derivatives (optorb_deriv for one determinant,
vmc/optorb.f90:5-95) of the oracle, pinned by finite differences of ln psi_D
under phi_io -> phi_io + a phi_jo, and optorb_define's selection of the
varied pairs (vmc/optorb.f90:838-1030) on closed- and open-shell cases."""
import copy

import numpy as np
import pytest


def _with_virtuals(s, n, seed=5):
    """The molecule with n extra (virtual) orbitals appended to its LCAO."""
    rng = np.random.default_rng(seed)
    t = copy.deepcopy(s)
    t.coef = np.vstack([np.asarray(s.coef, float), rng.normal(size=(n, s.coef.shape[1])) * 0.3])
    t._keep = []
    return t


def _lnpsid(oracle_mod, s, x):
    return np.log(abs(oracle_mod.OracleSystem(s).hpsi(x)["psid"]))


@pytest.mark.parametrize("config", ["tiny", "c0"])
def test_orb_o_finite_differences(oracle_mod, config):
    from champ_b200.engine import initial_configs, rng_states
    from champ_b200.orbital_opt import apply_step, orb_terms
    from champ_b200.system import make_synthetic
    s = _with_virtuals(make_synthetic(config), 3)
    terms = orb_terms(s, nadorb=3)
    assert len(terms) > 0
    rng = rng_states(3)
    x = initial_configs(s, rng)
    o = oracle_mod.OracleSystem(s)
    h = 1e-5
    for w in range(3):
        d = o.orb_o(x[w], terms)
        for t in range(len(terms)):
            da = np.zeros(len(terms))
            da[t] = h
            fp = _lnpsid(oracle_mod, apply_step(s, terms, da), x[w])
            fm = _lnpsid(oracle_mod, apply_step(s, terms, -da), x[w])
            fd = (fp - fm) / (2 * h)
            assert abs(d[t] - fd) <= 1e-6 * max(1.0, abs(fd)), (w, tuple(terms[t]), d[t], fd)


def test_orb_terms_rules():
    from champ_b200.orbital_opt import orb_terms
    from champ_b200.system import make_synthetic
    # closed shell, 4 doubly occupied orbitals + 3 external ones: only
    # occupied -> external pairs
    c0 = _with_virtuals(make_synthetic("c0"), 3)
    t = orb_terms(c0, nadorb=3)
    assert {tuple(v) for v in t} == {(io, jo) for io in range(1, 5) for jo in range(5, 8)}
    assert orb_terms(c0).shape == (0, 2)           # no external orbitals: nothing to mix in
    assert len(orb_terms(c0, nadorb=3, ncore=1)) == 9   # orbital 1 frozen as a core
    # open shell (3 up on orbitals 1-3, 2 down on 1-2): orbital 3 is singly
    # occupied, so (1,3) and (2,3) are varied (down spin holds 1, 2 without 3)
    # and (3,1), (3,2) are not (every spin holding 3 also holds 1 and 2)
    tiny = _with_virtuals(make_synthetic("tiny"), 2)
    t = {tuple(v) for v in orb_terms(tiny, nadorb=2)}
    assert (1, 3) in t and (2, 3) in t and (3, 1) not in t and (3, 2) not in t
    assert (3, 5) in t and (1, 5) in t and (5, 1) not in t
    # symmetry labels: pairs of different labels are dropped
    lab = [0, 1, 0, 1, 0, 1, 0, 1, 0]
    t2 = orb_terms(tiny, nadorb=2, irrep=lab)
    assert all(lab[a - 1] == lab[b - 1] for a, b in t2)


def test_orb_step_first_order(oracle_mod):
    """A small step along the derivatives changes ln psi_D by O . da."""
    from champ_b200.engine import initial_configs, rng_states
    from champ_b200.orbital_opt import apply_step, orb_terms
    from champ_b200.system import make_synthetic
    s = _with_virtuals(make_synthetic("tiny"), 2)
    terms = orb_terms(s, nadorb=2)
    rng = rng_states(2)
    x = initial_configs(s, rng)
    o = oracle_mod.OracleSystem(s)
    da = np.random.default_rng(1).normal(size=len(terms)) * 1e-6
    for w in range(2):
        pred = o.orb_o(x[w], terms) @ da
        got = _lnpsid(oracle_mod, apply_step(s, terms, da), x[w]) - _lnpsid(oracle_mod, s, x[w])
        assert abs(got - pred) <= 1e-3 * abs(pred) + 1e-12


def _md32():
    from champ_b200.system import make_synthetic, rotation_expansion
    rots = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]
    md, _ = rotation_expansion(make_synthetic("tiny"), rots, extra_orbitals=4)
    md.cdet = np.random.default_rng(3).normal(size=md.cdet.shape) * 0.3
    md.cdet[0] = 1.0
    return _with_virtuals(md, 2, seed=8)


def test_orb_o_finite_differences_multideterminant(oracle_mod):
    """Expansions (optorb_deriv's zmat and aaz terms, compute_zmat): d ln psi
    / d a of every varied pair of a 32-determinant expansion with permuted
    orbital lists against central differences of the expansion's psi_D."""
    from champ_b200.engine import initial_configs, rng_states
    from champ_b200.orbital_opt import apply_step, orb_terms
    s = _md32()
    terms = orb_terms(s, nadorb=2)
    assert len(terms) > 0
    rng = rng_states(3)
    x = initial_configs(s, rng)
    o = oracle_mod.OracleSystem(s)
    h = 1e-5
    worst = 0.0
    for w in range(3):
        d = o.orb_o(x[w], terms)
        for t in range(len(terms)):
            da = np.zeros(len(terms))
            da[t] = h
            fp = _lnpsid(oracle_mod, apply_step(s, terms, da), x[w])
            fm = _lnpsid(oracle_mod, apply_step(s, terms, -da), x[w])
            fd = (fp - fm) / (2 * h)
            worst = max(worst, abs(d[t] - fd) / max(1.0, abs(fd)))
            assert abs(d[t] - fd) <= 1e-6 * max(1.0, abs(fd)), (w, tuple(terms[t]), d[t], fd)
    print(f"{len(terms)} pairs, worst difference {worst:.1e}")
