"""Jastrow parameter derivatives of the oracle (deriv_jastrow4's gvalue),
pinned by:

* the cusp tables against the listing of dependent and varied e-e-n terms
  in the reference's cuspexact4 header (vmc/cuspexact4.f90:1-30);
* central finite differences of J = ln psi_J for every raw coefficient
  (a, b, c taken on their own, the asymptotic constants following a and b);
* central finite differences of J for every varied parameter of a jasderiv
  selection, the cusp-fixed e-e-n terms recomputed after each perturbation
  (cuspexact4) -- this checks the checkdepend4 map;
* the parser of the jasderiv block."""
import numpy as np
import pytest

from champ_b200 import jastrow_opt as jo
from champ_b200.system import cuspinit4, make_synthetic, nterms4


def _conf(oracle_mod, s, seed=3):
    o = oracle_mod.OracleSystem(s)
    st = oracle_mod.rng_states(seed + 1)
    x, _ = o.sites(st[seed])
    return o, x


def _J(oracle_mod, s, x):
    return oracle_mod.OracleSystem(s).jastrow(x)[0]


def test_cusp_tables_match_reference_listing():
    ee = [1, 4, 10, 19, 32, 49]
    en = [2, 6, 12, 22, 35, 53]
    for nord, ncum, nfree in ((5, 23, 15), (6, 37, 27), (7, 55, 43)):
        d, iwc4, nt = cuspinit4(nord)
        assert nt == nterms4(nord) == ncum
        assert iwc4[1:nord] == ee[:nord - 1]
        assert iwc4[nord:2 * nord - 1] == en[:nord - 1]
        s = make_synthetic("tiny")
        s.nordc = nord
        free = jo.default_jasderiv(s).iwjasc[0]
        assert len(free) == nfree
    s = make_synthetic("tiny")
    assert jo.default_jasderiv(s).iwjasc[0] == [3, 5, 7, 8, 9, 11, 13, 14, 15, 16, 17, 18, 20, 21, 23]
    with pytest.raises(ValueError):
        jo.checkdepend4(5, [[1, 3]])      # a cusp-fixed term may not be varied


def _perturbed(s, part, idx, h):
    import copy
    t = copy.copy(s)
    t.a4, t.b, t.c = np.array(s.a4, float).copy(), np.array(s.b, float).copy(), np.array(s.c, float).copy()
    getattr(t, part)[idx] += h
    t._keep = []
    return t


def _two_spin_classes(s):
    """Separate e-e functions for like and unlike spins (nspin2b = 2)."""
    s.nspin2b = 2
    b = np.array(s.b, float)
    s.b = np.vstack([b[:1], b[:1] * 0.8 + 0.01])
    s.b[1, 0] = 0.25                 # like-spin cusp
    s._keep = []
    return s


@pytest.mark.parametrize("nspin2b", [1, 2])
def test_raw_derivatives_finite_differences(oracle_mod, nspin2b):
    s = make_synthetic("tiny")
    if nspin2b == 2:
        _two_spin_classes(s)
    o, x = _conf(oracle_mod, s)
    raw = o.jas_raw(x)
    lay = jo.raw_layout(s)
    assert raw.size == lay["nraw"]
    h = 1e-5
    checked = 0
    for r in range(lay["nraw"]):
        if r < lay["b"]:
            part, idx = "a4", divmod(r - lay["a"], lay["NA"])
        elif r < lay["c"]:
            part, idx = "b", divmod(r - lay["b"], lay["NB"])
        else:
            part, idx = "c", divmod(r - lay["c"], lay["NT"])
        fd = (_J(oracle_mod, _perturbed(s, part, idx, h), x) -
              _J(oracle_mod, _perturbed(s, part, idx, -h), x)) / (2 * h)
        assert abs(fd - raw[r]) <= 2e-7 * max(1.0, abs(raw[r])), (part, idx, fd, raw[r])
        checked += 1
    assert checked == lay["nraw"]


def test_param_map_finite_differences(oracle_mod):
    s = make_synthetic("tiny")
    o, x = _conf(oracle_mod, s, seed=5)
    jd = jo.default_jasderiv(s)
    P = jo.param_map(s, jd)
    g = o.jas_raw(x) @ P
    h = 1e-5
    for k in range(jd.nparmj):
        e = np.zeros(jd.nparmj)
        e[k] = h
        fd = (_J(oracle_mod, jo.apply_step(s, jd, e), x) - _J(oracle_mod, jo.apply_step(s, jd, -e), x)) / (2 * h)
        assert abs(fd - g[k]) <= 2e-7 * max(1.0, abs(g[k])), (k, fd, g[k])


def test_apply_step_keeps_cusp_conditions():
    s = make_synthetic("tiny")
    jd = jo.default_jasderiv(s)
    t = jo.apply_step(s, jd, np.random.default_rng(1).normal(0, 0.01, jd.nparmj))
    d, iwc4, nt = cuspinit4(s.nordc)
    for it in range(s.nctype):
        assert np.max(np.abs(d[1:, 1:] @ t.c[it])) < 1e-12
    # a(1), b(1) are not in the default selection and stay put
    assert np.array_equal(t.a4[:, 0], s.a4[:, 0]) and np.array_equal(t.b[:, 0], s.b[:, 0])


def test_read_jasderiv():
    text = """# comment line
jasderiv
4 4 5 15 0 0 0
3 4 5 6
3 4 5 6
2 3 4 5 6
3 5 7 8 9 11 13 14 15 16 17 18 20 21 23

end
"""
    jd = jo.read_jasderiv(text, nctype=2)
    assert jd.iwjasa == [[3, 4, 5, 6], [3, 4, 5, 6]]
    assert jd.iwjasb == [[2, 3, 4, 5, 6]]
    assert jd.iwjasc == [[3, 5, 7, 8, 9, 11, 13, 14, 15, 16, 17, 18, 20, 21, 23], []]
    assert jd.nparmj == 4 + 4 + 5 + 15
    with pytest.raises(ValueError):
        jo.read_jasderiv("nothing here", nctype=1)


def test_sr_delta_over_the_joint_vector(oracle_mod):
    """SR step over [Jastrow | CI]: sums of oracle samples of the tiny
    system's Jastrow derivatives; the step is a descent direction of the
    SR metric (g . dp = -tau g S^-1 g < 0) and leaves the held entry."""
    from champ_b200 import optimize
    s = make_synthetic("tiny")
    o = oracle_mod.OracleSystem(s)
    P = jo.param_map(s, jo.default_jasderiv(s))
    st = oracle_mod.rng_states(24)
    O, E = [], []
    for w in range(24):
        x, _ = o.sites(st[w])
        O.append(o.jas_raw(x) @ P)
        E.append(o.hpsi(x)["energy"])
    O, E = np.array(O), np.array(E)
    sums = dict(o=O.sum(0), eo=(E[:, None] * O).sum(0), oo=O.T @ O, wsum=float(len(E)))
    S, g = optimize.sr_matrices(sums, E.mean())
    dp = optimize.sr_delta(sums, E.mean(), tau=0.05, adiag=0.1, fixed=3)
    assert dp[3] == 0.0
    keep = [k for k in range(len(g)) if k != 3]
    assert g[keep] @ dp[keep] < 0
