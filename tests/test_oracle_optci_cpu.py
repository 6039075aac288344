"""CI-coefficient derivatives for wave-function optimisation (optci_deloc's
ci_o, SR sums of optwf_store) in the oracle, pinned by:

* linearity of psi in the CI coefficients: sum_k c_k d ln psi / d c_k = 1;
* central finite differences of ln psi with respect to each coefficient;
* the SR sums equal the weighted sums of the per-walker derivatives and
  local energies of every sweep."""
import copy

import numpy as np
import pytest

ROTS = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]


def _system():
    from champ_b200.system import make_synthetic, rotation_expansion
    md, _ = rotation_expansion(make_synthetic("tiny"), ROTS, extra_orbitals=4)
    md.cdet = np.random.default_rng(17).normal(size=md.cdet.shape)
    return md


def _walkers(oracle_mod, s, W):
    o = oracle_mod.OracleSystem(s)
    st = oracle_mod.rng_states(W)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    return o, np.array(xs), st


def test_ci_derivatives_linearity_and_fd(oracle_mod):
    s = _system()
    o, xs, st = _walkers(oracle_mod, s, 3)
    ws = oracle_mod.OracleWalkers(o, xs, st.copy())
    ci = ws.ci_o()
    for w in range(3):
        assert np.dot(s.cdet, ci[w]) == pytest.approx(1.0, abs=1e-12)
    eps = 1e-6
    for k in (0, 3, 11, 31):
        lp, lm = [], []
        for sgn, out in ((1, lp), (-1, lm)):
            t = copy.copy(s)
            t.cdet = s.cdet.copy()
            t.cdet[k] += sgn * eps
            t._keep = []
            ot = oracle_mod.OracleSystem(t)
            for x in xs:
                out.append(np.log(abs(ot.hpsi(x)["psid"])))
        fd = (np.array(lp) - np.array(lm)) / (2 * eps)
        assert np.allclose(fd, ci[:, k], rtol=1e-6, atol=1e-8), k


def test_sr_sums(oracle_mod):
    s = _system()
    o, xs, st = _walkers(oracle_mod, s, 4)
    ws = oracle_mod.OracleWalkers(o, xs, st.copy())
    ws.opt_ci(True)
    nd = s.cdet.size
    so, seo, soo, sw = np.zeros(nd), np.zeros(nd), np.zeros((nd, nd)), 0.0
    for _ in range(3):
        ws.steps(1, 1)
        ci = ws.ci_o()
        e = ws.state()[0]                            # eold of the sweep's hpsi
        so += ci.sum(0)
        soo += ci.T @ ci
        sw += ci.shape[0]
        seo += (e[:, None] * ci).sum(0)
    r = ws.opt_ci_sums()
    assert r["wsum"] == pytest.approx(sw)
    assert np.allclose(r["o"], so, rtol=1e-12, atol=1e-12)
    assert np.allclose(r["oo"], soo, rtol=1e-12, atol=1e-12)
    assert np.allclose(r["eo"], seo, rtol=1e-11, atol=1e-11)
    again = ws.opt_ci_sums()                         # read and reset
    assert again["wsum"] == 0 and not again["o"].any()


def test_sr_identities_and_step(oracle_mod):
    """S c = 0 and g . c = 0 (psi is linear in c); the SR step keeps the fixed
    coefficient and moves along -S^-1 g on the others."""
    from champ_b200 import optimize
    s = _system()
    o, xs, st = _walkers(oracle_mod, s, 6)
    ws = oracle_mod.OracleWalkers(o, xs, st.copy())
    ws.opt_ci(True)
    es = []
    for _ in range(4):
        ws.steps(1, 1)
        es.append(ws.state()[0])
    sums = ws.opt_ci_sums()
    e = float(np.mean(es))
    S, g = optimize.sr_matrices(sums, e)
    c = s.cdet
    assert np.max(np.abs(S @ c)) < 1e-9 * max(1.0, np.max(np.abs(S)))
    assert abs(g @ c) < 1e-9 * max(1.0, np.max(np.abs(g)))
    new = optimize.sr_step(sums, c, e, tau=0.05, adiag=0.01)
    assert new[0] == c[0]
    keep = np.arange(1, c.size)
    Sr = S[np.ix_(keep, keep)].copy()
    Sr[np.diag_indices_from(Sr)] *= 1.01
    assert np.allclose(Sr @ (new[1:] - c[1:]), -0.05 * g[1:], rtol=1e-8, atol=1e-12)
