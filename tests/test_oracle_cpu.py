"""CPU tests: the oracle against the reference's golden vectors and its own
self-consistency; no GPU needed."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, rel_err


def test_matinv_golden(oracle_mod):
    # tests/unit_test/test_matinv.f90: identity and unit lower-triangular shear
    import ctypes as C
    L = oracle_mod.lib()
    a = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1], float)  # column-major a(3,3)
    det = np.zeros(1)
    assert L.or_matinv(oracle_mod.dp(a), 3, oracle_mod.dp(det)) == 0
    assert np.array_equal(a, [1, 0, 0, 0, 1, 0, 0, 0, 1]) and det[0] == 1.0
    b = np.array([1, 0, 0, 5, 1, 0, 0, 0, 1], float)
    assert L.or_matinv(oracle_mod.dp(b), 3, oracle_mod.dp(det)) == 0
    assert np.array_equal(b, [1, 0, 0, -5, 1, 0, 0, 0, 1]) and det[0] == 1.0


def test_matinv_random_vs_numpy(oracle_mod):
    rng = np.random.default_rng(7)
    for n in (1, 2, 3, 7, 20, 60):
        m = rng.normal(size=(n, n))
        a = np.asfortranarray(m).ravel(order="F").copy()
        det = np.zeros(1)
        assert oracle_mod.lib().or_matinv(oracle_mod.dp(a), n, oracle_mod.dp(det)) == 0
        inv = a.reshape(n, n, order="F")
        assert rel_err(inv, np.linalg.inv(m)) < 1e-10
        assert abs(det[0] - np.linalg.det(m)) <= 1e-9 * abs(np.linalg.det(m))


def test_pot_nn_water(oracle_mod):
    # tests/unit_test/test_electron_repulsion.f90: water, valence charges 6/1
    cent = np.array([[0.0, 0.0, 0.0], [-1.43042870599673, 0.0, -1.10715696499747],
                     [1.43042870599673, 0.0, -1.10715696499747]])
    znuc = np.array([6.0, 1.0])
    iw = np.array([0, 1, 1], np.int32)
    import ctypes as C
    pe = oracle_mod.lib().or_pot_nn(3, oracle_mod.dp(cent.ravel().copy()), oracle_mod.dp(znuc),
                                    iw.ctypes.data_as(C.POINTER(C.c_int32)))
    assert abs(np.float32(pe) - np.float32(6.98361052364638)) <= 1e-6
    from champ_b200.system import pot_nn
    assert abs(pot_nn(cent, znuc, iw) - pe) < 1e-13


def test_rng_golden(oracle_mod):
    z = np.load(os.path.join(GOLDEN, "rng_default_seed.npz"))
    st = oracle_mod.rng_states(4)
    assert np.array_equal(st, z["jump_states"])
    d = np.zeros(64)
    s0 = st[0].copy()
    oracle_mod.lib().or_rng_uniform(oracle_mod.u64(s0), 64, oracle_mod.dp(d))
    assert np.array_equal(d, z["draws"])


def test_rng_against_reference_c(oracle_mod):
    path = oracle_mod.REF_RNG
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (CHAMP sources absent)")
    import ctypes as C
    lib = C.CDLL(path)
    lib.next_uniform_double.restype = C.c_double
    irn = (C.c_int32 * 8)(*oracle_mod.seed_ints())
    lib.xoroshiro_set_state(irn)
    for _ in range(5):
        lib.jump()
    ref = [lib.next_uniform_double() for _ in range(1000)]
    st = oracle_mod.rng_states(6)[5].copy()
    d = np.zeros(1000)
    oracle_mod.lib().or_rng_uniform(oracle_mod.u64(st), 1000, oracle_mod.dp(d))
    assert np.array_equal(d, ref)


def test_nterms_and_cusp():
    from champ_b200.system import cuspexact4, cuspinit4, nterms4
    assert nterms4(5) == 23 and nterms4(2) == 2 and nterms4(0) == 0
    c = np.random.default_rng(1).normal(0, 0.05, size=(2, 23))
    cuspexact4(c, 5)
    d, iwc4, nt = cuspinit4(5)
    # every cusp constraint row of cuspinit4 is satisfied after cuspexact4
    for it in range(2):
        for i in range(1, 2 * (5 - 1) + 1):
            assert abs(np.dot(d[i, 1:], c[it])) < 1e-14


def _tiny(oracle_mod):
    from champ_b200.system import make_synthetic
    s = make_synthetic("tiny")
    return s, oracle_mod.OracleSystem(s)


def test_finite_difference_self_consistency(oracle_mod):
    s, o = _tiny(oracle_mod)
    st = oracle_mod.rng_states(1)
    x, _ = o.sites(st[0])
    psij, v, d2 = o.jastrow(x)
    orb, dorb, ddorb = o.orbitals(x)
    eps = 1e-5
    for i in range(s.nelec):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, k] += eps
            xm[i, k] -= eps
            g = (o.jastrow(xp)[0] - o.jastrow(xm)[0]) / (2 * eps)
            assert abs(g - v[i, k]) < 1e-7
            go = (o.orbitals(xp)[0][:, i] - o.orbitals(xm)[0][:, i]) / (2 * eps)
            assert np.max(np.abs(go - dorb[k, i, :])) < 1e-7
    h = o.hpsi(x)

    def psi(xx):
        r = o.hpsi(xx)
        return r["psid"] * np.exp(r["psij"])

    p0, lap, e2 = psi(x), 0.0, 1e-4
    for i in range(s.nelec):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, k] += e2
            xm[i, k] -= e2
            lap += (psi(xp) - 2 * p0 + psi(xm)) / e2 ** 2
    assert abs(-0.5 * lap / p0 - h["ekin"]) < 1e-5 * max(1.0, abs(h["ekin"]))


def _h2_run(oracle_mod, nranks):
    from champ_b200.champ_io import load_npz
    s = load_npz(os.path.join(GOLDEN, "vmc_h2_system.npz"))
    o = oracle_mod.OracleSystem(s)
    st = oracle_mod.rng_states(nranks)
    xs, sts = [], []
    for r in range(nranks):
        x, s2 = o.sites(st[r])
        xs.append(x)
        sts.append(s2)
    w = oracle_mod.OracleWalkers(o, np.array(xs), np.array(sts))
    w.steps(50)
    w.end_block()
    w.zerest()
    for _ in range(200):
        w.steps(50)
        w.end_block()
    return w.results()


@pytest.mark.parametrize("nranks,eref,sref", [(1, -1.0046458, 0.0084583), (2, -1.0090406, 0.0054465)])
def test_h2_ci_energy(oracle_mod, nranks, eref, sref):
    # tests/CI_test/VMC-H2/VMC_H2_STO-CVB1_energy_hydrogen.sh, judged with
    # tools/compare_value.py:26: |E - E_ref| <= 2 sqrt(err^2 + err_ref^2)
    r = _h2_run(oracle_mod, nranks)
    assert abs(r["energy"] - eref) <= 2 * np.sqrt(r["err"] ** 2 + sref ** 2)
    assert 0.5 < r["accept"] < 0.95
