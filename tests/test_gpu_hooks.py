"""Per-electron routines (cw_psie, cw_grad, cw_commit, cw_update_ymat)
against the oracle's psie / compute_determinante_grad / metrop6 accept
branch / update_ymat, move by move on identical inputs.

The test plays a Fortran driver that keeps metrop6's electron loop on the
host (vmc/metrop_mov1_slat.f90:131-630): for every electron it takes the
drift at the old position, proposes a point (a seeded Gaussian step), asks
for psi at the point and the drift there, decides with a Metropolis test on
the oracle's ratio, and commits the same decisions on both sides.  Both
walks therefore visit the same configurations whatever the sensitivity of
the trajectory, and every move's psi_D, J and drifts are compared:

* the 120-electron benchmark molecule with its model trial orbitals (four
  partner passes of the move Jastrow, 60x60 Sherman-Morrison commits);
* the 10^4-determinant, 40-electron molecule (1-4-fold excitations);
* a 37-electron chain (odd spin counts) and a 32-determinant expansion with
  permuted orbital lists;
* the 120-electron shapes with random orthonormal orbitals through the
  mixed path, with its stated bounds (the model-orbital molecule's FP32
  errors are amplified by its conditioning; its bounds are those of the
  mixed-path tests).

Tolerances (relative to max(1, |value|) for J and the drift, to |psi_D|):
FP64 1e-9 for psi_D and J and 1e-8 for the drift, or, where larger, thirty
times the oracle's own FP64 error on the same walk (the largest difference
between its Sherman-Morrison psi_D and a fresh hpsi, taken at four points
of the sweep).  The
engine applies Sherman-Morrison only on accepted moves and the oracle on
every proposal, as CHAMP does; the inverses then differ by rounding, which
the condition of the Slater matrix amplifies (row-normalised condition
numbers of 1e6 on the 120-electron model molecule, against 1e1 on a real
molecule with optimised orbitals); it amplifies the rounding of the
orbital values themselves (the two sides sum the LCAO in different orders,
and the model orbitals are sums of strongly cancelling terms): on that
molecule the two walks' psi_D differ by 3-13 times the oracle's own drift
and the drifts by up to 46 times, so its factor is 100.  The same shapes
with random orthonormal orbitals ("c1r") take the common factor.  Mixed path: psi_D 2e-3 (the
determinant bound), J 5e-5, drift 5e-4, or thirty times the oracle's FP64
error scaled by 1e7 (FP32 against FP64 rounding), where larger.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _systems(name):
    from champ_b200.system import make_chain, make_synthetic, rotation_expansion
    if name == "c1":
        return make_synthetic("c1")
    if name == "c1r":
        return make_synthetic("c1", orbitals="random")
    if name == "c2":
        return make_synthetic("c2")
    if name == "chain37":
        return make_chain(37, 4037)
    if name == "md32":
        rots = [(0, 2, 3, 0.3), (0, 1, 5, -0.25), (0, 0, 6, 0.15), (1, 1, 4, 0.2), (1, 0, 7, -0.1)]
        md, _ = rotation_expansion(make_synthetic("tiny"), rots, extra_orbitals=4)
        md.cdet = np.random.default_rng(3).normal(size=md.cdet.shape) * 0.3
        md.cdet[0] = 1.0
        return md
    raise ValueError(name)


def _drive(oracle_mod, s, W, precision, tol, sweeps=1, step=0.3, equil=10, seed=7, own_factor=30.0):
    from champ_b200.engine import Engine, initial_configs, rng_states
    rng = rng_states(W)
    x = initial_configs(s, rng)
    o = oracle_mod.OracleSystem(s)
    pre = oracle_mod.OracleWalkers(o, x, rng)
    pre.steps(equil, 8)
    x, rng = pre.walkers()
    eng = Engine(s, precision=precision)
    eng.set_walkers(x, rng)
    ow = oracle_mod.OracleWalkers(o, x, rng)
    gen = np.random.default_rng(seed)
    worst = dict(psid=0.0, psij=0.0, vold=0.0, vnew=0.0)
    own = 0.0
    nacc = 0
    xs = x.copy()
    for sw in range(sweeps):
        for i in range(s.nelec):
            vg = eng.grad(i, 1)
            vo = np.array([ow.grad(w, i, 1) for w in range(W)])
            worst["vold"] = max(worst["vold"], float(np.max(np.abs(vg - vo) / np.maximum(1.0, np.abs(vo)))))
            xnew = xs[:, i, :] + step * gen.normal(size=(W, 3))
            pg, jg = eng.psie(i, xnew)
            po, jo = np.zeros(W), np.zeros(W)
            for w in range(W):
                po[w], jo[w] = ow.psie(w, i, xnew[w])
            worst["psid"] = max(worst["psid"], float(np.max(np.abs(pg - po) / np.abs(po))))
            worst["psij"] = max(worst["psij"], float(np.max(np.abs(jg - jo) / np.maximum(1.0, np.abs(jo)))))
            vg = eng.grad(i, 0)
            vo = np.array([ow.grad(w, i, 0) for w in range(W)])
            worst["vnew"] = max(worst["vnew"], float(np.max(np.abs(vg - vo) / np.maximum(1.0, np.abs(vo)))))
            _, psido, psijo = ow.state()
            p = np.minimum(1.0, (po / psido) ** 2 * np.exp(2 * (jo - psijo)))
            acc = (gen.random(W) < p).astype(np.int32)
            nacc += int(acc.sum())
            eng.commit(i, acc)
            for w in range(W):
                ow.commit(w, i, acc[w], po[w], jo[w])
                ow.update_ymat(w, i)
            eng.update_ymat(i)
            xs[acc == 1, i, :] = xnew[acc == 1]
            if (i + 1) % max(1, s.nelec // 4) == 0 or i == s.nelec - 1:
                # the oracle's own FP64 error on this walk so far: its
                # Sherman-Morrison psi_D against a fresh full recompute
                _, po_sm, _ = ow.state()
                for w in range(W):
                    fresh = o.hpsi(xs[w])["psid"]
                    own = max(own, abs(po_sm[w] - fresh) / abs(fresh))
    scale = own_factor * own * (1.0 if precision == "fp64" else 1e7)
    tol = {k: max(t, scale) for k, t in tol.items()}
    print(f"{s.name} {precision}: worst relative differences {worst}, oracle's own error {own:.2e}, "
          f"{nacc} of {W * s.nelec * sweeps} accepted")
    for k, t in tol.items():
        assert worst[k] <= t, (k, worst[k], t)
    assert 0 < nacc < W * s.nelec * sweeps
    # the engine's walk is the host's walk
    xg, _ = eng.walkers()
    assert np.array_equal(xg, xs)
    # state after the moves, then the sweep's full recompute (hpsi)
    _, pg, jg = eng.state()
    _, po, jo = ow.state()
    assert np.max(np.abs(pg - po) / np.abs(po)) <= tol["psid"]
    assert np.max(np.abs(jg - jo) / np.maximum(1.0, np.abs(jo))) <= tol["psij"]
    h = eng.hpsi()
    for w in range(W):
        r = o.hpsi(xs[w])
        etol = max(1e-9, scale) if precision == "fp64" else max(5e-5, scale)
        assert abs(h["energy"][w] - r["energy"]) <= etol * max(1.0, abs(r["energy"]))
    return eng


FP64 = dict(psid=1e-9, psij=1e-9, vold=1e-8, vnew=1e-8)


@pytest.mark.parametrize("name,W,own_factor", [("c1r", 4, 30.0), ("c1", 4, 100.0), ("c2", 4, 30.0),
                                               ("chain37", 8, 30.0), ("md32", 8, 30.0)])
def test_hooks_fp64(oracle_mod, name, W, own_factor):
    _drive(oracle_mod, _systems(name), W, "fp64", FP64, own_factor=own_factor)


def test_hooks_mixed_c1r(oracle_mod):
    _drive(oracle_mod, _systems("c1r"), 4, "mixed", dict(psid=2e-3, psij=5e-5, vold=5e-4, vnew=5e-4))


def test_hooks_state_errors():
    """Calls out of order are refused, not guessed."""
    from champ_b200.engine import Engine, EngineError, initial_configs, rng_states
    from champ_b200.system import make_synthetic
    s = make_synthetic("tiny")
    eng = Engine(s)
    with pytest.raises(EngineError, match="no walkers"):
        eng.grad(0, 1)
    rng = rng_states(4)
    eng.set_walkers(initial_configs(s, rng), rng)
    with pytest.raises(EngineError, match="needs its cw_psie"):
        eng.grad(1, 0)
    with pytest.raises(EngineError, match="needs its cw_psie"):
        eng.commit(1, np.zeros(4, np.int32))
    with pytest.raises(EngineError, match="outside"):
        eng.psie(s.nelec, np.zeros((4, 3)))
    x, _ = eng.walkers()
    eng.psie(0, x[:, 0, :])
    with pytest.raises(EngineError, match="needs its cw_psie"):
        eng.commit(1, np.zeros(4, np.int32))
    eng.commit(0, np.ones(4, np.int32))   # same point: the walk stays where it was
    assert np.array_equal(eng.walkers()[0], x)
