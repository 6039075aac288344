"""GPU stream parity at the shapes the benchmarks time.

The small-molecule parity tests run at most 8 electrons, where the move
Jastrow's partner loop makes a single pass and the Slater matrices are 4x4.
These cases run the same engine paths at the benchmark sizes against the
oracle, on identical electron configurations and random streams:

* 120 electrons, 30 centres, 540 Gaussians in VMC (FP64): partner loop in
  four passes, 60x60 Sherman-Morrison commits
  (vmc/metrop_mov1_slat.f90:131-630, vmc/determinante.f90:40-62);
* the same molecule through the mixed path: identical decisions except
  near-threshold ones, counted and bounded;
* the 10^4-determinant, 40-electron DMC molecule (FP64): 1-4-fold
  excitation solves in the multideterminant move kernels
  (dmc/dmc_ps_mov1.f90:293-447, vmc/multideterminante.f90:3-146);
* the 120-electron molecule in DMC and chains of 200 and 37 electrons in
  VMC (100x100 Slater matrices at the upper end of the batched job sizes).

metrop6 builds each proposal in a frame set by the drift component
perpendicular to the electron-nucleus axis; where that component is small
the frame, and so the proposed point, depends very strongly on the last
bits of the drift.  From unequilibrated starts, and for the atom-like model
trial orbitals of the benchmark molecules even after equilibration, the
oracle's own walk moves by 1e-5 .. 1e-3 relative within one sweep when its
start is perturbed by 1e-14, so walks of two correct implementations cannot
agree to 1e-9 there.  The VMC walk comparisons below therefore start from
configurations equilibrated by the oracle and use the same molecules with
seeded random orthonormal orbitals (same sizes and code paths, and a walk
that moves by 1e-11 under that perturbation); the model-orbital molecules
are compared move by move on identical inputs in test_gpu_hooks.py.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _vmc_pair(oracle_mod, s, W, precision="fp64", equil=10):
    """Engine and oracle walkers on identical configurations equilibrated by
    `equil` oracle sweeps from the sites start, with identical streams."""
    from champ_b200.engine import Engine, initial_configs, rng_states
    rng = rng_states(W)
    x = initial_configs(s, rng)
    o = oracle_mod.OracleSystem(s)
    if equil:
        ow = oracle_mod.OracleWalkers(o, x, rng)
        ow.steps(equil, 8)
        x, rng = ow.walkers()
    eng = Engine(s, precision=precision)
    eng.set_walkers(x, rng)
    ow = oracle_mod.OracleWalkers(o, x, rng)
    return eng, ow


def _stream_parity(eng, ow, steps, tol_x=1e-9, tol_e=1e-9):
    for step in range(steps):
        eng.vmc_steps(1)
        ow.steps(1, 8)
        xg, rg = eng.walkers()
        xo, ro = ow.walkers()
        assert np.array_equal(rg, ro), f"random streams diverged at step {step}"
        sg, so = eng.sums(), ow.sums()
        assert np.array_equal(sg[:, 4], so[:, 4]), f"acceptance counts differ at step {step}"
        assert rel_err(xg, xo) < tol_x
        eg, pg, jg = eng.state()
        eo, po, jo = ow.state()
        assert np.max(np.abs(eg - eo) / np.maximum(1.0, np.abs(eo))) < tol_e
        assert np.max(np.abs(jg - jo) / np.maximum(1.0, np.abs(jo))) < tol_e
        assert np.max(np.abs(pg - po) / np.abs(po)) < 1e-8
        assert rel_err(sg[:, :4], so[:, :4]) < tol_e
    return sg


def test_c1_vmc_stream_parity(oracle_mod):
    """120 electrons, FP64: same streams, decisions, positions and E_L."""
    from champ_b200.system import make_synthetic
    s = make_synthetic("c1", orbitals="random")
    eng, ow = _vmc_pair(oracle_mod, s, 4)
    sg = _stream_parity(eng, ow, 2)
    # both accepted and rejected moves occurred (commit and restore paths)
    assert 0 < sg[:, 4].sum() < 2 * 4 * s.nelec


def test_c1_mixed_decisions(oracle_mod):
    """120 electrons through the mixed path against the FP64 oracle for one
    sweep.  A decision can flip only where the FP64 acceptance probability
    lies within the mixed path's ratio error (about 1e-6 relative) of the
    uniform draw; a flipped walker's later proposals differ, so its stream
    diverges.  Bound: at most one of the 8 walkers (960 decisions); every
    other walker takes the oracle's decisions with positions within 1e-5
    and E_L within the mixed local-energy bound."""
    from champ_b200.system import make_synthetic
    s = make_synthetic("c1", orbitals="random")
    W = 8
    eng, ow = _vmc_pair(oracle_mod, s, W, precision="mixed")
    eng.vmc_steps(1)
    ow.steps(1, 8)
    xg, rg = eng.walkers()
    xo, ro = ow.walkers()
    sg, so = eng.sums(), ow.sums()
    same = np.all(rg == ro, axis=1) & (sg[:, 4] == so[:, 4])
    flipped = int(W - same.sum())
    print(f"c1 mixed: {flipped} of {W} walkers with a near-threshold flip")
    assert flipped <= 1
    eg, _, _ = eng.state()
    eo, _, _ = ow.state()
    for w in np.nonzero(same)[0]:
        assert rel_err(xg[w], xo[w]) < 1e-5
        assert abs(eg[w] - eo[w]) <= 5e-5 * max(1.0, abs(eo[w]))


def _dmc_pair(oracle_mod, s, W, vmc_steps, tau, precision="fp64"):
    from champ_b200.engine import Dmc, Engine
    o = oracle_mod.OracleSystem(s)
    mw = 4 * W
    st = oracle_mod.rng_states(mw + 2)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    vw = oracle_mod.OracleWalkers(o, np.array(xs), st[:W])
    vw.steps(vmc_steps, 8)
    x, r = vw.walkers()
    e0 = float(np.median(vw.state()[0]))
    rng = np.concatenate([r, st[W:mw]])
    dg = Dmc(Engine(s, precision=precision), x, rng, st[mw], tau=tau, etrial=e0, mwalk=mw)
    do = oracle_mod.OracleDmc(o, x, rng, st[mw], tau=tau, etrial=e0, mwalk=mw)
    return dg, do


def _dmc_compare(dg, do, step, tol=1e-9):
    xg, wg, eg, rg = dg.walkers()
    xo, wo, eo, ro = do.walkers()
    assert len(wg) == len(wo), f"population sizes differ at step {step}"
    assert np.array_equal(rg, ro), f"move streams diverged at step {step}"
    assert rel_err(xg, xo) < tol
    assert rel_err(wg, wo) < tol
    assert np.max(np.abs(eg - eo) / np.maximum(1.0, np.abs(eo))) < tol


def test_c2_dmc_parity(oracle_mod):
    """10^4 determinants (1-4-fold excitations), 40 electrons, FP64 DMC:
    identical populations, streams, weights, positions and energies."""
    from champ_b200.system import make_synthetic
    s = make_synthetic("c2")
    dg, do = _dmc_pair(oracle_mod, s, 4, 10, 0.01)
    for step in range(2):
        dg.steps(1)
        do.steps(1, 8)
        _dmc_compare(dg, do, step)
    assert dg.counts()["accepted"] > 0


def test_c1_dmc_parity(oracle_mod):
    """The 120-electron molecule through the DMC move kernels (FP64)."""
    from champ_b200.system import make_synthetic
    s = make_synthetic("c1")
    dg, do = _dmc_pair(oracle_mod, s, 4, 10, 0.01)
    for step in range(2):
        dg.steps(1)
        do.steps(1, 8)
        _dmc_compare(dg, do, step)


@pytest.mark.parametrize("nelec,orbitals", [(200, "random"), (37, "model")])
def test_chain_vmc_stream_parity(oracle_mod, nelec, orbitals):
    """Chain molecules of the batched job distribution: 200 electrons
    (100x100 Slater matrices, seven partner passes of the move Jastrow) and
    an odd count (19 up, 18 down) with its model trial orbitals."""
    from champ_b200.system import make_chain
    s = make_chain(nelec, 4000 + nelec, orbitals=orbitals)
    big = nelec > 100
    eng, ow = _vmc_pair(oracle_mod, s, 2 if big else 8, equil=4 if big else 10)
    _stream_parity(eng, ow, 1 if big else 2)


@pytest.mark.parametrize("nelec", [400, 333])
def test_large_spin_hpsi(oracle_mod, nelec):
    """Spins of 200 and 167 electrons, beyond what shared memory holds for
    the Slater inverse (matinv, vmc/matinv.f90:22-92) and c~: the engine
    factorises in the walker's own inverse block in global memory.  The
    odd count (167 up, 166 down) takes the per-spin c~ kernel.  Local
    energy, psi_D and the inverse against the oracle at the sites start."""
    from champ_b200.engine import Engine, initial_configs, rng_states
    from champ_b200.system import make_chain
    s = make_chain(nelec, 4000 + nelec, orbitals="random")
    W = 2
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s)
    eng.set_walkers(x, rng)
    o = oracle_mod.OracleSystem(s)
    h = eng.hpsi()
    slmi, det = eng.slater()
    r = o.hpsi(x[0])
    assert abs(h["energy"][0] - r["energy"]) <= 1e-9 * max(1.0, abs(r["energy"]))
    assert abs(h["psid"][0] - r["psid"]) <= 1e-9 * abs(r["psid"])
    rs, rdet = o.slater(x[0])
    for iab, nel in enumerate((s.nup, s.ndn)):
        assert rel_err(slmi[0, iab, :nel * nel], rs[iab, :nel * nel]) < 1e-9
        assert abs(det[0, iab] - rdet[iab]) <= 1e-9 * abs(rdet[iab])
    eng.vmc_steps(1)   # the move path at these sizes runs (untiled commit, global inverse)
    assert np.all(eng.walker_status() == 0)
