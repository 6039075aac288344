"""Ragged batches (cw_batch_set_ragged): the moves of systems of different
electron, centre, basis and orbital counts in one launch per move stage.
Every system takes the walk it takes alone: the same random streams and
accept/reject decisions, bitwise the same walk in mixed precision, and in
FP64 positions and sums equal to rounding (the move Jastrow and LCAO bodies
are compiled into kernels that read the system's constant block from global
memory instead of the parameter space, and the compiler may contract a
different set of multiply-adds: 1e-10 relative after four sweeps).  The LCAO
work items cover the tensor-core tiles and both SIMT shapes (orbital counts
above 16 and even, odd, and 16 or fewer), and systems that cannot join are
refused with the reason."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems():
    from champ_b200.system import make_chain, make_synthetic
    # orbitals: 20 (tensor-core tiles), 17 (odd: SIMT), 8, 4 and 11 (SIMT)
    return [make_chain(40, 63), make_chain(33, 64), make_chain(16, 61), make_synthetic("tiny"),
            make_chain(21, 62)]


def _engines(systems, walkers, precision="fp64"):
    from champ_b200.engine import Engine, initial_configs, rng_states
    out = []
    off = 0
    for s, w in zip(systems, walkers):
        rng = rng_states(off + w)[off:].copy()
        off += w
        e = Engine(s, precision=precision)
        e.set_walkers(initial_configs(s, rng), rng)
        out.append(e)
    return out


def _alone(systems, walkers, precision):
    out = []
    for e in _engines(systems, walkers, precision):
        e.vmc_steps(2)
        e.end_block()
        e.vmc_steps(2)
        out.append((e.walkers(), e.sums(), e.results()))
        e.close()
    return out


# FP64: relative agreement of positions, sums and energies with the walk alone
RTOL_FP64 = 1e-9


def _same_walk(e, wa, sa, ra, precision, i):
    wb = e.walkers()
    assert np.array_equal(wb[1], wa[1]), f"system {i}: random streams (decisions) differ"
    if precision == "mixed":
        assert np.array_equal(wb[0], wa[0]), f"system {i}: walk differs"
        assert np.array_equal(e.sums(), sa), f"system {i}: sums differ"
        assert e.results()["energy"] == ra["energy"]
        return
    scale = np.abs(wa[0]).max()
    assert np.abs(wb[0] - wa[0]).max() <= RTOL_FP64 * scale, f"system {i}: walk differs"
    assert np.allclose(e.sums(), sa, rtol=RTOL_FP64, atol=RTOL_FP64 * np.abs(sa).max()), f"system {i}: sums differ"
    assert abs(e.results()["energy"] - ra["energy"]) <= RTOL_FP64 * abs(ra["energy"])


def _check_ragged(systems, walkers, precision):
    from champ_b200.engine import Batch
    alone = _alone(systems, walkers, precision)
    engines = _engines(systems, walkers, precision)
    b = Batch(engines, ragged=True)
    b.vmc_steps(2)
    info = b.info()
    assert info["ragged"] and info["ragged_launches"] > 0 and info["system_launches"] > 0
    # one launch per move stage: six per electron of the largest system, plus rotqua
    nmax = max(s.nelec for s in systems)
    assert info["ragged_launches"] == 6 * nmax + 1
    if precision == "fp64":
        assert info["lcao_bn"] in (32, 48, 64, 80)
    assert b.last_ms() > 0
    for e in engines:
        e.end_block()
    b.vmc_steps(1)
    for e in engines:
        e.vmc_steps(1)          # a context continues on its own after the batch
    for i, (e, (wa, sa, ra)) in enumerate(zip(engines, alone)):
        _same_walk(e, wa, sa, ra, precision, i)
    # a new population in one system: the ragged graph is rebuilt for it
    x, r = engines[3].walkers()
    engines[3].set_walkers(x[:20], r[:20])
    b.vmc_steps(1)
    b.close()
    for e in engines:
        e.close()


def test_ragged_fp64_matches_alone():
    _check_ragged(_systems(), (96, 64, 48, 40, 72), "fp64")


def test_ragged_mixed_matches_alone():
    _check_ragged(_systems()[:3] + _systems()[4:], (80, 64, 48, 72), "mixed")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ragged_bands_match_alone(precision):
    """Three bands of systems, each its own chain of ragged launches."""
    from champ_b200.engine import Batch
    systems = _systems()
    walkers = (96, 64, 48, 40, 72)
    alone = _alone(systems, walkers, precision)
    engines = _engines(systems, walkers, precision)
    b = Batch(engines, ragged=3)
    b.vmc_steps(2)
    info = b.info()
    assert info["bands_asked"] == 3 and info["bands"] == 3
    nel = sorted((s.nelec for s in systems), reverse=True)
    assert 6 * nel[0] + 1 < info["ragged_launches"] <= 6 * sum(nel) + 1
    for e in engines:
        e.end_block()
    b.vmc_steps(2)
    for i, (e, (wa, sa, ra)) in enumerate(zip(engines, alone)):
        _same_walk(e, wa, sa, ra, precision, i)
    b.close()
    for e in engines:
        e.close()


def test_ragged_back_to_child_graphs():
    """Switching ragged mode off returns to the child-graph batch, same walk."""
    from champ_b200.engine import Batch
    systems = _systems()[:3]
    walkers = (40, 32, 24)
    alone = _alone(systems, walkers, "fp64")
    engines = _engines(systems, walkers)
    b = Batch(engines, ragged=True)
    b.vmc_steps(2)
    for e in engines:
        e.end_block()
    b.set_ragged(False)
    b.vmc_steps(2)
    assert not b.info()["ragged"]
    for i, (e, (wa, sa, ra)) in enumerate(zip(engines, alone)):
        _same_walk(e, wa, sa, ra, "fp64", i)
    b.close()
    for e in engines:
        e.close()


def test_ragged_refusals():
    from champ_b200.engine import Batch, EngineError
    from champ_b200.system import make_synthetic, rotation_expansion
    systems = _systems()[:2]
    e64 = _engines(systems[:1], (16,))[0]
    emx = _engines(systems[1:], (16,), "mixed")[0]
    b = Batch([e64, emx])
    with pytest.raises(EngineError, match="mix FP64 and mixed"):
        b.set_ragged(True)
    b.close()
    md, _ = rotation_expansion(make_synthetic("tiny"), [(0, 2, 3, 0.3), (1, 1, 4, 0.2)], extra_orbitals=4)
    emd = _engines([md], (16,))[0]
    b = Batch([e64, emd])
    with pytest.raises(EngineError, match="multideterminant"):
        b.set_ragged(True)
    b.vmc_steps(1)             # still usable as a child-graph batch
    b.close()
    for e in (e64, emx, emd):
        e.close()
