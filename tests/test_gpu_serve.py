"""Request loop on the GPU: a job's result is the same alone and in a mix of
jobs sharing the device (bitwise: each job owns its walker streams and its
context), jobs are admitted against the HBM budget, and the memory estimate
bounds what a context really allocates."""
import pytest

from champ_b200 import serve
from champ_b200.system import make_chain

pytestmark = pytest.mark.gpu


def _jobs(arrivals=(0.0, 0.0, 0.0)):
    specs = [(8, 96, 0), (14, 64, 96), (21, 64, 160)]   # (electrons, walkers, first stream)
    return [serve.Job(jid=i, system=make_chain(n, 40 + i), nwalk=w, target_err=0.0, max_blocks=3, nstep=4,
                      arrival=arrivals[i], seed_offset=off)
            for i, (n, w, off) in enumerate(specs)]


def test_result_same_alone_and_in_mix():
    alone = []
    for j in _jobs():
        srv = serve.Server(1 << 34)
        (done,) = srv.run([j])
        alone.append((done.energy, done.err, done.blocks))
    mixed = serve.Server(1 << 34).run(_jobs(arrivals=(0.0, 0.01, 0.02)))
    for a, m in zip(alone, sorted(mixed, key=lambda j: j.jid)):
        assert (m.energy, m.err, m.blocks) == a


def test_budget_admission_and_estimate():
    jobs = _jobs()
    for j in jobs:
        j.est_bytes = serve.estimate_bytes(j.system, j.nwalk)
    budget = jobs[0].est_bytes + jobs[1].est_bytes + jobs[2].est_bytes // 2
    srv = serve.Server(budget)
    out = srv.run(jobs)
    assert srv.peak_bytes <= budget
    admits = {j: t for t, ev, j in srv.timeline if ev == "admit"}
    dones = {j: t for t, ev, j in srv.timeline if ev == "done"}
    assert admits[2] >= min(dones[0], dones[1])        # the third job waited for memory
    for j in out:
        assert not j.failed and j.blocks == 3
        assert 0 < j.device_bytes <= j.est_bytes         # the estimate bounds the allocation
        assert j.est_bytes <= 3 * j.device_bytes


def test_larger_context_runs_after_smaller_one_is_created():
    """Kernel shared-memory limits are per device: creating a smaller system's
    context must not shrink what an earlier, larger context launches with."""
    from champ_b200.engine import Engine, initial_configs, rng_states
    big, small = make_chain(48, 5), make_chain(8, 6)
    engines = []
    for s in (big, small):
        rng = rng_states(32)
        e = Engine(s)
        e.set_walkers(initial_configs(s, rng), rng)
        engines.append(e)
    for e in engines:
        e.vmc_steps(1)
    for e in engines:
        e.close()
