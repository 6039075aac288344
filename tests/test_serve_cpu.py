"""Request loop (champ_b200.serve) on the host: admission against the HBM
budget, first-come-first-served order, round-robin blocks, completion by
target error or block budget, refusal of jobs larger than the budget.  A fake
engine and a virtual clock stand in for the GPU."""
import math

import numpy as np
import pytest

from champ_b200 import serve
from champ_b200.system import make_chain


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


class FakeEngine:
    """Each block costs `block_s` seconds; the error bar falls as 1/sqrt(blocks)."""

    def __init__(self, job, clock, log, block_s=0.01):
        self.job, self.clock, self.log, self.block_s = job, clock, log, block_s
        self.blocks = 0
        self.closed = False

    def device_bytes(self):
        return int(self.job.est_bytes * 0.9)

    def vmc_steps(self, n):
        self.clock.t += self.block_s
        self.log.append(self.job.jid)

    def end_block(self):
        self.blocks += 1

    def results(self):
        return dict(energy=-float(self.job.jid), err=0.01 / math.sqrt(self.blocks))

    def close(self):
        self.closed = True


def _jobs(specs):
    out = []
    for jid, (nelec, nwalk, arrival, target, cap) in enumerate(specs):
        out.append(serve.Job(jid=jid, system=make_chain(nelec, 100 + jid), nwalk=nwalk, target_err=target,
                             max_blocks=cap, nstep=2, arrival=arrival))
    return out


def _server(budget, clock, log):
    return serve.Server(budget, engine_factory=lambda j: FakeEngine(j, clock, log), clock=clock, sleep=clock.sleep,
                        executor=serve.InlineExecutor())


def test_budget_and_fifo_admission():
    clock, log = Clock(), []
    jobs = _jobs([(16, 256, 0.0, 0.004, 50), (16, 256, 0.0, 0.004, 50), (16, 256, 0.0, 0.004, 50)])
    one = serve.estimate_bytes(jobs[0].system, 256)
    srv = _server(2 * one + one // 2, clock, log)   # room for two of the three at a time
    srv.run(jobs)
    assert srv.peak_bytes <= srv.budget
    admits = [(t, j) for t, ev, j in srv.timeline if ev == "admit"]
    assert [j for _, j in admits] == [0, 1, 2]      # arrival order
    assert admits[0][0] == admits[1][0] == 0.0      # two fit at once
    first_done = min(t for t, ev, j in srv.timeline if ev == "done")
    assert admits[2][0] >= first_done               # the third waited for memory
    for j in jobs:
        assert j.reached and j.err <= j.target_err and j.blocks >= 2
        assert j.latency == j.done - j.arrival > 0


def test_round_robin_and_block_cap():
    clock, log = Clock(), []
    jobs = _jobs([(8, 64, 0.0, 1e-9, 3), (8, 64, 0.0, 1e-9, 5)])
    srv = _server(1 << 40, clock, log)
    srv.run(jobs)
    assert log[:4] == [0, 1, 0, 1]                  # blocks alternate
    assert [j.blocks for j in jobs] == [3, 5]       # capped, target out of reach
    assert not any(j.reached for j in jobs)


def test_arrivals_over_time_and_refusal():
    clock, log = Clock(), []
    jobs = _jobs([(8, 64, 0.5, 0.006, 20), (8, 64, 2.0, 0.006, 20), (64, 100000, 0.1, 0.006, 20)])
    small = serve.estimate_bytes(jobs[0].system, 64)
    srv = _server(4 * small, clock, log)
    out = srv.run(jobs)
    big = [j for j in out if j.nwalk == 100000][0]
    assert big.failed and big.blocks == 0           # larger than the whole budget: refused
    for j in out:
        if not j.failed:
            assert j.admitted >= j.arrival and j.reached
    s = serve.summary(out, clock.t)
    assert s["finished"] == 2 and s["refused"] == 1
    assert s["p50_s"] <= s["p99_s"]


def test_poisson_arrivals_seeded():
    a = serve.poisson_arrivals(50, 4.0, 7)
    b = serve.poisson_arrivals(50, 4.0, 7)
    assert np.array_equal(a, b) and np.all(np.diff(a) > 0)
    assert 50 / a[-1] == pytest.approx(4.0, rel=0.35)


def test_chain_generator_sizes():
    for n in (8, 37, 200):
        s = make_chain(n, 3)
        assert s.nelec == n and s.nup + s.ndn == n
        assert abs(s.nbasis / n - 4.5) < 0.6
        assert s.norb == s.nup


def test_failed_creation_does_not_stop_the_loop():
    clock, log = Clock(), []
    jobs = _jobs([(8, 64, 0.0, 0.006, 20), (8, 64, 0.0, 0.006, 20), (8, 64, 0.0, 0.006, 20)])

    def factory(j):
        if j.jid == 1:
            raise RuntimeError("cw_create failed (status 3): out of device memory")
        return FakeEngine(j, clock, log)

    srv = serve.Server(1 << 40, engine_factory=factory, clock=clock, sleep=clock.sleep,
                        executor=serve.InlineExecutor())
    out = srv.run(jobs)
    assert "out of device memory" in out[1].failed and out[1].blocks == 0
    assert out[0].reached and out[2].reached
    assert ("fail" in [ev for _, ev, j in srv.timeline if j == 1])


class BigEngine(FakeEngine):
    """A context that holds more than its job's estimate (multideterminant)."""

    def device_bytes(self):
        return 3 * serve.estimate_bytes(self.job.system, self.job.nwalk)


def test_charge_is_what_the_context_holds():
    clock, log = Clock(), []
    jobs = _jobs([(16, 256, 0.0, 0.004, 50), (16, 256, 0.0, 0.004, 50)])
    one = serve.estimate_bytes(jobs[0].system, 256)
    # the budget holds both estimates, but only one context of three times the estimate
    srv = serve.Server(4 * one, engine_factory=lambda j: BigEngine(j, clock, log), clock=clock, sleep=clock.sleep,
                        executor=serve.InlineExecutor())
    srv.run(jobs)
    assert srv.peak_bytes <= srv.budget
    admits = [t for t, ev, j in srv.timeline if ev == "admit"]
    first_done = min(t for t, ev, j in srv.timeline if ev == "done")
    assert len(admits) == 2 and admits[1] >= first_done   # the second waited for the real charge
    assert all(j.reached for j in jobs)
    # a context larger than the whole budget is refused after creation
    clock2, log2 = Clock(), []
    jb = _jobs([(16, 256, 0.0, 0.004, 50)])
    srv2 = serve.Server(2 * one, engine_factory=lambda j: BigEngine(j, clock2, log2), clock=clock2,
                        sleep=clock2.sleep, executor=serve.InlineExecutor())
    out = srv2.run(jb)
    assert out[0].failed and out[0].blocks == 0


class SleepEngine:
    """A block takes `block_s` seconds of wall time on a worker thread (the
    device's share of a real block), with the GIL released."""

    def __init__(self, job, block_s=0.05):
        import time
        self.job, self.block_s, self.sleep = job, block_s, time.sleep
        self.blocks = 0

    def device_bytes(self):
        return 0

    def vmc_steps(self, n):
        self.sleep(self.block_s)

    def end_block(self):
        self.blocks += 1

    def results(self):
        return dict(energy=-1.0, err=1.0)

    def close(self):
        pass


@pytest.mark.parametrize("slots", [1, 2, 4])
def test_worker_slots_overlap(slots):
    """Worker threads: every admitted job has a block in flight, at most
    `slots` at once, and blocks of different jobs overlap in time."""
    import time
    jobs = _jobs([(16, 64, 0.0, 1e-9, 3)] * 4)
    srv = serve.Server(1 << 40, engine_factory=lambda j: SleepEngine(j), slots=slots)
    t0 = time.perf_counter()
    srv.run(jobs)
    wall = time.perf_counter() - t0
    assert all(j.blocks == 3 and not j.failed for j in jobs)
    assert srv.peak_running == slots
    # the most blocks running at any instant
    ev = sorted([(s, 1) for _, s, e in srv.blocks] + [(e, -1) for _, s, e in srv.blocks], key=lambda x: (x[0], x[1]))
    most = run = 0
    for _, d in ev:
        run += d
        most = max(most, run)
    assert most == slots
    assert wall < 12 * 0.05 / slots + 0.3      # 12 blocks of 50 ms, `slots` at a time
