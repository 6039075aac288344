"""Request loop for VMC energy jobs on one GPU (continuous admission).

A job is a system, a walker count, a target error bar and a block budget.
Jobs arrive over time.  A job is admitted as soon as its device-memory
estimate fits into what the HBM budget has left, first come first served (a
job never overtakes an earlier one that does not fit yet).  From then on it
keeps its engine context -- walker population, Slater inverses, Jastrow
tables, accumulators -- resident on the device until it finishes.  At most
``slots`` jobs are admitted at a time; every admitted job has one block in
flight (a block is ``nstep`` sweeps followed by the block average, CHAMP's
acuest), issued from a worker thread on the job's own CUDA stream, so the
blocks of different jobs run on the device at the same time (each kernel
carries its own system's constants).  Newly arrived jobs are admitted
whenever a block ends.  A job finishes when its error bar reaches the target
(after at least two blocks) or its block budget is spent; its context is
then released and the jobs waiting for memory or a slot are admitted.

A job is charged the larger of its estimate and the bytes its context
really holds (``cw_device_bytes``, read after creation): the estimate is an
upper bound for single-determinant systems only, so a multideterminant job
whose context turns out larger than what is left is released again and waits,
first in line, for that much memory.  A job whose context creation or block
fails (out of device memory, a singular walker) is marked failed and the
loop serves the others.

Time-to-result of a job = completion time - arrival time.  Each job draws
its walkers' streams from its own range (``seed_offset``), so a job's
result does not depend on which other jobs share the device.

``executor`` replaces the worker threads (``InlineExecutor`` runs the blocks
in flight one after the other on the loop's own thread: the round-robin
order of a single host thread, used by the host-side tests).
CHAMP itself has no request loop (one job per MPI run); this module is the
serving layer the engine's C ABI is designed for.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import dataclasses
import itertools
import math
import time

import numpy as np


@dataclasses.dataclass
class Job:
    jid: int
    system: object
    nwalk: int
    target_err: float
    max_blocks: int
    nstep: int = 10
    arrival: float = 0.0        # seconds after the loop starts
    seed_offset: int = 0        # first random stream of the job's walkers
    # filled in by the server
    est_bytes: int = 0
    device_bytes: int = 0
    admitted: float = math.nan
    done: float = math.nan
    energy: float = math.nan
    err: float = math.nan
    blocks: int = 0
    moves: int = 0
    reached: bool = False
    failed: str = ""

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def estimate_bytes(system, nwalk: int, precision: str = "fp64", chunk_bytes: int = 1 << 30) -> int:
    """Device bytes a context of `system` with `nwalk` walkers allocates: the
    walker state, move and local-energy scratch of the engine (the same
    arrays, one value per element), plus the system tables (radial grids,
    coefficients), with a 10% margin.  An upper bound of cw_device_bytes for
    single-determinant jobs."""
    N, M, K, O = system.nelec, system.ncent, system.nbasis, system.norb
    nmax = max(system.nup, system.ndn)
    NQ = max(int(getattr(system, "nquad", 0) or 0), 1)
    W = nwalk
    d = 8
    walker = (3 * N + 4 + 3 * NQ + N + N + 3 * N + 5 + 2 * nmax * nmax + 2 + N * nmax + 3 * N * nmax
              + N * N + 3 * N * N + 3 * N + 1 + 2 * M * N + 8 + 1)
    move = 64 + N + 3 * N + 3 * N + 1 + 3 + 4 * K + 4 * O + 2 * M
    hpsi = 1 + 1 + 1 + 2 + 4 * N + N * nmax + 5 * M * N
    if getattr(system, "nloc", 0):
        hpsi += N * K
    per_e = W * 5 * (K + O) * d
    chunk = min(max(1, chunk_bytes // max(per_e, 1)), N)
    scratch = W * chunk * 5 * (K + O)
    total = d * (W * (walker + move + hpsi) + scratch)
    if precision == "mixed":
        kp = (K + 31) // 32 * 32
        total += 4 * (2 * W * 4 * kp + 2 * W * chunk * 5 * kp) + 8 * O * kp
    rwf = np.asarray(system.rwf)
    tables = 8 * (2 * rwf.size + rwf.shape[0] * (rwf.shape[-1] + 1) + K * O * 3 + nmax * K) + (1 << 20)
    return int(1.10 * (total + tables))


def _engine_for(job: Job, precision: str, device: int):
    from .engine import Engine, rng_states, start_population
    eng = Engine(job.system, device=device, precision=precision)
    rng = rng_states(job.seed_offset + job.nwalk)[job.seed_offset:].copy()
    start_population(eng, job.system, rng)
    return eng


def _block(eng, nstep: int):
    """One block of a job: (block averages, device-clock start and end in ns,
    or None where the engine keeps no device clock)."""
    stamp = getattr(eng, "stamp", None)
    if stamp:
        stamp()
    eng.vmc_steps(nstep)
    eng.end_block()
    if stamp:
        stamp()
    r = eng.results()
    dev = tuple(int(v) for v in eng.stamps()[-2:]) if stamp else None
    return r, dev


class InlineExecutor:
    """Runs the submitted calls on the calling thread, one after the other in
    submission order, when the server waits for them."""

    def __init__(self):
        self.queue = []

    def submit(self, fn, *args):
        f = cf.Future()
        self.queue.append((f, fn, args))
        return f

    def wait(self, fs, timeout=None, return_when=cf.FIRST_COMPLETED):
        queue, self.queue = self.queue, []
        for f, fn, args in queue:
            try:
                f.set_result(fn(*args))
            except Exception as exc:
                f.set_exception(exc)
        return set(fs), set()

    def shutdown(self, wait: bool = True):
        pass


class Server:
    """One GPU, one HBM budget; `run` serves a list of jobs with arrival times,
    at most `slots` of them on the device at once."""

    def __init__(self, budget_bytes: int, precision: str = "fp64", device: int = 0, engine_factory=None,
                 clock=time.perf_counter, sleep=time.sleep, slots: int = 8, executor=None):
        self.budget = int(budget_bytes)
        self.precision = precision
        self.device = device
        self.factory = engine_factory or (lambda job: _engine_for(job, precision, device))
        self.clock = clock
        self.sleep = sleep
        self.slots = max(1, int(slots))
        self.executor = executor
        self.peak_bytes = 0          # largest sum of admitted estimates
        self.peak_running = 0        # most jobs with a block in flight at once
        self.timeline = []           # (time, event, job id)
        self.blocks = []             # (job id, start, end) of every block, host clock
        self.device_blocks = []      # (job id, start ns, end ns) of every block, device clock

    def run(self, jobs):
        jobs = sorted(jobs, key=lambda j: (j.arrival, j.jid))
        for j in jobs:
            j.est_bytes = estimate_bytes(j.system, j.nwalk, self.precision)
        pending = collections.deque(jobs)
        waiting = collections.deque()
        inflight = {}                  # future -> (submission number, job, engine, start time)
        seq = itertools.count()
        used = 0
        pool = self.executor or cf.ThreadPoolExecutor(max_workers=self.slots)
        t0 = self.clock()

        def now():
            return self.clock() - t0

        def submit(j, eng):
            start = now()
            inflight[pool.submit(_block, eng, j.nstep)] = (next(seq), j, eng, start)
            self.peak_running = max(self.peak_running, len(inflight))

        def arrive_and_admit():
            nonlocal used
            t = now()
            while pending and pending[0].arrival <= t:
                j = pending.popleft()
                waiting.append(j)
                self.timeline.append((t, "arrive", j.jid))
            while waiting and len(inflight) < self.slots:
                j = waiting[0]
                if j.est_bytes > self.budget:      # can never fit: refuse, do not block the queue
                    waiting.popleft()
                    j.failed = f"needs {j.est_bytes} bytes, budget {self.budget}"
                    j.done = now()
                    self.timeline.append((j.done, "refuse", j.jid))
                    continue
                if used + j.est_bytes > self.budget:
                    break
                waiting.popleft()
                try:
                    eng = self.factory(j)
                except Exception as exc:           # e.g. out of device memory: this job fails, the loop goes on
                    j.failed = f"context creation failed: {exc}"
                    j.done = now()
                    self.timeline.append((j.done, "fail", j.jid))
                    continue
                j.device_bytes = int(eng.device_bytes())
                # the estimate bounds single-determinant contexts only: charge
                # what the context really holds when that is more
                charge = max(j.est_bytes, j.device_bytes)
                if used + charge > self.budget:
                    eng.close()
                    j.est_bytes = charge
                    if charge > self.budget:
                        j.failed = f"holds {charge} bytes, budget {self.budget}"
                        j.done = now()
                        self.timeline.append((j.done, "refuse", j.jid))
                        continue
                    waiting.appendleft(j)          # waits, first in line, for the memory it really needs
                    break
                j.est_bytes = charge
                used += charge
                self.peak_bytes = max(self.peak_bytes, used)
                j.admitted = now()
                self.timeline.append((j.admitted, "admit", j.jid))
                submit(j, eng)

        try:
            while pending or waiting or inflight:
                arrive_and_admit()
                if not inflight:
                    if pending:
                        self.sleep(max(0.0, pending[0].arrival - now()))
                    continue
                timeout = max(0.0, pending[0].arrival - now()) if pending else None
                done, _ = getattr(pool, "wait", cf.wait)(list(inflight), timeout=timeout,
                                                         return_when=cf.FIRST_COMPLETED)
                for f in sorted(done, key=lambda f: inflight[f][0]):
                    _, j, eng, start = inflight.pop(f)
                    end = now()
                    self.blocks.append((j.jid, start, end))
                    try:
                        r, dev = f.result()
                    except Exception as exc:           # a failed block ends this job only
                        j.failed = f"block failed: {exc}"
                        j.done = end
                        self.timeline.append((j.done, "fail", j.jid))
                        eng.close()
                        used -= j.est_bytes
                        continue
                    if dev:
                        self.device_blocks.append((j.jid, *dev))
                    j.blocks += 1
                    j.moves += j.nstep * j.nwalk * j.system.nelec
                    j.energy, j.err = float(r["energy"]), float(r["err"])
                    j.reached = j.blocks >= 2 and j.err <= j.target_err
                    if j.reached or j.blocks >= j.max_blocks:
                        j.done = end
                        self.timeline.append((j.done, "done", j.jid))
                        eng.close()
                        used -= j.est_bytes
                    else:
                        submit(j, eng)
        finally:
            if self.executor is None:
                pool.shutdown(wait=True)
        return jobs


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    """Arrival times (s) of n jobs of a Poisson stream with `rate` jobs/s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def summary(jobs, makespan: float) -> dict:
    """p50/p99 time-to-result of the finished jobs and aggregate throughput."""
    ok = [j for j in jobs if not j.failed]
    lat = np.array([j.latency for j in ok]) if ok else np.zeros(1)
    moves = sum(j.moves for j in ok)
    return dict(p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
                mean_s=float(lat.mean()), jobs=len(jobs), finished=len(ok),
                reached_target=sum(1 for j in ok if j.reached), refused=len(jobs) - len(ok),
                moves_per_s=moves / makespan if makespan > 0 else 0.0, makespan_s=makespan)
