"""Independent walker populations on several GPUs (one process per GPU).

The walk is embarrassingly parallel: CHAMP runs one Markov chain per MPI rank
(VMC) or one population per rank (DMC, dmc_one_mpi1).  Here each rank drives
one GPU with its own population; the only exchanges are the timing (maximum
over ranks) and the final estimate, merged by inverse variance.

* ``rank_streams``   random streams of a rank: streams r*W .. r*W+W-1 of the
                     seed (CHAMP's rank streams, seed jumped once per stream),
                     so replicas never share a stream.
* ``merge_estimates`` inverse-variance mean of per-rank (E, err) pairs.
* ``Replicas``       torch.distributed plumbing: NCCL on GPUs, gloo on CPUs
                     (the tests run two gloo processes on the host).
"""
from __future__ import annotations

import datetime
import os

import numpy as np


def rank_streams(rank: int, nwalk: int, streams_fn):
    """Streams of `rank` among replicas of `nwalk` walkers each."""
    allr = streams_fn(nwalk * (rank + 1))
    return np.ascontiguousarray(allr[rank * nwalk:(rank + 1) * nwalk])


def merge_estimates(values, errors):
    """Inverse-variance mean and its error of independent estimates."""
    v = np.asarray(values, float)
    e = np.asarray(errors, float)
    if np.any(e <= 0):
        return float(np.mean(v)), 0.0
    wts = 1.0 / e ** 2
    return float(np.sum(wts * v) / np.sum(wts)), float(1.0 / np.sqrt(np.sum(wts)))


class Replicas:
    """Rank/world from the launcher's environment (torchrun); a process group
    only when world_size > 1."""

    def __init__(self, backend: str | None = None, timeout_s: int = 300):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.backend = backend
        if self.world > 1:
            import torch.distributed as dist
            self.backend = backend or ("nccl" if self._cuda() else "gloo")
            if self.backend == "nccl":
                import torch
                torch.cuda.set_device(self.local)
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = dist

    @staticmethod
    def _cuda():
        try:
            import torch
            return torch.cuda.is_available()
        except Exception:
            return False

    def _device(self):
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.pg is not None:
            self.pg.barrier()
        if self.backend == "nccl" or (self.pg is None and self._cuda()):
            import torch
            torch.cuda.synchronize(self.local)

    def max(self, v: float) -> float:
        if self.pg is None:
            return float(v)
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=self._device())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if self.pg is None:
            return float(v)
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=self._device())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def merged_energy(self, energy: float, err: float):
        """Inverse-variance merge of every rank's (energy, err), on every rank."""
        if self.pg is None:
            return float(energy), float(err)
        import torch
        t = torch.tensor([energy, err], dtype=torch.float64, device=self._device())
        out = [torch.zeros_like(t) for _ in range(self.world)]
        self.pg.all_gather(out, t)
        vals = [float(x[0]) for x in out]
        errs = [float(x[1]) for x in out]
        return merge_estimates(vals, errs)

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()
            self.pg = None
