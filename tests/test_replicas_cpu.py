"""Replicas on several devices (one process per GPU) exchange only the
timing maximum and the final estimate.  Two gloo processes on the host
exercise the same plumbing: disjoint per-rank random streams, max over
ranks, and the inverse-variance merge of each rank's VMC estimate."""
import json
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys
    root = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
    sys.path.insert(0, root)
    from champ_b200.replicas import Replicas, rank_streams
    from champ_b200.system import make_synthetic
    from oracle import oracle
    rep = Replicas(backend="gloo", timeout_s=60)
    s = make_synthetic("tiny")
    o = oracle.OracleSystem(s)
    W = 4
    st = rank_streams(rep.rank, W, oracle.rng_states)
    xs = []
    for w in range(W):
        x, st[w] = o.sites(st[w])
        xs.append(x)
    ow = oracle.OracleWalkers(o, np.array(xs), st)
    for _ in range(3):
        ow.steps(2)
        ow.end_block()
    r = ow.results()
    e, err = rep.merged_energy(r["energy"], r["err"])
    tmax = rep.max(float(rep.rank + 1))
    rep.barrier()
    rep.close()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump(dict(streams=rank_streams(rank, W, oracle.rng_states).tolist(), energy=r["energy"], err=r["err"],
                       merged=[e, err], tmax=tmax), f)


def test_two_gloo_replicas(tmp_path, oracle_mod):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    r = [json.load(open(tmp_path / f"r{k}.json")) for k in range(2)]
    s0, s1 = np.array(r[0]["streams"], np.uint64), np.array(r[1]["streams"], np.uint64)
    assert not (set(map(tuple, s0)) & set(map(tuple, s1))), "replicas share a random stream"
    assert np.array_equal(np.vstack([s0, s1]), oracle_mod.rng_states(8))
    from champ_b200.replicas import merge_estimates
    e, err = merge_estimates([r[0]["energy"], r[1]["energy"]], [r[0]["err"], r[1]["err"]])
    for k in range(2):
        assert r[k]["merged"] == pytest.approx([e, err], rel=1e-12)
        assert r[k]["tmax"] == 2.0
