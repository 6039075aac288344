"""Throughput benchmark of the B200 walker engine (VMC, electron-moves/s).

A step is one metrop6 sweep (vmc/metrop_mov1_slat.f90:3): every electron of
every walker offered one accelerated-Metropolis move, then the full local
energy (hpsi) and the weighted sums.  Default workload: the 120-electron,
30-centre, 540-Gaussian synthetic molecule with 8192 walkers.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times CHAMP's own CPU algorithm for the same workload.  The
CHAMP Fortran build needs gfortran/MPI, absent on this image, so the timed CPU
implementation is the FP64 C++ restatement in oracle/ (kind "port") run with
one walker per host thread, as CHAMP runs one walker per MPI rank.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (synthetic config, walkers, description)
    "c1": ("c1", 8192, "vmc-c1: 30 centres on a zig-zag chain (15 Cl-like Z=7 with BFD-form ECP, 15 H-like; "
                       "neutral), 120 electrons (60/60), 540 Gaussians, 60 orbitals (model-Hamiltonian trial "
                       "orbitals), order-5 Jastrow, 8192 walkers"),
    "c0": ("c0", 1024, "vmc-c0: 3 centres (Z 6/1/1, ECP on the heavy atom), 8 electrons (4/4), 60 Gaussians, "
                       "4 orbitals, order-5 Jastrow, 1024 walkers"),
    "c2": ("c2", 16384, "dmc-c2: 12 centres (9 C-like Z=4 with BFD-form ECP, 3 H-like), 40 electrons (20/20), "
                        "300 Gaussians, 80 orbitals (model-Hamiltonian trial orbitals), 10^4 determinants "
                        "(1-4-fold excitations, |c_k|~k^-1.5), "
                        "order-5 Jastrow, 16384 walkers, tau=0.01, branching on"),
    "c3": ("chain", 0, "batched-c3: 64 chain molecules of seeded sizes (8-200 electrons, ~4.5 x electrons "
                       "Gaussians, Cl-like Z=7 with BFD-form ECP and H-like centres, seeded random orthonormal "
                       "orbitals, order-5 Jastrow), 256-4096 walkers each, all resident at once; a step is one "
                       "sweep of every system, issued concurrently on one stream per system"),
    "c4": ("chain", 0, "serve-c4: seeded Poisson arrivals of VMC energy jobs, each a chain molecule of the "
                       "batched distribution (8-200 electrons, ~4.5 x electrons Gaussians, Cl-like Z=7 with ECP "
                       "and H-like centres), 256-1024 walkers, target error 0.5 mHa within a block budget, "
                       "admitted against an HBM budget on one GPU"),
}


def jm_traffic(W):
    """DRAM bytes per k_jastrow_move launch at W walkers, from the committed ncu
    capture (per-walker traffic: the e-n table and pair rows of each walker)."""
    p = os.path.join(ROOT, "profiles", "k_jastrow_move_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return (d["dram_bytes_read"] + d["dram_bytes_write"]) * W / d["walkers"]


def update_bytes(system, W, acc):
    """Bytes one k_decide + k_commit pair moves at W walkers and acceptance
    `acc` in the engine's lazy update: k_decide reads the inverse column (n),
    the new orbital rows (4 O) and the move scratch (~12 doubles) and writes
    the state of an accepted walker (~N: position, nearest-centre rows);
    k_commit, for the accepted walkers only, reads and writes the spin's
    inverse (2 n^2), the column and orbital row (2 n), the orbital and
    gradient rows of the electron (8 n), the e-n row (2 M) and the pair
    table rows (fso, fijo, fjo: 14 N)."""
    N, M, O = system.nelec, system.ncent, system.norb
    n = max(system.nup, system.ndn)
    decide = 8 * (n + 4 * O + 12 + N)
    commit = 8 * (2 * n * n + 2 * n + 8 * n + 2 * M + 14 * N)
    return W * (decide + acc * commit)


def update_traffic(W):
    """DRAM bytes of one k_decide + k_commit pair at W walkers, from the
    committed ncu capture (per-walker traffic scaled by the walker count)."""
    p = os.path.join(ROOT, "profiles", "k_decide_commit_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d["dram_bytes_per_pair"] * W / d["walkers"]


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def algorithmic(system, W):
    """Work per launch of the move-stage kernels (FP64 reference algorithm)."""
    N, M, K, O = system.nelec, system.ncent, system.nbasis, system.norb
    T = system.c.shape[1] if system.c.ndim == 2 else 0
    ns = max(system.nup, system.ndn)
    f_jastrow_move = 8 * (N - 1) * M * T + 8 * (N - 1) * system.nordb + 8 * M * system.norda
    f_move = 2 * 4 * K * O + 30 * K + 2 * ns + 2 * ns * ns + f_jastrow_move + 6 * ns
    b_move = 8 * (2 * ns * ns + 6 * N + 8 * (N - 1) + 4 * O)
    f_jastrow_full = 9 * N * (N - 1) * M * T
    return dict(f_jastrow_move=W * f_jastrow_move, f_move=W * f_move, b_move=W * b_move,
                f_jastrow_full=W * f_jastrow_full)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in (self.out or "").splitlines():
            p = [v.strip() for v in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                smax.append(float(p[1]))
            except ValueError:
                continue
            for nm, v in zip(names, p[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(ngpus):
    """One process per GPU (torchrun): the replica plumbing of champ_b200.replicas."""
    from champ_b200.replicas import Replicas
    rep = Replicas()
    return rep.rank, rep.world, rep.local, rep


def max_over_ranks(v, rep, local):
    return rep.max(v)


def barrier(rep, local):
    rep.barrier()


def cpu_port_rate(system, walkers_cpu, nthreads, min_seconds=10.0, max_steps=4, seed_offset=0, warm_sweeps=1):
    """Oracle (FP64 C++ restatement of CHAMP) on host threads: electron-moves/s."""
    from oracle import oracle
    oracle.build()
    o = oracle.OracleSystem(system)
    rng = oracle.rng_states(walkers_cpu + seed_offset)[seed_offset:].copy()
    xs = []
    for w in range(walkers_cpu):
        x, rng[w] = o.sites(rng[w])
        xs.append(x)
    ow = oracle.OracleWalkers(o, np.array(xs), rng)
    ow.steps(warm_sweeps, nthreads)  # untimed warm-up sweeps
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps:
        ow.steps(1, nthreads)
        steps += 1
        if time.perf_counter() - t0 >= min_seconds:
            break
    dt = time.perf_counter() - t0
    return walkers_cpu * system.nelec * steps / dt, steps, dt


def run_reference(args):
    rank, world, local, pg = dist_setup(args.gpus)
    if rank != 0:
        pg.close()
        return 0
    from champ_b200.system import make_synthetic
    cfg, W, desc = CONFIGS[args.config]
    system = make_synthetic(cfg)
    nthreads = os.cpu_count() or 1
    rates = []
    for k in range(max(1, args.steps)):
        rate, steps, dt = cpu_port_rate(system, nthreads, nthreads, min_seconds=5.0, max_steps=100,
                                        warm_sweeps=max(1, args.warmup) if k == 0 else 1)
        rates.append(rate)
    v = statistics.median(rates)
    line = {
        "impl": "reference", "metric": "electron-moves/s", "value": v, "unit": "electron-moves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "walkers": W, "walkers_cpu": nthreads, "precision": "fp64"},
        "cpu_baseline": {"value": v, "unit": "electron-moves/s", "cores": nthreads, "kind": "port",
                         "sample": f"{nthreads} walkers (one per host thread, as one per CHAMP MPI rank), "
                                   f"metrop6 sweeps for >=5 s per step, median over {len(rates)} steps"},
        "e2e": {"value": v, "unit": "electron-moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    pg.close()
    return 0


def cpu_port_dmc_rate(system, nwalk_cpu, nthreads, min_seconds=10.0, max_steps=200):
    """Oracle DMC (dmc_ps + branching + splitj) on host threads: electron-moves/s."""
    from oracle import oracle
    oracle.build()
    o = oracle.OracleSystem(system)
    mw = 4 * nwalk_cpu + 1
    rng = oracle.rng_states(mw + 1)
    xs = []
    for w in range(nwalk_cpu):
        x, rng[w] = o.sites(rng[w])
        xs.append(x)
    e0 = float(np.median([o.hpsi(x)["energy"] for x in xs]))
    d = oracle.OracleDmc(o, np.array(xs), rng[:mw], rng[mw], tau=0.01, etrial=e0, mwalk=mw)
    d.steps(1, nthreads)
    t0 = time.perf_counter()
    moves = 0
    steps = 0
    while steps < max_steps:
        nw = d.results()["nwalk"]
        d.steps(1, nthreads)
        moves += nw * system.nelec
        steps += 1
        if time.perf_counter() - t0 >= min_seconds:
            break
    dt = time.perf_counter() - t0
    return moves / dt, steps, dt


def run_dmc(args):
    """DMC workload (config c2): electron-moves/s of dmc_ps steps."""
    import torch
    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    from champ_b200.engine import Dmc, Engine, rng_states, start_population
    from champ_b200.system import make_synthetic
    cfg, W, desc = CONFIGS[args.config]
    if args.walkers:
        W = args.walkers
    system = make_synthetic(cfg)
    mw = 3 * W + 1   # capacity for the branching of a crude (random-orbital) trial function
    rng_all = rng_states((mw + 1) * (rank + 1))
    rng = rng_all[rank * (mw + 1):].copy()
    eng = Engine(system, device=local, precision=args.precision)
    start_population(eng, system, rng[:W].copy())
    eng.vmc_steps(args.equil)
    xv, _ = eng.walkers()
    e0 = float(np.median(eng.state()[0]))   # robust against the heavy tails of E_L near nodes
    dmc = Dmc(eng, xv, rng[:mw], rng[mw], tau=0.01, etrial=e0, mwalk=mw)
    for _ in range(args.warmup):
        dmc.steps(1)
    moves = 0
    ms = 0.0
    launches = 0
    with ClockSampler(local) as clk:
        barrier(pg, local)
        for _ in range(args.steps):
            nw = dmc.population()
            dmc.steps(1)
            ms += dmc.last_ms()
            launches += eng.launches()
            moves += nw * system.nelec
        barrier(pg, local)
    ms_max = max_over_ranks(ms, pg, local)
    value = moves * world / (ms_max * 1e-3)
    eng.profile(True)
    dmc.steps(1)
    stages = eng.stage_times()
    eng.profile(False)
    if rank != 0:
        pg.close()
        return 0
    cpu_rate, cpu_steps, cpu_dt = cpu_port_dmc_rate(system, os.cpu_count() or 1, os.cpu_count() or 1)
    top = max(stages.items(), key=lambda kv: kv[1][0])
    line = {
        "metric": "electron-moves/s", "value": value, "unit": "electron-moves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "mixed", "data": "synthetic",
        "config": {"workload": desc, "walkers": W, "mwalk": mw, "electrons": system.nelec,
                   "determinants": int(system.iworbd.shape[0]), "precision": args.precision,
                   "l2": "per-walker state (about 0.7 MB per walker) exceeds the 126 MB L2",
                   "parallelism": f"replicas x{world} (independent populations)"},
        "top_stage": {"name": top[0], "ms": top[1][0], "launches": top[1][1]},
        "stages_ms_per_step": {k: round(v[0], 3) for k, v in stages.items() if v[1]},
        "cpu_baseline": {"value": cpu_rate, "unit": "electron-moves/s", "cores": os.cpu_count() or 1,
                         "kind": "port", "sample": f"oracle DMC, {os.cpu_count()} walkers on {os.cpu_count()} threads, "
                                                   f"{cpu_steps} steps ({cpu_dt:.1f} s)"},
        "clocks": clk.summary(),
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)
    pg.close()
    return 0


def device_overlap(blocks, slots):
    """Device-clock view of the served blocks: the summed block time over the
    time the device held at least one block (above 1: blocks of different
    jobs ran at the same time), and the most blocks in flight at once."""
    if not blocks:
        return None
    ev = sorted([(s, 1) for _, s, _ in blocks] + [(e, -1) for _, _, e in blocks])
    run = most = 0
    busy = 0
    last = None
    for tns, d in ev:
        if run > 0 and last is not None:
            busy += tns - last
        run += d
        most = max(most, run)
        last = tns
    total = sum(e - s for _, s, e in blocks)
    return {"blocks": len(blocks), "worker_slots": slots, "sum_block_s": round(total * 1e-9, 4),
            "device_occupied_s": round(busy * 1e-9, 4), "ratio": round(total / max(busy, 1), 3),
            "most_in_flight": most}


def run_serve(args):
    """Serving loop (config c4): p50/p99 time-to-result of a Poisson stream of jobs."""
    import torch
    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    from champ_b200 import serve
    from champ_b200.system import make_chain
    _, _, desc = CONFIGS[args.config]
    njobs = max(16, args.steps)
    rng = np.random.default_rng(4242 + rank)
    nel = rng.integers(8, 201, size=njobs)
    nwk = rng.integers(256, 1025, size=njobs)
    arrivals = serve.poisson_arrivals(njobs, args.rate, 99 + rank)
    budget = int(args.budget_gb * (1 << 30))

    def jobs(n, t):
        return [serve.Job(jid=i, system=make_chain(int(nel[i]), 1000 + i), nwalk=int(nwk[i]), target_err=5e-4,
                          max_blocks=12, nstep=5, arrival=float(t[i]) if t is not None else 0.0,
                          seed_offset=int(np.sum(nwk[:i]))) for i in range(n)]

    # warm-up: the module loads and every kernel is compiled into the context once
    serve.Server(budget, precision=args.precision, device=local, slots=args.slots).run(jobs(min(args.warmup, 2), None))
    srv = serve.Server(budget, precision=args.precision, device=local, slots=args.slots)
    job_list = jobs(njobs, arrivals)     # the molecules are generated before the clock starts
    with ClockSampler(local) as clk:
        barrier(pg, local)
        t0 = time.perf_counter()
        done = srv.run(job_list)
        torch.cuda.synchronize(local)
        makespan = time.perf_counter() - t0
        barrier(pg, local)
    summ = serve.summary(done, makespan)
    p50 = max_over_ranks(summ["p50_s"], pg, local)
    if rank != 0:
        pg.close()
        return 0
    line = {
        "metric": "job time-to-result p50", "value": p50, "unit": "s", "n_gpus": world, "steps": njobs,
        "warmup": args.warmup, "ms_per_step": 1e3 * makespan / njobs, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "mixed",
        "data": "synthetic",
        "config": {"workload": desc, "jobs": njobs, "rate_per_s": args.rate, "hbm_budget_gb": args.budget_gb,
                   "precision": args.precision, "block": "5 sweeps", "max_blocks": 12,
                   "worker_slots": args.slots,
                   "parallelism": f"replicas x{world} (independent job streams)"},
        "serving": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in summ.items()},
        "peak_admitted_gb": round(srv.peak_bytes / (1 << 30), 3),
        "overlap": device_overlap(srv.device_blocks, args.slots),
        "e2e": {"value": p50, "unit": "s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "path": "host job specs -> engine contexts (walkers and streams uploaded) -> block results read back"},
        "clocks": clk.summary(),
        "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)
    pg.close()
    return 0


def batched_rate(systems, walkers, precision, device, steps, warmup, slots, mode="graph", bands=1):
    """Sweeps of every system's own context, all at once: mode "graph" runs
    them as one CUDA graph of the contexts' sweep graphs (cw_batch_vmc_steps,
    one launch per sweep, timed with the batch's events); mode "ragged" as one
    launch per move stage over every system's walkers (cw_batch_set_ragged,
    same graph launch and timing); mode "threads"
    issues each context's sweeps from `slots` worker threads on its own stream
    (timed from device-clock stamps; the summed device time of the contexts'
    own sweeps is returned too).  Returns electron-moves/s over the device
    span of the timed sweeps, the wall time, that sum (None for "graph"), the
    span, the launches and the autotuned tiles."""
    import concurrent.futures as cf
    from champ_b200.engine import Engine, rng_states, start_population
    engines = []
    tiles = {}
    off = 0
    for s, w in zip(systems, walkers):
        e = Engine(s, device=device, precision=precision)
        start_population(e, s, rng_states(off + w)[off:].copy())
        off += w
        if precision == "fp64":   # per-system LCAO tiles (the mixed path's tensor-core kernel has one)
            ch = e.autotune(3)
            key = f"{ch['lcao_move_tile']}/{ch['lcao_all_tile']}"
            tiles[key] = tiles.get(key, 0) + 1
        engines.append(e)

    moves = sum(w * s.nelec for s, w in zip(systems, walkers)) * steps
    extra_launches = 0
    if mode in ("graph", "ragged"):
        # one CUDA graph per sweep: the systems' own sweep graphs as child
        # nodes, or (ragged) one launch per move stage over all systems
        from champ_b200.engine import Batch
        b = Batch(engines, ragged=(bands if mode == "ragged" else 0))
        b.vmc_steps(warmup)                                      # captures + warm-up
        t0 = time.perf_counter()
        b.vmc_steps(steps)
        wall = time.perf_counter() - t0
        span_s = b.last_ms() * 1e-3
        if mode == "ragged":
            info = b.info()
            extra_launches = steps * (info["ragged_launches"] + info["system_launches"])
            tiles = {"ragged_lcao_tile": info["lcao_bn"], "bands": info["bands"]}
        b.close()
        own_s = None
    else:
        def sweep(e, n):
            e.stamp()
            e.vmc_steps(n)
            e.stamp()
            e.sync()

        with cf.ThreadPoolExecutor(max_workers=slots) as pool:
            list(pool.map(lambda e: sweep(e, warmup), engines))  # graph capture + warm-up
            t0 = time.perf_counter()
            list(pool.map(lambda e: sweep(e, steps), engines))
            wall = time.perf_counter() - t0
        st = [e.stamps()[-2:] for e in engines]
        span_s = (max(int(b) for _, b in st) - min(int(a) for a, _ in st)) * 1e-9
        own_s = sum(int(b) - int(a) for a, b in st) * 1e-9
    launches = sum(e.launches() for e in engines) + extra_launches
    for e in engines:
        e.close()
    return moves / span_s, wall, own_s, span_s, launches, tiles


def run_batched(args):
    """Config c3: many uneven systems resident at once, swept concurrently."""
    import torch
    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    from champ_b200 import serve
    from champ_b200.system import make_chain
    _, _, desc = CONFIGS[args.config]
    nsys = args.systems
    rng = np.random.default_rng(5151 + rank)
    nel = rng.integers(8, 201, size=nsys)
    nwk = rng.integers(256, 4097, size=nsys)
    systems = [make_chain(int(n), 3000 + 97 * rank + i, orbitals="random") for i, n in enumerate(nel)]
    budget = args.budget_gb * (1 << 30)
    need = sum(serve.estimate_bytes(s, int(w), "mixed") for s, w in zip(systems, nwk))
    scale = min(1.0, budget / need)
    walkers = [max(64, int(w * scale)) for w in nwk]
    res, rag = {}, {}
    with ClockSampler(local) as clk:
        for prec in ("fp64", "mixed"):
            barrier(pg, local)
            res[prec] = batched_rate(systems, walkers, prec, local, args.steps, max(args.warmup, 1), args.slots)
            barrier(pg, local)
            for nb in (1, args.bands):
                rag[(prec, nb)] = batched_rate(systems, walkers, prec, local, args.steps, max(args.warmup, 1),
                                               args.slots, mode="ragged", bands=nb)
                barrier(pg, local)
        barrier(pg, local)
        threads = batched_rate(systems, walkers, args.precision, local, args.steps, max(args.warmup, 1), args.slots,
                               mode="threads")
        barrier(pg, local)
    value = max_over_ranks(1.0 / res[args.precision][0], pg, local)
    value = world / value
    if rank != 0:
        pg.close()
        return 0
    r = res[args.precision]
    moves_step = sum(w * s.nelec for s, w in zip(systems, walkers))
    line = {
        "metric": "electron-moves/s", "value": value, "unit": "electron-moves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * r[3] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "mixed", "data": "synthetic",
        "config": {"workload": desc, "systems": nsys, "electrons_min_max": [int(nel.min()), int(nel.max())],
                   "walkers_total": int(sum(walkers)), "walker_scale": round(scale, 4),
                   "walker_note": "drawn counts scaled so that all systems' contexts fit the HBM budget at once",
                   "hbm_budget_gb": args.budget_gb, "precision": args.precision,
                   "batching": "all systems' sweeps in one CUDA graph (cw_batch_vmc_steps)",
                   "l2": "per-walker state of every system far exceeds the 126 MB L2",
                   "parallelism": f"replicas x{world}"},
        "batched": {p: {"moves_per_s": round(v[0], 1), "device_span_s": round(v[3], 4), "wall_s": round(v[1], 4),
                        "mode": "one CUDA graph of all systems' sweep graphs, one launch per sweep"}
                    for p, v in res.items()},
        "batched_ragged": {f"{p}_bands{nb}": {"moves_per_s": round(v[0], 1), "device_span_s": round(v[3], 4),
                                              "wall_s": round(v[1], 4), "launches": v[4], "lcao_tile": v[5],
                                              "mode": "one launch per move stage over the walkers of every system "
                                                      "of a band (cw_batch_set_ragged), bands side by side, "
                                                      "systems' hpsi on their own streams, one graph"}
                           for (p, nb), v in rag.items()},
        "batched_threads": {"precision": args.precision, "moves_per_s": round(threads[0], 1),
                            "device_span_s": round(threads[3], 4),
                            "sum_of_context_device_s": round(threads[2], 4),
                            "concurrency": round(threads[2] / threads[3], 2), "wall_s": round(threads[1], 4),
                            "mode": f"each system's sweeps from {args.slots} worker threads on its own stream"},
        "mixed_over_fp64": round(res["mixed"][0] / res["fp64"][0], 3),
        "autotuned_lcao_tiles": {"note": "N tiles (move/all-electron) picked per system by cw_autotune, FP64 path",
                                 "systems_per_choice": res["fp64"][5]},
        "e2e": {"value": None, "unit": "electron-moves/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "path": "not measured for the batched config"},
        "clocks": clk.summary(), "gpu_launches": int(r[4]),
        "moves_per_step": int(moves_step),
    }
    print(json.dumps(line))
    pg.close()
    return 0


def efficiency_run(system, x, rng, precision, device, nblk=10, nstep=5):
    """nblk blocks of nstep sweeps from the given walkers and streams: the
    block estimate of CHAMP's finwrt (walkers in the role of ranks), the
    device time of the sweeps, and the per-walker sums of the first block."""
    from champ_b200.engine import Engine
    e = Engine(system, device=device, precision=precision)
    e.set_walkers(x, rng)
    ms = 0.0
    first = None
    for b in range(nblk):
        e.vmc_steps(nstep)
        ms += e.last_ms()
        if b == 0:
            first = (e.walkers()[1], e.sums())
        e.end_block()
    r = e.results()
    e.close()
    r = {k: float(v) for k, v in r.items()}
    r["t_s"] = ms * 1e-3
    r["efficiency"] = 1.0 / (r["err"] ** 2 * r["t_s"]) if r["err"] > 0 else None
    return r, first


def run_ours(args):
    import torch
    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    from champ_b200.engine import Engine, start_population, rng_states
    from champ_b200.system import make_synthetic
    cfg, W, desc = CONFIGS[args.config]
    if args.walkers:
        W = args.walkers
    system = make_synthetic(cfg)
    # replica r runs its own walkers: streams r*W .. r*W+W-1 of the default seed
    from champ_b200.replicas import rank_streams
    rng = rank_streams(rank, W, rng_states)
    eng = Engine(system, device=local, precision=args.precision)
    start_population(eng, system, rng)
    # equilibration from the sites start (discarded), then the timed steps
    eng.vmc_steps(args.equil)
    x_eq, rng_eq = eng.walkers()
    eng.set_walkers(x_eq, rng_eq)
    for _ in range(args.warmup):
        eng.vmc_steps(1)
    # --- timed region: K steps, walkers resident in HBM -------------------
    with ClockSampler(local) as clk:
        barrier(pg, local)
        eng.vmc_steps(args.steps)
        barrier(pg, local)
    ms_dev = eng.last_ms()
    launches = eng.launches()
    ms_max = max_over_ranks(ms_dev, pg, local)
    moves = W * system.nelec * args.steps * world
    value = moves / (ms_max * 1e-3)
    # --- per-stage timing pass (CUDA events around every launch) ----------
    eng.profile(True)
    eng.vmc_steps(1)
    stages = eng.stage_times()
    eng.profile(False)
    # --- e2e: the C-ABI calls of a caller that keeps walkers in host memory
    x_h = torch.empty((W, system.nelec, 3), dtype=torch.float64, pin_memory=True).numpy()
    r_h = torch.empty((W, 4), dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    xx, rr = eng.walkers()
    x_h[...] = xx
    r_h[...] = rr
    e2e_steps = max(1, min(args.steps, 2))
    barrier(pg, local)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        eng.set_walkers(x_h, r_h)          # H2D: positions + streams (zerest recompute)
        eng.vmc_steps(1)
        eng.walkers(x_h, r_h)              # D2H: positions + streams, into the pinned buffers
        eng.end_block()                    # D2H: per-walker sums
    barrier(pg, local)
    e2e_s = max_over_ranks(time.perf_counter() - t0, pg, local)
    e2e = W * system.nelec * e2e_steps * world / e2e_s
    eng.close()
    # --- efficiency 1/(err^2 t): FP64 and mixed from the same equilibrated
    # walkers and streams, 10 blocks each (outside the timed region) --------
    eff = {}
    first = {}
    for prec in ("fp64", "mixed"):
        eff[prec], first[prec] = efficiency_run(system, x_eq, rng_eq, prec, local, nblk=args.blocks,
                                                nstep=args.block_steps)
    (r64, s64), (rmx, smx) = first["fp64"], first["mixed"]
    same = np.all(r64 == rmx, axis=1) & (s64[:, 4] == smx[:, 4])
    wsum = float(s64[same, 0].sum())
    bias = (float(smx[same, 1].sum()) - float(s64[same, 1].sum())) / wsum if wsum > 0 else None
    if rank != 0:
        pg.close()
        return 0
    peaks, peak_kind = load_peaks()
    # the move Jastrow runs in FP64 (fp64 path) or FP32 (mixed path): its
    # roofline denominator is the measured FMA peak of that pipe
    fp64 = args.precision == "fp64"
    fma_peak = None
    try:
        import ctypes as C
        from champ_b200.abi import load_engine
        t = np.zeros(1)
        if load_engine().cw_fma_peak(local, 1 if fp64 else 0, t.ctypes.data_as(C.POINTER(C.c_double))) == 0:
            fma_peak = float(t[0])
    except Exception:
        fma_peak = None
    alg = algorithmic(system, W)
    ms_jm, n_jm = stages["jastrow_move"]
    ms_acc, n_acc = stages["accept"]
    total_stage = sum(v[0] for v in stages.values())
    top = max(stages.items(), key=lambda kv: kv[1][0])
    jm_tflops = alg["f_jastrow_move"] / (ms_jm / n_jm * 1e-3) / 1e12
    roof = {"kernel": ("k_jastrow_move" if fp64 else "k_jastrow_move_f32") + " (jastrow4e, one electron, all walkers)",
            "bound": "fp64-simt" if fp64 else "fp32-simt",
            "achieved": jm_tflops, "peak": fma_peak, "unit": "TFLOP/s",
            "frac": (jm_tflops / fma_peak) if fma_peak else None,
            "peak_source": f"measured {'FP64' if fp64 else 'FP32'} FMA probe (cw_fma_peak) on this GPU",
            "traffic": jm_traffic(W) if fp64 else None,
            "traffic_source": "dram bytes of one ncu capture at 2048 walkers, scaled by the walker count",
            "share_of_step": ms_jm / total_stage,
            "work_per_launch": "8*(N-1)*M*T + 8*(N-1)*nordb + 8*M*norda FLOP per walker (T=23 e-e-n terms)"}
    # HBM-bound move update: k_decide (ratio, drift, accept) + k_commit
    # (Sherman-Morrison rows, orbital rows, Jastrow pair rows of the accepted
    # walkers; the engine updates lazily, so its bytes scale with acceptance)
    ms_cm, n_cm = stages["commit"]
    upd_ms = ms_acc / n_acc + ms_cm / n_cm
    acc_frac = eff[args.precision]["accept"]
    b_upd = update_bytes(system, W, acc_frac)
    upd_gbs = b_upd / (upd_ms * 1e-3) / 1e9
    roof_hbm = {"kernel": "k_decide + k_commit (ratio, accept, Sherman-Morrison and table commit)", "bound": "hbm",
                "achieved": upd_gbs, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                "frac": upd_gbs / peaks.get("hbm_gbs"), "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})",
                "traffic": update_traffic(W),
                "work_per_launch": "engine's lazy update per walker-move: 8*(n + 4 O + 12 + N) B read by k_decide, "
                                  "plus for an accepted move 8*(2 n^2 + 2 n + 8 n + 2 M + 14 N) B in k_commit; "
                                  f"acceptance {acc_frac:.3f}"}
    cpu_rate, cpu_steps, cpu_dt = cpu_port_rate(system, os.cpu_count() or 1, os.cpu_count() or 1,
                                                min_seconds=10.0, max_steps=1000)
    h2d = W * system.nelec * 3 * 8 + W * 32
    d2h = h2d + W * 8 * 8
    ef64, efmx = eff["fp64"], eff["mixed"]
    diff = efmx["energy"] - ef64["energy"]
    line = {
        "metric": "electron-moves/s", "value": value, "unit": "electron-moves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "mixed",
        "data": "synthetic",
        "config": {"workload": desc, "walkers": W, "electrons": system.nelec, "basis": system.nbasis,
                   "orbitals": system.norb, "centres": system.ncent, "precision": args.precision,
                   "equilibration_sweeps": args.equil,
                   "l2": "per-walker state (3.8 GB of Jastrow pair tables alone) exceeds the 126 MB L2",
                   "parallelism": f"replicas x{world} (independent walker populations, no data-path collective)"},
        "e2e": {"value": e2e, "unit": "electron-moves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "cw_set_walkers (pinned host x, rng; includes the zerest hpsi of every walker) + "
                        "cw_vmc_steps(1) + cw_get_walkers (into the pinned x, rng) + cw_end_block"},
        "roofline": roof, "roofline_hbm": roof_hbm,
        "efficiency_fp64": {"value": ef64["efficiency"], "unit": "1/(Ha^2 s)", "energy": ef64["energy"],
                            "err": ef64["err"], "sigma": ef64["sigma"], "tcorr": ef64["tcorr"],
                            "accept": ef64["accept"], "t_s": ef64["t_s"]},
        "efficiency_mixed": {"value": efmx["efficiency"], "unit": "1/(Ha^2 s)", "energy": efmx["energy"],
                             "err": efmx["err"], "sigma": efmx["sigma"], "tcorr": efmx["tcorr"],
                             "accept": efmx["accept"], "t_s": efmx["t_s"]},
        "efficiency_ratio_mixed_over_fp64": (efmx["efficiency"] / ef64["efficiency"])
        if ef64["efficiency"] and efmx["efficiency"] else None,
        "mean_E_diff_mHa": {"value": diff * 1e3, "combined_err_mHa": 1e3 * (ef64["err"] ** 2 + efmx["err"] ** 2) ** 0.5,
                            "bias_matched_mHa": bias * 1e3 if bias is not None else None,
                            "matched_walkers": int(same.sum()), "target_mHa": 0.1,
                            "note": f"{args.blocks} blocks x {args.block_steps} sweeps per precision from the same "
                                    "equilibrated walkers and streams; walks part where a near-threshold decision "
                                    "differs, so the difference of the means is statistical; the bias is the mean "
                                    "E_L difference over the first block's walkers whose decisions all agreed"},
        "top_stage": {"name": top[0], "ms": top[1][0], "launches": top[1][1]},
        "stages_ms_per_step": {k: round(v[0], 3) for k, v in stages.items()},
        "cpu_baseline": {"value": cpu_rate, "unit": "electron-moves/s", "cores": os.cpu_count() or 1, "kind": "port",
                         "sample": f"{os.cpu_count()} walkers x {cpu_steps} sweeps ({cpu_dt:.1f} s), "
                                   "oracle C++ FP64 restatement, one walker per host thread"},
        "clocks": clk.summary(),
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)
    pg.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1", choices=sorted(CONFIGS))
    ap.add_argument("--walkers", type=int, default=0)
    ap.add_argument("--equil", type=int, default=50, help="equilibration sweeps before the timed steps")
    ap.add_argument("--blocks", type=int, default=10, help="blocks of each efficiency run")
    ap.add_argument("--block-steps", type=int, default=5, help="sweeps per block of the efficiency runs")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--rate", type=float, default=4.0, help="c4: job arrivals per second")
    ap.add_argument("--budget-gb", type=float, default=None,
                    help="c3/c4: HBM budget of the resident contexts (default 120 for c3, 16 for c4)")
    ap.add_argument("--systems", type=int, default=64, help="c3: systems resident at once")
    ap.add_argument("--slots", type=int, default=16, help="c3/c4: worker threads (contexts with work in flight)")
    ap.add_argument("--bands", type=int, default=4, help="c3: bands of systems of the banded ragged run")
    args = ap.parse_args()
    if args.budget_gb is None:
        args.budget_gb = 120.0 if args.config == "c3" else 16.0
    if args.impl == "reference":
        if args.config in ("c3", "c4"):
            print(json.dumps({"impl": "reference", "unavailable": "CHAMP runs one system per job (no batching "
                                                                  "across systems, no request loop)"}))
            return 0
        return run_reference(args)
    if args.config == "c2":
        return run_dmc(args)
    if args.config == "c4":
        return run_serve(args)
    if args.config == "c3":
        return run_batched(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
