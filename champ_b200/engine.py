"""Host-side mirror of CHAMP's VMC driver over the CUDA walker engine.

``Engine`` owns one ``cw_ctx`` (one molecule, one walker population) and
exposes the batched drop-ins for CHAMP's per-walker routines with CHAMP's
names and argument meaning:

* ``set_walkers``  — mc_configs_start + zerest (vmc/mc_configs.f90:33,
  vmc/acuest.f90:179)
* ``vmc_steps``    — rotqua + metrop6 per step (vmc/vmc.f90:108-134)
* ``end_block``    — acuest + acuest_reduce (vmc/acuest.f90:61)
* ``results``      — finwrt (vmc/finwrt.f90:75)
* ``hpsi``         — hpsi (vmc/hpsi.f90:3)
* ``orbitals``, ``jastrow``, ``slater`` — orbitals / jastrow_factor /
  determinant parity hooks.

``Dmc`` drives a diffusion Monte Carlo population over the same context:
``init`` (dmc/init.f90), ``steps`` (rotqua + dmc_ps + splitj + acues1,
dmc/dmc.f90:88-107), ``end_block`` (acuest) and ``results`` (finwrt).

Every call goes through the C ABI of include/champ_b200.h; a nonzero status
raises ``EngineError`` carrying cw_last_error, the way CHAMP's fatal_error
aborts (module/m_error.f90:31).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import CW_PREC_FP64, CW_PREC_MIXED, dptr, load_engine, u64ptr

DEFAULT_SEED = "18123437465549275475255231234865"  # vmc/parser.f90:315


class EngineError(RuntimeError):
    def __init__(self, msg, code=0):
        super().__init__(msg)
        self.code = code


CW_ERR_SINGULAR = 4


def seed_ints(cseed: str = DEFAULT_SEED) -> np.ndarray:
    """read(cseed,'(8i4)') irn (vmc/parser.f90:651)."""
    if len(cseed) < 32:
        raise ValueError("Random number seed is shorter than 32 characters.")
    return np.array([int(cseed[4 * i:4 * i + 4]) for i in range(8)], np.int32)


def rng_states(nwalk: int, cseed: str = DEFAULT_SEED) -> np.ndarray:
    """Stream of walker w = setrn(seed) + w jumps, as CHAMP's MPI rank w."""
    lib = load_engine()
    out = np.zeros((nwalk, 4), np.uint64)
    irn = seed_ints(cseed)
    rc = lib.cw_rng_states(irn.ctypes.data_as(C.POINTER(C.c_int32)), nwalk, u64ptr(out))
    if rc:
        raise EngineError("cw_rng_states failed")
    return out


def initial_configs(system, rng: np.ndarray):
    """sites-based initial electrons of every walker; advances rng in place."""
    lib = load_engine()
    desc = system.desc()
    W = rng.shape[0]
    x = np.zeros((W, system.nelec, 3))
    rc = lib.cw_sites(C.byref(desc), W, u64ptr(rng), dptr(x))
    if rc:
        raise EngineError("cw_sites failed")
    return x


def start_population(eng, system, rng: np.ndarray, max_redraws: int = 32):
    """mc_configs_start (vmc/mc_configs.f90:33) for every walker of `eng`:
    sites start positions drawn from each walker's stream (rng [W][4],
    advanced in place), then cw_set_walkers.  A walker whose Slater matrix is
    singular at its start (two same-spin electrons where the occupied
    orbitals cannot tell them apart) draws a new sites start from its own,
    further advanced, stream; CHAMP would stop the run there (matinv).
    Returns the start positions."""
    x = initial_configs(system, rng)
    for _ in range(max_redraws):
        try:
            eng.set_walkers(x, rng)
            return x
        except EngineError as e:
            if e.code != CW_ERR_SINGULAR:
                raise
        bad = np.nonzero(eng.walker_status() & 1)[0]
        sub = np.ascontiguousarray(rng[bad])
        x[bad] = initial_configs(system, sub)
        rng[bad] = sub
    raise EngineError(f"walkers still singular after {max_redraws} new start draws", CW_ERR_SINGULAR)


class Engine:
    def __init__(self, system, device: int = 0, precision: str = "fp64"):
        self.lib = load_engine()
        self.system = system
        self._desc = system.desc()
        self.h = C.c_void_p()
        prec = {"fp64": CW_PREC_FP64, "mixed": CW_PREC_MIXED}[precision]
        rc = self.lib.cw_create(C.byref(self.h), C.byref(self._desc), device, prec)
        self._check(rc, "cw_create")
        self.W = 0

    def _check(self, rc, what):
        if rc:
            msg = self.lib.cw_last_error(self.h).decode() if self.h else ""
            raise EngineError(f"{what} failed (status {rc}): {msg}", rc)

    def close(self):
        if self.h:
            self.lib.cw_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- walkers -----------------------------------------------------------
    def set_walkers(self, x, rng):
        x = np.ascontiguousarray(x, np.float64)
        rng = np.ascontiguousarray(rng, np.uint64)
        self.W = rng.shape[0]
        self._check(self.lib.cw_set_walkers(self.h, self.W, dptr(x), u64ptr(rng)), "cw_set_walkers")

    def walker_status(self):
        """Per-walker status words (bit 0 singular Slater matrix, bit 1
        non-finite local energy, bit 2 proposal rejection loop gave up)."""
        out = np.zeros(self.W, np.int32)
        self._check(self.lib.cw_walker_status(self.h, out.ctypes.data_as(C.POINTER(C.c_int32))), "cw_walker_status")
        return out

    def autotune(self, reps: int = 5) -> dict:
        """Pick the LCAO GEMM tiles of this context by timing (cw_autotune);
        returns the chosen N tiles."""
        out = np.zeros(2, np.int32)
        self._check(self.lib.cw_autotune(self.h, int(reps), out.ctypes.data_as(C.POINTER(C.c_int32))), "cw_autotune")
        return dict(lcao_move_tile=int(out[0]), lcao_all_tile=int(out[1]))

    def sync(self):
        """Wait for the context's queued work."""
        self._check(self.lib.cw_sync(self.h), "cw_sync")

    def stamp(self):
        """Enqueue a device-clock stamp on the context's stream."""
        self._check(self.lib.cw_stamp(self.h), "cw_stamp")

    def stamps(self):
        """All device-clock stamps of the context so far (ns), after its
        queued work has finished."""
        n = self.lib.cw_stamps(self.h, None, 0)
        out = np.zeros(max(n, 1), np.int64)
        n = self.lib.cw_stamps(self.h, out.ctypes.data_as(C.POINTER(C.c_int64)), n)
        if n < 0:
            self._check(n, "cw_stamps")
        return out[:n]

    # -- per-electron routines (a metrop6 kept on the host) ---------------
    def psie(self, iel: int, xnew):
        """psie of electron iel at xnew [W][3] for every walker: (psid, psij)."""
        xnew = np.ascontiguousarray(xnew, np.float64)
        psid, psij = np.zeros(self.W), np.zeros(self.W)
        self._check(self.lib.cw_psie(self.h, iel, dptr(xnew), dptr(psid), dptr(psij)), "cw_psie")
        return psid, psij

    def grad(self, iel: int, iflag_move: int):
        """compute_determinante_grad of electron iel: [W][3] at the current
        position (iflag_move=1) or at the point of the last psie (0)."""
        vd = np.zeros((self.W, 3))
        self._check(self.lib.cw_grad(self.h, iel, iflag_move, dptr(vd)), "cw_grad")
        return vd

    def commit(self, iel: int, accept):
        """jassav + detsav for the walkers with accept[w] set, restore for the others."""
        a = np.ascontiguousarray(accept, np.int32)
        self._check(self.lib.cw_commit(self.h, iel, a.ctypes.data_as(C.POINTER(C.c_int32))), "cw_commit")

    def update_ymat(self, iel: int):
        self._check(self.lib.cw_update_ymat(self.h, iel), "cw_update_ymat")

    def walkers(self, x=None, rng=None):
        """Positions [W][nelec][3] and random streams [W][4]; written into
        the given C-contiguous arrays when passed (e.g. pinned host buffers,
        which the device writes directly), else into new ones."""
        if x is None:
            x = np.zeros((self.W, self.system.nelec, 3))
        if rng is None:
            rng = np.zeros((self.W, 4), np.uint64)
        if x.shape != (self.W, self.system.nelec, 3) or rng.shape != (self.W, 4):
            raise ValueError(f"walkers: arrays of shape {x.shape}, {rng.shape} for {self.W} walkers")
        self._check(self.lib.cw_get_walkers(self.h, dptr(x), u64ptr(rng)), "cw_get_walkers")
        return x, rng

    # -- VMC driver --------------------------------------------------------
    def vmc_steps(self, nstep: int):
        self._check(self.lib.cw_vmc_steps(self.h, nstep), "cw_vmc_steps")

    def last_ms(self) -> float:
        return float(self.lib.cw_last_ms(self.h))

    def launches(self) -> int:
        return int(self.lib.cw_launches(self.h))

    def device_bytes(self) -> int:
        """Bytes of device memory the context holds (tables, walkers, scratch)."""
        return int(self.lib.cw_device_bytes(self.h))

    def profile(self, enable: bool = True):
        self._check(self.lib.cw_profile(self.h, 1 if enable else 0), "cw_profile")

    def stage_times(self) -> dict:
        from .abi import STAGES
        ms = np.zeros(len(STAGES))
        n = (C.c_long * len(STAGES))()
        self._check(self.lib.cw_stage_times(self.h, dptr(ms), n), "cw_stage_times")
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(STAGES)}

    def end_block(self) -> float:
        e = np.zeros(1)
        self._check(self.lib.cw_end_block(self.h, dptr(e)), "cw_end_block")
        return float(e[0])

    def results(self) -> dict:
        o = np.zeros(8)
        self._check(self.lib.cw_results(self.h, dptr(o)), "cw_results")
        return dict(energy=o[0], err=o[1], sigma=o[2], tcorr=o[3], accept=o[4], pe=o[5], ke=o[6],
                    nblocks=o[7])

    def results_state(self, istate: int) -> dict:
        """Block results of state `istate` of a multi-state wave function."""
        o = np.zeros(8)
        self._check(self.lib.cw_results_state(self.h, istate, dptr(o)), "cw_results_state")
        return dict(energy=o[0], err=o[1], pe=o[5], ke=o[6], nblocks=o[7])

    def state_energies(self):
        """Local energy and psi_D of every state at the last hpsi: [W][nstates] each."""
        ns = self.system.nstates
        e, p = np.zeros((self.W, ns)), np.zeros((self.W, ns))
        self._check(self.lib.cw_state_energies(self.h, dptr(e), dptr(p)), "cw_state_energies")
        return e, p

    # -- wave-function optimisation (Jastrow and CI parameters) ------------
    def opt_ci(self, enable: bool = True, overlap: bool = True):
        self._check(self.lib.cw_opt_ci(self.h, 1 if enable else 0, 1 if overlap else 0), "cw_opt_ci")
        self._opt_np = self.system.iworbd.shape[0] if enable else 0
        self._opt_njas = 0

    def opt_setup(self, ci: bool = False, jas_map=None, overlap: bool = True):
        """Derivatives and SR sums over the optimisation vector [Jastrow
        parameters | CI coefficients]; jas_map is the [nraw, njas] map of
        jastrow_opt.param_map (None: no Jastrow parameters)."""
        njas = 0 if jas_map is None else int(np.asarray(jas_map).shape[1])
        m = None if jas_map is None else np.ascontiguousarray(jas_map, dtype=np.float64)
        if m is not None and m.shape[0] != self.jas_nraw():
            raise ValueError(f"jas_map has {m.shape[0]} rows, the engine's raw vector {self.jas_nraw()}")
        self._check(self.lib.cw_opt_setup(self.h, 1 if ci else 0, njas, dptr(m) if m is not None else None,
                                          1 if overlap else 0), "cw_opt_setup")
        self._opt_njas = njas
        self._opt_np = njas + (self.system.iworbd.shape[0] if ci else 0) + getattr(self, "_opt_norb", 0)

    def opt_orb(self, ideriv):
        """Orbital rotations (io, jo), 1-based, of the optimisation vector;
        they join it at the next opt_setup (empty: none)."""
        d = np.ascontiguousarray(np.asarray(ideriv, np.int32).reshape(-1, 2))
        self._check(self.lib.cw_opt_orb(self.h, d.shape[0], d.ctypes.data_as(C.POINTER(C.c_int32))), "cw_opt_orb")
        self._opt_norb = d.shape[0]

    def orb_o(self):
        out = np.zeros((self.W, getattr(self, "_opt_norb", 0)))
        self._check(self.lib.cw_orb_o(self.h, dptr(out)), "cw_orb_o")
        return out

    def jas_nraw(self) -> int:
        n = C.c_int(0)
        self._check(self.lib.cw_jas_nraw(self.h, C.byref(n)), "cw_jas_nraw")
        return n.value

    def jas_raw(self):
        out = np.zeros((self.W, self.jas_nraw()))
        self._check(self.lib.cw_jas_raw(self.h, dptr(out)), "cw_jas_raw")
        return out

    def jas_o(self):
        out = np.zeros((self.W, self._opt_njas))
        self._check(self.lib.cw_jas_o(self.h, dptr(out)), "cw_jas_o")
        return out

    def opt_sums(self, overlap: bool = True):
        n = self._opt_np
        o, eo, w = np.zeros(n), np.zeros(n), np.zeros(1)
        oo = np.zeros((n, n)) if overlap else None
        self._check(self.lib.cw_opt_sums(self.h, dptr(o), dptr(eo), dptr(oo) if overlap else None, dptr(w)),
                    "cw_opt_sums")
        return dict(o=o, eo=eo, oo=oo, wsum=float(w[0]))

    def ci_o(self):
        nd = self.system.iworbd.shape[0]
        out = np.zeros((self.W, nd))
        self._check(self.lib.cw_ci_o(self.h, dptr(out)), "cw_ci_o")
        return out

    def opt_ci_sums(self, overlap: bool = True):
        nd = self.system.iworbd.shape[0]
        o, eo, w = np.zeros(nd), np.zeros(nd), np.zeros(1)
        oo = np.zeros((nd, nd)) if overlap else None
        self._check(self.lib.cw_opt_ci_sums(self.h, dptr(o), dptr(eo), dptr(oo) if overlap else None, dptr(w)),
                    "cw_opt_ci_sums")
        return dict(o=o, eo=eo, oo=oo, wsum=float(w[0]))

    def sums(self):
        out = np.zeros((self.W, 5))
        self._check(self.lib.cw_get_sums(self.h, dptr(out)), "cw_get_sums")
        return out

    def state(self):
        e, p, j = np.zeros(self.W), np.zeros(self.W), np.zeros(self.W)
        self._check(self.lib.cw_get_state(self.h, dptr(e), dptr(p), dptr(j)), "cw_get_state")
        return e, p, j

    # -- checkpoint / restart (dumper / startr) ---------------------------
    def checkpoint(self) -> bytes:
        n = int(self.lib.cw_checkpoint_bytes(self.h))
        if n < 0:
            self._check(1, "cw_checkpoint_bytes")
        buf = C.create_string_buffer(n)
        self._check(self.lib.cw_checkpoint(self.h, buf, n), "cw_checkpoint")
        return buf.raw

    def restore(self, data: bytes):
        buf = C.create_string_buffer(data, len(data))
        self._check(self.lib.cw_restore(self.h, buf, len(data)), "cw_restore")
        n = C.c_int()
        if self.lib.cw_dmc_walkers(self.h, C.byref(n), None, None, None, None) == 0:
            self.W = int(n.value)
        else:
            self.W = int(np.frombuffer(data[8 + 9 * 8:8 + 10 * 8], np.int64)[0])

    # -- per-walker routines ----------------------------------------------
    def hpsi(self, quad=None) -> dict:
        W = self.W
        e, p, j, k = np.zeros(W), np.zeros(W), np.zeros(W), np.zeros(W)
        if quad is None:
            rc = self.lib.cw_hpsi(self.h, None, None, None, dptr(e), dptr(p), dptr(j), dptr(k))
        else:
            q = [np.ascontiguousarray(a, np.float64) for a in quad]
            rc = self.lib.cw_hpsi(self.h, dptr(q[0]), dptr(q[1]), dptr(q[2]), dptr(e), dptr(p), dptr(j), dptr(k))
        self._check(rc, "cw_hpsi")
        return dict(energy=e, psid=p, psij=j, ekin=k)

    def orbitals(self):
        s = self.system
        orb = np.zeros((self.W, s.norb, s.nelec))
        dorb = np.zeros((self.W, 3, s.nelec, s.norb))
        ddorb = np.zeros((self.W, s.nelec, s.norb))
        self._check(self.lib.cw_orbitals(self.h, dptr(orb), dptr(dorb), dptr(ddorb)), "cw_orbitals")
        return orb, dorb, ddorb

    def jastrow(self):
        psij = np.zeros(self.W)
        v = np.zeros((self.W, self.system.nelec, 3))
        d2 = np.zeros(self.W)
        self._check(self.lib.cw_jastrow(self.h, dptr(psij), dptr(v), dptr(d2)), "cw_jastrow")
        return psij, v, d2

    def slater(self):
        nmax = max(self.system.nup, self.system.ndn)
        slmi = np.zeros((self.W, 2, nmax * nmax))
        det = np.zeros((self.W, 2))
        self._check(self.lib.cw_slater(self.h, dptr(slmi), dptr(det)), "cw_slater")
        return slmi, det


class Batch:
    """Several engines (one device) advanced together: each cw_batch_vmc_steps
    call runs nstep sweeps of every engine through one CUDA graph launch per
    sweep (the engines' own sweep graphs as parallel child nodes), or, with
    ``ragged`` = True or a band count, through one launch per move stage over
    the walkers of every engine of a band (bands of systems of about equal
    work, side by side)."""

    def __init__(self, engines, ragged: bool | int = False):
        self.engines = list(engines)
        self.lib = self.engines[0].lib
        arr = (C.c_void_p * len(self.engines))(*[e.h for e in self.engines])
        h = C.c_void_p()
        rc = self.lib.cw_batch_create(C.byref(h), arr, len(self.engines))
        if rc:
            raise EngineError(f"cw_batch_create failed (status {rc})", rc)
        self.h = h
        if ragged:
            self.set_ragged(ragged)

    def set_ragged(self, bands: bool | int):
        rc = self.lib.cw_batch_set_ragged(self.h, int(bands))
        if rc:
            msg = self.lib.cw_batch_last_error(self.h).decode()
            raise EngineError(f"cw_batch_set_ragged failed (status {rc}): {msg}", rc)

    def info(self) -> dict:
        v = (C.c_int64 * 5)()
        rc = self.lib.cw_batch_info(self.h, v)
        if rc:
            raise EngineError(f"cw_batch_info failed (status {rc})", rc)
        return {"ragged": bool(v[0]), "bands_asked": int(v[0]), "lcao_bn": int(v[1]),
                "ragged_launches": int(v[2]), "system_launches": int(v[3]), "bands": int(v[4])}

    def vmc_steps(self, nstep: int):
        rc = self.lib.cw_batch_vmc_steps(self.h, int(nstep))
        if rc:
            msg = self.lib.cw_batch_last_error(self.h).decode()
            raise EngineError(f"cw_batch_vmc_steps failed (status {rc}): {msg}", rc)

    def last_ms(self) -> float:
        return float(self.lib.cw_batch_last_ms(self.h))

    def close(self):
        if self.h:
            self.lib.cw_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Dmc:
    """One DMC population (one CHAMP rank's walkers) on an ``Engine``."""

    def __init__(self, engine: Engine, x, rng, pop_rng, tau: float, etrial: float, mwalk: int | None = None,
                 nfprod: int = 100):
        self.e = engine
        x = np.ascontiguousarray(x, np.float64)
        W = x.shape[0]
        self.mwalk = int(mwalk or int(1.5 * W) + 1)
        rng = np.ascontiguousarray(rng, np.uint64)
        if rng.shape[0] < self.mwalk:
            raise ValueError(f"rng holds {rng.shape[0]} streams, mwalk={self.mwalk} slots need one each")
        pop = np.ascontiguousarray(pop_rng, np.uint64).reshape(4)
        rc = engine.lib.cw_dmc_init(engine.h, W, self.mwalk, dptr(x), u64ptr(rng), u64ptr(pop), float(tau),
                                    float(etrial), int(nfprod))
        engine._check(rc, "cw_dmc_init")
        engine.W = W

    @classmethod
    def attach(cls, engine: "Engine", mwalk: int):
        """Wrap the DMC population of an engine restored from a checkpoint."""
        d = cls.__new__(cls)
        d.e = engine
        d.mwalk = int(mwalk)
        return d

    def steps(self, n: int):
        self.e._check(self.e.lib.cw_dmc_steps(self.e.h, n), "cw_dmc_steps")

    def end_block(self):
        self.e._check(self.e.lib.cw_dmc_end_block(self.e.h), "cw_dmc_end_block")

    def results(self) -> dict:
        o = np.zeros(12)
        self.e._check(self.e.lib.cw_dmc_results(self.e.h, dptr(o)), "cw_dmc_results")
        return dict(energy=o[0], err=o[1], nwalk=int(o[2]), eest=o[3], accept=o[4], taueff=o[5], pe=o[6],
                    ke=o[7], nblocks=o[8], fprod=o[9], eigv=o[10], wdsumo=o[11])

    def walkers(self):
        N = self.e.system.nelec
        n = C.c_int()
        x = np.zeros((self.mwalk, N, 3))
        wt = np.zeros(self.mwalk)
        eo = np.zeros(self.mwalk)
        r = np.zeros((self.mwalk, 4), np.uint64)
        self.e._check(self.e.lib.cw_dmc_walkers(self.e.h, C.byref(n), dptr(x), dptr(wt), dptr(eo), u64ptr(r)),
                      "cw_dmc_walkers")
        k = n.value
        self.e.W = k
        return x[:k], wt[:k], eo[:k], r[:k]

    def last_ms(self) -> float:
        return self.e.last_ms()

    def set_tmoves(self, icasula: int):
        self.e._check(self.e.lib.cw_dmc_set_tmoves(self.e.h, int(icasula)), "cw_dmc_set_tmoves")

    def counts(self) -> dict:
        o = (C.c_long * 4)()
        self.e._check(self.e.lib.cw_dmc_counts(self.e.h, o), "cw_dmc_counts")
        return dict(accepted=o[0], node_crossings=o[1], branchings=o[2], tmoves=o[3])

    def population(self) -> int:
        n = C.c_int()
        self.e._check(self.e.lib.cw_dmc_walkers(self.e.h, C.byref(n), None, None, None, None), "cw_dmc_walkers")
        return int(n.value)
