"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and bench.py's
CPU-baseline leg.  The engine package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_RNG = os.path.join(HERE, "_ref", "libxoshiro_ref.so")

_dp = C.POINTER(C.c_double)
_u64 = C.POINTER(C.c_uint64)
_i32 = C.POINTER(C.c_int32)


def build(force: bool = False):
    if force or not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        V = C.c_void_p
        L.or_sys_create.restype = V
        L.or_sys_create.argtypes = [C.c_void_p]
        L.or_sys_destroy.argtypes = [V]
        L.or_nterms4.argtypes = [C.c_int]
        L.or_pot_nn.restype = C.c_double
        L.or_pot_nn.argtypes = [C.c_int, _dp, _dp, _i32]
        L.or_matinv.argtypes = [_dp, C.c_int, _dp]
        L.or_rng_states.argtypes = [_i32, C.c_int, _u64]
        L.or_rng_uniform.argtypes = [_u64, C.c_int, _dp]
        L.or_gesqua.argtypes = [C.POINTER(C.c_int), _dp, _dp, _dp, _dp]
        L.or_sites.argtypes = [V, _u64, _dp]
        L.or_orbitals.argtypes = [V, _dp, _dp, _dp, _dp]
        L.or_jastrow.argtypes = [V, _dp, _dp, _dp, _dp]
        L.or_jas_nraw.argtypes = [V]
        L.or_jas_raw.argtypes = [V, _dp, _dp]
        L.or_slater.argtypes = [V, _dp, _dp, _dp]
        L.or_hpsi.argtypes = [V, _dp, _dp, _dp, _dp, _dp]
        L.or_walkers_create.restype = V
        L.or_walkers_create.argtypes = [V, C.c_int, _dp, _u64]
        L.or_walkers_destroy.argtypes = [V]
        L.or_vmc_steps.argtypes = [V, C.c_int, C.c_int]
        L.or_zerest.argtypes = [V]
        L.or_end_block.argtypes = [V, _dp]
        L.or_results.argtypes = [V, _dp]
        L.or_results_state.argtypes = [V, C.c_int, _dp]
        L.or_results_state.restype = C.c_int
        L.or_state_energies.argtypes = [V, _dp, _dp]
        L.or_opt_ci.argtypes = [V, C.c_int]
        L.or_ci_o.argtypes = [V, _dp]
        L.or_opt_ci_sums.argtypes = [V, _dp, _dp, _dp, _dp]
        L.or_get_walkers.argtypes = [V, _dp, _u64]
        L.or_get_sums.argtypes = [V, _dp]
        L.or_get_state.argtypes = [V, _dp, _dp, _dp]
        _lib = L
    return _lib


def dp(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def u64(a):
    return a.ctypes.data_as(_u64)


DEFAULT_SEED = "18123437465549275475255231234865"  # CHAMP default, vmc/parser.f90:315


def seed_ints(cseed: str = DEFAULT_SEED):
    """read(cseed,'(8i4)') irn (vmc/parser.f90:651)."""
    return np.array([int(cseed[4 * i:4 * i + 4]) for i in range(8)], np.int32)


def rng_states(nwalk: int, cseed: str = DEFAULT_SEED):
    out = np.zeros((nwalk, 4), np.uint64)
    irn = seed_ints(cseed)
    lib().or_rng_states(irn.ctypes.data_as(_i32), nwalk, u64(out))
    return out


class OracleSystem:
    def __init__(self, system):
        self.system = system
        self._desc = system.desc()
        self.h = lib().or_sys_create(C.addressof(self._desc))
        self.N = system.nelec

    def __del__(self):
        try:
            lib().or_sys_destroy(self.h)
        except Exception:
            pass

    def orbitals(self, x):
        s = self.system
        orb = np.zeros((s.norb, s.nelec))
        dorb = np.zeros((3, s.nelec, s.norb))
        ddorb = np.zeros((s.nelec, s.norb))
        lib().or_orbitals(self.h, dp(np.ascontiguousarray(x, float)), dp(orb), dp(dorb), dp(ddorb))
        return orb, dorb, ddorb

    def jastrow(self, x):
        psij = np.zeros(1)
        v = np.zeros((self.N, 3))
        d2 = np.zeros(1)
        lib().or_jastrow(self.h, dp(np.ascontiguousarray(x, float)), dp(psij), dp(v), dp(d2))
        return psij[0], v, d2[0]

    def jas_raw(self, x):
        """Raw Jastrow parameter derivatives dJ/dp of one configuration
        (a part, b part, c part; see Walker::jas_raw)."""
        out = np.zeros(lib().or_jas_nraw(self.h))
        lib().or_jas_raw(self.h, dp(np.ascontiguousarray(x, float)), dp(out))
        return out

    def slater(self, x):
        s = self.system
        nmax = max(s.nup, s.ndn)
        slmi = np.zeros((2, nmax * nmax))
        det = np.zeros(2)
        rc = lib().or_slater(self.h, dp(np.ascontiguousarray(x, float)), dp(slmi), dp(det))
        if rc:
            raise RuntimeError("singular Slater matrix")
        return slmi, det

    def hpsi(self, x, quad=None):
        out = np.zeros(6)
        if quad is None:
            rc = lib().or_hpsi(self.h, dp(np.ascontiguousarray(x, float)), None, None, None, dp(out))
        else:
            xq, yq, zq = (np.ascontiguousarray(q, float) for q in quad)
            rc = lib().or_hpsi(self.h, dp(np.ascontiguousarray(x, float)), dp(xq), dp(yq), dp(zq), dp(out))
        if rc:
            raise RuntimeError("singular Slater matrix")
        return dict(energy=out[0], psid=out[1], psij=out[2], ekin=out[3], pe_local=out[4], vpsp=out[5])

    def tmove_elements(self, x, quad=None, cap=1 << 16):
        """T-move elements of one configuration after hpsi (nonloc, and
        multideterminant_tmove for an expansion): rows (iel, ic, iq,
        term_radial_jas, t_vpsp) of every quadrature point, and psi_D."""
        L = lib()
        L.or_tmove_elements.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp]
        L.or_tmove_elements.restype = C.c_int
        out = np.zeros((cap, 5))
        psid = np.zeros(1)
        if quad is None:
            q = [None, None, None]
        else:
            q = [dp(np.ascontiguousarray(a, float)) for a in quad]
        n = L.or_tmove_elements(self.h, dp(np.ascontiguousarray(x, float)), q[0], q[1], q[2], cap, dp(out), dp(psid))
        if n < 0:
            raise RuntimeError("singular Slater matrix")
        return out[:min(n, cap)], float(psid[0])

    def orb_o(self, x, ideriv):
        """Orbital-rotation derivatives of one configuration for the 1-based
        pairs ideriv [n][2] (one determinant)."""
        L = lib()
        L.or_orb_o.argtypes = [C.c_void_p, _dp, C.c_int, _i32, _dp]
        d = np.ascontiguousarray(np.asarray(ideriv, np.int32).reshape(-1, 2))
        out = np.zeros(d.shape[0])
        if L.or_orb_o(self.h, dp(np.ascontiguousarray(x, float)), d.shape[0], d.ctypes.data_as(_i32), dp(out)):
            raise RuntimeError("singular Slater matrix")
        return out

    def sites(self, state):
        x = np.zeros((self.N, 3))
        st = np.ascontiguousarray(state, np.uint64).copy()
        lib().or_sites(self.h, u64(st), dp(x))
        return x, st


class OracleWalkers:
    def __init__(self, osys: OracleSystem, x, rng):
        self.osys = osys
        x = np.ascontiguousarray(x, float)
        rng = np.ascontiguousarray(rng, np.uint64)
        self.W = rng.shape[0]
        self.h = lib().or_walkers_create(osys.h, self.W, dp(x), u64(rng))

    def __del__(self):
        try:
            lib().or_walkers_destroy(self.h)
        except Exception:
            pass

    def steps(self, nstep, nthreads=1):
        rc = lib().or_vmc_steps(self.h, nstep, nthreads)
        if rc:
            raise RuntimeError("oracle walker failed (singular matrix)")

    def zerest(self):
        lib().or_zerest(self.h)

    def end_block(self):
        e = np.zeros(1)
        lib().or_end_block(self.h, dp(e))
        return e[0]

    def results(self):
        out = np.zeros(8)
        lib().or_results(self.h, dp(out))
        return dict(energy=out[0], err=out[1], sigma=out[2], tcorr=out[3], accept=out[4], pe=out[5],
                    ke=out[6], nblocks=out[7])

    def results_state(self, istate: int):
        out = np.zeros(8)
        if lib().or_results_state(self.h, istate, dp(out)):
            raise ValueError(f"state {istate} out of range")
        return dict(energy=out[0], err=out[1], pe=out[5], ke=out[6], nblocks=out[7])

    def state_energies(self, nstates: int):
        e = np.zeros((self.W, nstates))
        p = np.zeros((self.W, nstates))
        lib().or_state_energies(self.h, dp(e), dp(p))
        return e, p

    def opt_ci(self, enable=True):
        lib().or_opt_ci(self.h, 1 if enable else 0)

    def ci_o(self):
        nd = self.osys.system.iworbd.shape[0]
        out = np.zeros((self.W, nd))
        lib().or_ci_o(self.h, dp(out))
        return out

    def opt_ci_sums(self):
        nd = self.osys.system.iworbd.shape[0]
        o, eo, oo, w = np.zeros(nd), np.zeros(nd), np.zeros((nd, nd)), np.zeros(1)
        lib().or_opt_ci_sums(self.h, dp(o), dp(eo), dp(oo), dp(w))
        return dict(o=o, eo=eo, oo=oo, wsum=float(w[0]))

    def walkers(self):
        x = np.zeros((self.W, self.osys.N, 3))
        r = np.zeros((self.W, 4), np.uint64)
        lib().or_get_walkers(self.h, dp(x), u64(r))
        return x, r

    def sums(self):
        out = np.zeros((self.W, 5))
        lib().or_get_sums(self.h, dp(out))
        return out

    def state(self):
        e = np.zeros(self.W)
        p = np.zeros(self.W)
        j = np.zeros(self.W)
        lib().or_get_state(self.h, dp(e), dp(p), dp(j))
        return e, p, j

    # per-electron routines of walker k (a metrop6 kept on the host)
    def psie(self, k, iel, xnew3):
        """psie (vmc/hpsie.f90:3) of electron iel of walker k at xnew3: (psid, psij)."""
        L = lib()
        L.or_w1_psie.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp]
        out = np.zeros(2)
        if L.or_w1_psie(self.h, k, iel, dp(np.ascontiguousarray(xnew3, float)), dp(out)):
            raise RuntimeError("singular multideterminant table")
        return out[0], out[1]

    def grad(self, k, iel, iflag_move):
        """compute_determinante_grad: drift of electron iel, 1 = current, 0 = at the last psie point."""
        L = lib()
        L.or_w1_grad.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp]
        v = np.zeros(3)
        L.or_w1_grad(self.h, k, iel, iflag_move, dp(v))
        return v

    def commit(self, k, iel, accept, psidn=0.0, psijn=0.0):
        """metrop6's accept branch (jassav, detsav) or distancese_restore."""
        L = lib()
        L.or_w1_commit.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
        L.or_w1_commit(self.h, k, iel, 1 if accept else 0, float(psidn), float(psijn))

    def update_ymat(self, k, iel):
        L = lib()
        L.or_w1_update_ymat.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.or_w1_update_ymat(self.h, k, iel)


class OracleDmc:
    """DMC population of the oracle (dmc_ps + branching + splitj)."""

    def __init__(self, osys: OracleSystem, x, rng, pop_rng, tau, etrial, mwalk=None, nfprod=100):
        L = lib()
        L.or_dmc_create.restype = C.c_void_p
        L.or_dmc_create.argtypes = [C.c_void_p, C.c_int, _dp, _u64, _u64, C.c_double, C.c_double, C.c_int, C.c_int]
        L.or_dmc_destroy.argtypes = [C.c_void_p]
        L.or_dmc_steps.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.or_dmc_end_block.argtypes = [C.c_void_p]
        L.or_dmc_results.argtypes = [C.c_void_p, _dp]
        L.or_dmc_walkers.argtypes = [C.c_void_p, _dp, _dp, _dp, _u64]
        self.osys = osys
        x = np.ascontiguousarray(x, float)
        W = x.shape[0]
        self.mwalk = mwalk or int(1.5 * W) + 1
        rng = np.ascontiguousarray(rng, np.uint64)
        assert rng.shape[0] >= self.mwalk
        pop = np.ascontiguousarray(pop_rng, np.uint64)
        self.h = L.or_dmc_create(osys.h, W, dp(x), u64(rng), u64(pop), tau, etrial, self.mwalk, nfprod)

    def __del__(self):
        try:
            lib().or_dmc_destroy(self.h)
        except Exception:
            pass

    def steps(self, n, nthreads=1):
        if lib().or_dmc_steps(self.h, n, nthreads):
            raise RuntimeError("oracle DMC failed")

    def set_tmoves(self, icasula: int):
        L = lib()
        L.or_dmc_set_tmoves.argtypes = [C.c_void_p, C.c_int]
        if L.or_dmc_set_tmoves(self.h, icasula):
            raise ValueError("unsupported T-move setting")

    def tmoves(self) -> int:
        L = lib()
        L.or_dmc_tmoves.argtypes = [C.c_void_p]
        L.or_dmc_tmoves.restype = C.c_long
        return int(L.or_dmc_tmoves(self.h))

    def end_block(self):
        lib().or_dmc_end_block(self.h)

    def results(self):
        o = np.zeros(12)
        lib().or_dmc_results(self.h, dp(o))
        return dict(energy=o[0], err=o[1], nwalk=int(o[2]), eest=o[3], accept=o[4], taueff=o[5], pe=o[6],
                    ke=o[7], nblocks=o[8], fprod=o[9], eigv=o[10], wdsumo=o[11])

    def walkers(self):
        N = self.osys.N
        x = np.zeros((self.mwalk, N, 3))
        wt = np.zeros(self.mwalk)
        e = np.zeros(self.mwalk)
        r = np.zeros((self.mwalk, 4), np.uint64)
        n = lib().or_dmc_walkers(self.h, dp(x), dp(wt), dp(e), u64(r))
        return x[:n], wt[:n], e[:n], r[:n]
