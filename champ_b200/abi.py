"""ctypes mirror of include/champ_b200.h.

The structure layout below must match ``cw_system_desc`` field for field.
``load_engine`` opens the CUDA engine library built in-tree; it raises when
the library is missing, so no product path can silently run without it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ENGINE_LIB = os.path.join(HERE, "libchamp_b200.so")

CW_NCOEF = 5
CW_MPS_L = 4
CW_MGAUSS = 16
CW_MPS_QUAD = 86

CW_PREC_FP64 = 0
CW_PREC_MIXED = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class CwSystemDesc(C.Structure):
    _fields_ = [
        ("nelec", C.c_int32), ("nup", C.c_int32),
        ("ncent", C.c_int32), ("nctype", C.c_int32),
        ("iwctype", _ip), ("cent", _dp), ("znuc", _dp), ("pecent", C.c_double),
        ("mrwf", C.c_int32), ("mrwf_pts", C.c_int32),
        ("nrbas", _ip), ("igrid", _ip), ("nr", _ip),
        ("arg", _dp), ("r0", _dp), ("rwf", _dp), ("d2rwf", _dp), ("ce", _dp), ("ae", _dp),
        ("rmaxwf", _dp),
        ("mbastyp", C.c_int32), ("nbastyp", _ip), ("iwlbas", _ip), ("iwrwf", _ip),
        ("nbasis", C.c_int32), ("norb", C.c_int32), ("coef", _dp),
        ("ndet", C.c_int32), ("iworbd", _ip), ("cdet", _dp),
        ("norda", C.c_int32), ("nordb", C.c_int32), ("nordc", C.c_int32),
        ("isc", C.c_int32), ("nspin2b", C.c_int32), ("nocuspb", C.c_int32),
        ("scalek", C.c_double), ("a4", _dp), ("b", _dp), ("c", _dp),
        ("nloc", C.c_int32), ("lpot", _ip), ("necp_term", _ip), ("necp_power", _ip),
        ("ecp_exponent", _dp), ("ecp_coef", _dp),
        ("nquad", C.c_int32), ("xq0", _dp), ("yq0", _dp), ("zq0", _dp), ("wq", _dp),
        ("deltar", C.c_double), ("deltat", C.c_double), ("fbias", C.c_double),
        ("nstates", C.c_int32), ("iguiding", C.c_int32), ("weights_g", _dp),
    ]


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def u64ptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def optd(a):
    return dptr(a) if a is not None else None


_engine = None


def load_engine(path: str | None = None):
    """Open the CUDA engine library (built by champ_b200.build)."""
    global _engine
    if _engine is not None and path is None:
        return _engine
    p = path or ENGINE_LIB
    if not os.path.exists(p):
        raise RuntimeError(
            f"CUDA engine library {p} is missing: build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)")
    lib = C.CDLL(p)
    V = C.c_void_p
    lib.cw_create.argtypes = [C.POINTER(V), C.POINTER(CwSystemDesc), C.c_int, C.c_int]
    lib.cw_create.restype = C.c_int
    lib.cw_destroy.argtypes = [V]
    lib.cw_destroy.restype = None
    lib.cw_last_error.argtypes = [V]
    lib.cw_last_error.restype = C.c_char_p
    lib.cw_sync.argtypes = [V]
    lib.cw_set_walkers.argtypes = [V, C.c_int, _dp, C.POINTER(C.c_uint64)]
    lib.cw_get_walkers.argtypes = [V, _dp, C.POINTER(C.c_uint64)]
    lib.cw_vmc_steps.argtypes = [V, C.c_int]
    lib.cw_end_block.argtypes = [V, _dp]
    lib.cw_results.argtypes = [V, _dp]
    lib.cw_hpsi.argtypes = [V, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
    lib.cw_orbitals.argtypes = [V, _dp, _dp, _dp]
    lib.cw_jastrow.argtypes = [V, _dp, _dp, _dp]
    lib.cw_slater.argtypes = [V, _dp, _dp]
    lib.cw_get_sums.argtypes = [V, _dp]
    lib.cw_get_state.argtypes = [V, _dp, _dp, _dp]
    lib.cw_last_ms.argtypes = [V]
    lib.cw_last_ms.restype = C.c_double
    lib.cw_launches.argtypes = [V]
    lib.cw_launches.restype = C.c_long
    lib.cw_device_bytes.argtypes = [V]
    lib.cw_device_bytes.restype = C.c_size_t
    lib.cw_results_state.argtypes = [V, C.c_int, _dp]
    lib.cw_state_energies.argtypes = [V, _dp, _dp]
    lib.cw_opt_ci.argtypes = [V, C.c_int, C.c_int]
    lib.cw_opt_ci_sums.argtypes = [V, _dp, _dp, _dp, _dp]
    lib.cw_ci_o.argtypes = [V, _dp]
    lib.cw_opt_setup.argtypes = [V, C.c_int, C.c_int, _dp, C.c_int]
    lib.cw_opt_sums.argtypes = [V, _dp, _dp, _dp, _dp]
    lib.cw_jas_nraw.argtypes = [V, C.POINTER(C.c_int)]
    lib.cw_jas_raw.argtypes = [V, _dp]
    lib.cw_jas_o.argtypes = [V, _dp]
    lib.cw_profile.argtypes = [V, C.c_int]
    lib.cw_profile.restype = C.c_int
    lib.cw_stage_times.argtypes = [V, _dp, C.POINTER(C.c_long)]
    lib.cw_stage_times.restype = C.c_int
    lib.cw_orbitals_noalloc.argtypes = [V, C.c_int, C.c_void_p, C.c_void_p]
    lib.cw_orbitals_noalloc.restype = C.c_int
    lib.cw_fma_peak.argtypes = [C.c_int, C.c_int, _dp]
    lib.cw_fma_peak.restype = C.c_int
    lib.cw_rng_states.argtypes = [C.POINTER(C.c_int32), C.c_int, C.POINTER(C.c_uint64)]
    lib.cw_sites.argtypes = [C.POINTER(CwSystemDesc), C.c_int, C.POINTER(C.c_uint64), _dp]
    lib.cw_dmc_init.argtypes = [V, C.c_int, C.c_int, _dp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                C.c_double, C.c_double, C.c_int]
    lib.cw_dmc_steps.argtypes = [V, C.c_int]
    lib.cw_dmc_end_block.argtypes = [V]
    lib.cw_dmc_results.argtypes = [V, _dp]
    lib.cw_dmc_walkers.argtypes = [V, C.POINTER(C.c_int), _dp, _dp, _dp, C.POINTER(C.c_uint64)]
    lib.cw_dmc_set_tmoves.argtypes = [V, C.c_int]
    lib.cw_dmc_counts.argtypes = [V, C.POINTER(C.c_long)]
    lib.cw_checkpoint_bytes.argtypes = [V]
    lib.cw_checkpoint_bytes.restype = C.c_long
    lib.cw_checkpoint.argtypes = [V, C.c_void_p, C.c_long]
    lib.cw_restore.argtypes = [V, C.c_void_p, C.c_long]
    lib.cw_walker_status.argtypes = [V, C.POINTER(C.c_int32)]
    lib.cw_stamp.argtypes = [V]
    lib.cw_autotune.argtypes = [V, C.c_int, C.POINTER(C.c_int32)]
    lib.cw_batch_create.argtypes = [C.POINTER(V), C.POINTER(V), C.c_int]
    lib.cw_batch_create.restype = C.c_int
    lib.cw_batch_vmc_steps.argtypes = [V, C.c_int]
    lib.cw_batch_vmc_steps.restype = C.c_int
    lib.cw_batch_last_ms.argtypes = [V]
    lib.cw_batch_last_ms.restype = C.c_float
    lib.cw_batch_last_error.argtypes = [V]
    lib.cw_batch_last_error.restype = C.c_char_p
    lib.cw_batch_destroy.argtypes = [V]
    lib.cw_batch_destroy.restype = None
    lib.cw_batch_set_ragged.argtypes = [V, C.c_int]
    lib.cw_batch_set_ragged.restype = C.c_int
    lib.cw_batch_info.argtypes = [V, C.POINTER(C.c_int64)]
    lib.cw_batch_info.restype = C.c_int
    lib.cw_stamps.argtypes = [V, C.POINTER(C.c_int64), C.c_int]
    lib.cw_psie.argtypes = [V, C.c_int, _dp, _dp, _dp]
    lib.cw_grad.argtypes = [V, C.c_int, C.c_int, _dp]
    lib.cw_commit.argtypes = [V, C.c_int, C.POINTER(C.c_int32)]
    lib.cw_update_ymat.argtypes = [V, C.c_int]
    lib.cw_opt_orb.argtypes = [V, C.c_int, C.POINTER(C.c_int32)]
    lib.cw_orb_o.argtypes = [V, _dp]
    for f in ("cw_dmc_set_tmoves", "cw_dmc_counts", "cw_checkpoint", "cw_restore", "cw_dmc_init", "cw_dmc_steps", "cw_dmc_end_block", "cw_dmc_results", "cw_dmc_walkers",
              "cw_rng_states", "cw_sites", "cw_sync", "cw_set_walkers", "cw_get_walkers", "cw_vmc_steps", "cw_end_block",
              "cw_results", "cw_hpsi", "cw_orbitals", "cw_jastrow", "cw_slater",
              "cw_get_sums", "cw_get_state", "cw_results_state", "cw_state_energies", "cw_opt_ci",
              "cw_opt_ci_sums", "cw_ci_o", "cw_opt_setup", "cw_opt_sums", "cw_jas_nraw", "cw_jas_raw", "cw_jas_o",
              "cw_walker_status", "cw_stamp", "cw_stamps", "cw_autotune", "cw_psie", "cw_grad", "cw_commit",
              "cw_update_ymat", "cw_opt_orb", "cw_orb_o"):
        getattr(lib, f).restype = C.c_int
    if path is None:
        _engine = lib
    return lib


EXPORTED_SYMBOLS = [
    "cw_create", "cw_destroy", "cw_last_error", "cw_sync", "cw_set_walkers", "cw_get_walkers",
    "cw_vmc_steps", "cw_end_block", "cw_results", "cw_hpsi", "cw_orbitals", "cw_jastrow",
    "cw_slater", "cw_get_sums", "cw_get_state", "cw_last_ms", "cw_rng_states", "cw_sites",
    "cw_launches", "cw_profile", "cw_stage_times", "cw_fma_peak", "cw_orbitals_noalloc",
    "cw_dmc_init", "cw_dmc_steps", "cw_dmc_end_block", "cw_dmc_results", "cw_dmc_walkers",
    "cw_checkpoint_bytes", "cw_checkpoint", "cw_restore", "cw_dmc_set_tmoves", "cw_dmc_counts",
    "cw_device_bytes", "cw_results_state", "cw_state_energies", "cw_opt_ci", "cw_opt_ci_sums", "cw_ci_o",
    "cw_opt_setup", "cw_opt_sums", "cw_jas_nraw", "cw_jas_raw", "cw_jas_o",
    "cw_walker_status", "cw_stamp", "cw_stamps", "cw_autotune", "cw_batch_create", "cw_batch_vmc_steps",
    "cw_batch_last_ms", "cw_batch_last_error", "cw_batch_destroy", "cw_batch_set_ragged", "cw_batch_info", "cw_psie", "cw_grad", "cw_commit", "cw_update_ymat", "cw_opt_orb", "cw_orb_o",
]
STAGES = ["rotqua", "propose", "jastrow_move", "basis_move", "lcao_move", "accept", "jastrow_full",
          "basis_all", "lcao_all", "scatter", "slater_inv", "ctilde", "ecp", "energy", "commit", "dmc_weights", "splitj", "mdet", "tmove"]
