"""CPU tests of the C ABI library: it loads, exports every entry point the
header declares, and its host-only helpers agree with the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "champ_b200.h")).read()
    return sorted(set(re.findall(r"\b(cw_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from champ_b200 import build
    from champ_b200.abi import load_engine
    build.build()
    return load_engine()


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
    from champ_b200.abi import EXPORTED_SYMBOLS
    assert sorted(EXPORTED_SYMBOLS) == names


def test_host_rng_states_match_oracle(lib, oracle_mod):
    from champ_b200.engine import rng_states
    assert np.array_equal(rng_states(9), oracle_mod.rng_states(9))


def test_host_sites_match_oracle(lib, oracle_mod):
    from champ_b200.engine import initial_configs, rng_states
    from champ_b200.system import make_synthetic
    s = make_synthetic("tiny")
    r = rng_states(3)
    x = initial_configs(s, r)
    o = oracle_mod.OracleSystem(s)
    r0 = oracle_mod.rng_states(3)
    for w in range(3):
        xo, so = o.sites(r0[w])
        assert np.array_equal(x[w], xo)
        assert np.array_equal(r[w], so)


def test_create_rejects_bad_input_without_gpu(lib):
    # argument validation happens before any device call
    from champ_b200.system import make_synthetic
    from champ_b200.abi import CW_PREC_FP64
    s = make_synthetic("tiny")
    d = s.desc()
    d.ndet = 0
    h = C.c_void_p()
    rc = lib.cw_create(C.byref(h), C.byref(d), 0, CW_PREC_FP64)
    assert rc == 1
    assert b"ndet" in lib.cw_last_error(h)
    lib.cw_destroy(h)
    d = s.desc()
    d.nquad = 40
    h = C.c_void_p()
    assert lib.cw_create(C.byref(h), C.byref(d), 0, CW_PREC_FP64) == 1
    assert b"nquad" in lib.cw_last_error(h)
    lib.cw_destroy(h)
