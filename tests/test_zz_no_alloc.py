"""cw_orbitals_noalloc — the allocation-free orbital entry point — against
cw_orbitals on the same walker positions.

The entry point serves callers that cannot call cudaMalloc while they run
(device memory owned by another allocator, or a step loop that cannot take
cudaMalloc's implicit device synchronisation); its scratch is a fixed array
inside the library.  The test allocates the device input/output buffers
itself (with torch) and calls the entry point twice in a row, since every
call reuses the same fixed array.  Kept in a file of its own, collected
last."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _reference_rows(eng, s):
    orb, dorb, ddorb = eng.orbitals()      # existing entry point cw_orbitals
    W, N, O = orb.shape[0], s.nelec, s.norb
    ref = np.zeros((W * N, 5, O))
    for w in range(W):
        for e in range(N):
            p = w * N + e
            ref[p, 0] = orb[w, :, e]
            for k in range(3):
                ref[p, 1 + k] = dorb[w, k, e, :]
            ref[p, 4] = ddorb[w, e, :]
    return ref


def test_orbitals_noalloc_matches_cw_orbitals():
    import torch
    from champ_b200.abi import load_engine
    from champ_b200.engine import Engine, initial_configs, rng_states
    from champ_b200.system import make_synthetic
    lib = load_engine()
    s = make_synthetic("c0")
    W = 8
    rng = rng_states(W)
    x = initial_configs(s, rng)
    eng = Engine(s, device=0)
    npts = W * s.nelec
    out = torch.empty((npts, 5, s.norb), dtype=torch.float64, device="cuda:0")
    for call, shift in enumerate((0.0, 0.37)):   # two calls in a row, different points
        xs = x + shift
        eng.set_walkers(xs, rng)
        ref = _reference_rows(eng, s)
        pts = torch.tensor(xs.reshape(npts, 3), dtype=torch.float64, device="cuda:0")
        out.fill_(np.nan)
        rc = lib.cw_orbitals_noalloc(eng.h, npts, C.c_void_p(pts.data_ptr()), C.c_void_p(out.data_ptr()))
        assert rc == 0, lib.cw_last_error(eng.h)
        assert lib.cw_sync(eng.h) == 0
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), f"call {call}: unwritten outputs"
        assert rel_err(got, ref) < TOL, f"call {call}"


def test_orbitals_noalloc_rejects_oversize():
    import torch
    from champ_b200.abi import load_engine
    from champ_b200.engine import Engine
    from champ_b200.system import make_synthetic
    lib = load_engine()
    s = make_synthetic("c0")
    eng = Engine(s, device=0)
    limit = (2 * 1024 * 1024) // (5 * s.nbasis)
    pts = torch.zeros((limit + 1, 3), dtype=torch.float64, device="cuda:0")
    out = torch.zeros((limit + 1, 5, s.norb), dtype=torch.float64, device="cuda:0")
    rc = lib.cw_orbitals_noalloc(eng.h, limit + 1, C.c_void_p(pts.data_ptr()), C.c_void_p(out.data_ptr()))
    assert rc == 1
    assert b"exceed the fixed scratch" in lib.cw_last_error(eng.h)
