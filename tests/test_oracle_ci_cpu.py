"""The oracle against CHAMP's own CI reference energy for a case with
pseudopotentials and a multideterminant expansion.

tests/CI_test/VMC-C4H6-ci1010_pVTZ-00500-dets (butadiene, BFD
pseudopotentials on C and H, BFD-T numerical basis with f functions, 500
determinants with up to double excitations per spin, Jastrow 5 5 0) runs
vmc.mov1 on 1 and 2 MPI ranks with CHAMP's default seed, 1 equilibration
block and 100 blocks of 20 steps (vmc_optimization_500.inp).  The oracle
runs the same schedule with walkers in the role of ranks, and the energy
must pass tools/compare_value.py:26 (|E - E_ref| <= 2 sqrt(err^2 +
err_ref^2)) against the references of
VMC_C4H6_ci1010_pVTZ_500-dets_butadiene_optimization.sh.  This pins the
restatement of the BFD pseudopotential quadrature (nonloc), the
multideterminant tables (multideterminante, update_ymat,
multideterminant_hpsi) and the f-function Slm together.  The case carries
no e-e-n Jastrow terms (nordc = 0)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

REFS = {1: (-26.1993642, 0.0233401), 2: (-26.181223, 0.0178963)}


def c4h6():
    from champ_b200.champ_io import load_npz
    return load_npz(os.path.join(GOLDEN, "vmc_c4h6_500_system.npz"))


@pytest.mark.parametrize("nranks", [1, 2])
def test_vmc_c4h6_500_dets_ci_energy(oracle_mod, nranks):
    s = c4h6()
    o = oracle_mod.OracleSystem(s)
    rng = oracle_mod.rng_states(nranks)
    xs = []
    for w in range(nranks):
        x, rng[w] = o.sites(rng[w])
        xs.append(x)
    ow = oracle_mod.OracleWalkers(o, np.array(xs), rng)
    ow.steps(20, nranks)      # vmc_nblkeq 1 block of vmc_nstep 20, discarded
    ow.zerest()
    for _ in range(100):      # vmc_nblk 100
        ow.steps(20, nranks)
        ow.end_block()
    r = ow.results()
    e_ref, err_ref = REFS[nranks]
    print(f"{nranks} rank(s): oracle {r['energy']:.5f} +- {r['err']:.5f}, CHAMP {e_ref} +- {err_ref}")
    assert abs(r["energy"] - e_ref) <= 2.0 * np.sqrt(r["err"] ** 2 + err_ref ** 2)
    assert 0.4 < r["accept"] < 0.7


def test_c4h6_fixture_shape():
    s = c4h6()
    assert (s.nelec, s.nup, s.ncent, s.nbasis, s.iworbd.shape[0]) == (22, 11, 10, 226, 500)
    assert s.nloc == 4 and list(s.lpot) == [2, 1] and s.nordc == 0
    assert int(s.iwlbas.max()) == 20   # f functions (Slm 11-20)
