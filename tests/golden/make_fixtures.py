"""Regenerates the committed golden fixtures of tests/golden/.

Run where the CHAMP sources are available, with CHAMP_REF set to the root
of that source tree (the script refuses to run without it).  Writes:

* rng_default_seed.npz — next_uniform_double draws and jump() states of the
  reference's own vmc/xoroshiro256starstar.c (compiled into oracle/_ref by
  oracle/Makefile) for CHAMP's default seed (vmc/parser.f90:315);
* vmc_h2_system.npz — the VMC-H2 CI case (tests/CI_test/VMC-H2) read from
  its CHAMP input files and pre-processed as read_bas_num does;
* vmc_c4h6_500_system.npz — the VMC-C4H6-ci1010_pVTZ-00500-dets CI case
  (BFD pseudopotentials, 500 determinants) read the same way.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
REF = os.environ.get("CHAMP_REF", "")


def rng_fixture():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REF}"], check=True)
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libxoshiro_ref.so"))
    lib.next_uniform_double.restype = C.c_double
    seed = "18123437465549275475255231234865"
    irn = (C.c_int32 * 8)(*[int(seed[4 * i:4 * i + 4]) for i in range(8)])
    lib.xoroshiro_set_state(irn)
    draws = np.array([lib.next_uniform_double() for _ in range(64)])
    lib.xoroshiro_set_state(irn)
    states = []
    for _ in range(4):
        st = (C.c_int32 * 8)()
        lib.xoroshiro_get_state(st)
        states.append(np.frombuffer(bytes(st), dtype=np.uint64).copy())
        lib.jump()
    np.savez(os.path.join(HERE, "rng_default_seed.npz"), draws=draws, jump_states=np.array(states))


def h2_fixture():
    from champ_b200.champ_io import load_champ, save_npz
    d = os.path.join(REF, "tests", "CI_test", "VMC-H2") + "/"
    s = load_champ("vmc_h2", d + "pool/champ_v3_h2.xyz", d + "pool/champ_v3_sto_cvb1_basis_pointers.bfinfo",
                   d + "pool", "sto_cvb1", d + "champ_v3_trexio_order_rhf.sto_cvb1.lcao", d + "rhf.det",
                   d + "jastrow.0", nelec=2, nup=1, nloc=0, znuc={"H": 1.0})
    save_npz(s, os.path.join(HERE, "vmc_h2_system.npz"))


def c4h6_fixture():
    """tests/CI_test/VMC-C4H6-ci1010_pVTZ-00500-dets: butadiene, BFD
    pseudopotentials (C: local + s channel, H: local), BFD-T numerical basis
    with f functions (226 AOs), 500 determinants, Jastrow 5 5 0 (no e-e-n
    terms).  Orbitals beyond the highest one the determinants use (89) are
    dropped: they do not enter psi."""
    from champ_b200.champ_io import load_champ, save_npz
    d = os.path.join(REF, "tests", "CI_test", "VMC-C4H6-ci1010_pVTZ-00500-dets") + "/"
    s = load_champ("vmc_c4h6_500", d + "pool/champ_v3_butadiene.xyz",
                   d + "pool/champ_v3_BFD-T_basis_pointers.bfinfo", d + "pool", "BFD-T",
                   d + "champ_v3_trexio_order_ci1010_pVTZ_1_orbitals.lcao", d + "TZ_1M_500.det",
                   d + "jastrow_good_b3lyp.0", nelec=22, nup=11, nloc=4, pp_dir=d + "pool", pp_id="BFD",
                   znuc={"C": 4.0, "H": 1.0})
    s.coef = s.coef[:int(s.iworbd.max())].copy()
    save_npz(s, os.path.join(HERE, "vmc_c4h6_500_system.npz"))


if __name__ == "__main__":
    if not REF or not os.path.isdir(os.path.join(REF, "src")):
        sys.exit("set CHAMP_REF to the root of a CHAMP source tree")
    rng_fixture()
    h2_fixture()
    c4h6_fixture()
    print("fixtures written to", HERE)
