"""Readers for CHAMP's input files (the formats vmc/read_data_parser.f90 reads).

Supported: .xyz molecule (read_molecule_file), basis pointers .bfinfo
(read_basis_num_info_file :2035), numerical radial basis grids
<basis>.basis.<atom> (read_bas_num vmc/read_bas_num.f90:11), .lcao
(read_orbitals_file :925), .det (read_determinants_file), Jastrow
(read_jastrow_file :532) and Gaussian ECPs <pp>.gauss_ecp.dat.<atom>
(readps_gauss vmc/read_bas_num.f90:338).
"""
from __future__ import annotations

import os

import numpy as np

from .abi import CW_MGAUSS, CW_MPS_L
from .system import System, assemble_basis, gesqua, nterms4, prepare_radial, SLM_OF_L


def _lines(path):
    with open(path) as f:
        return [ln.rstrip("\n") for ln in f]


def read_xyz(path):
    ln = _lines(path)
    n = int(ln[0].split()[0])
    labels, cent = [], []
    for k in range(2, 2 + n):
        p = ln[k].split()
        labels.append(p[0])
        cent.append([float(v) for v in p[1:4]])
    return labels, np.array(cent)


def read_bfinfo(path, ntypes):
    ln = [l for l in _lines(path) if l.strip() and not l.strip().startswith("#")]
    k = 0
    while not ln[k].split()[0] in ("qmc_bf_info", "basis"):
        k += 1
    k += 1
    out = []
    for _ in range(ntypes):
        counts = [int(v) for v in ln[k].split()[:6]]
        iwl = [int(v) for v in ln[k + 1].split()[:counts[0]]]
        iwr = [int(v) for v in ln[k + 2].split()[:counts[0]]]
        out.append(dict(nbastyp=counts[0], ns=counts[1:], iwlbas=iwl, iwrwf=iwr))
        k += 3
    return out


def read_basis_grid(path, nloc):
    ln = _lines(path)
    h = ln[0].split()
    nrbas, igrid, nr = int(h[0]), int(h[1]), int(h[2])
    arg, r0, icusp = float(h[3]), float(h[4]), int(h[5])
    k = 1
    lvals = None
    if nloc == 0:
        lvals = [int(v) for v in ln[1].split()[:nrbas]]
        k = 2
    data = np.array([[float(v) for v in ln[k + i].split()[:nrbas + 1]] for i in range(nr)])
    return dict(nrbas=nrbas, igrid=igrid, nr=nr, arg=arg, r0=r0, icusp=icusp, lvals=lvals,
                x=data[:, 0].copy(), rwf=np.ascontiguousarray(data[:, 1:].T))


def read_lcao(path):
    ln = [l for l in _lines(path) if l.strip() and not l.strip().startswith("#")]
    h = ln[0].split()
    norb, nbasis = int(h[1]), int(h[2])
    vals = []
    k = 1
    while len(vals) < norb * nbasis:
        vals.extend(float(v) for v in ln[k].split())
        k += 1
    return np.array(vals[:norb * nbasis]).reshape(norb, nbasis)


def read_det(path, nelec):
    ln = [l for l in _lines(path) if l.strip() and not l.strip().startswith("#")]
    h = ln[0].split()
    ndet = int(h[1])
    cdet = np.array([float(v) for v in ln[1].split()[:ndet]])
    iworbd = np.array([[int(v) for v in ln[2 + k].split()[:nelec]] for k in range(ndet)], np.int32)
    return cdet, iworbd


def expand_csf(ccsf, csfmap, ndet):
    """Determinant coefficients of every state from CSF coefficients
    (read_csfmap_file, vmc/read_data_parser.f90:1284): ccsf [nstates][ncsf],
    csfmap[icsf] = [(det index 1-based, coefficient), ...];
    cdet[k][jx] = sum_icsf ccsf[k][icsf] * c for every (jx, c) of csf icsf."""
    ccsf = np.atleast_2d(np.asarray(ccsf, float))
    if ccsf.shape[1] != len(csfmap):
        raise ValueError("CSFMAP: wrong number of csf")
    out = np.zeros((ccsf.shape[0], ndet))
    for k in range(ccsf.shape[0]):
        for icsf, terms in enumerate(csfmap):
            for jd, c in terms:
                if not 1 <= jd <= ndet:
                    raise ValueError("id in CSFMAP larger than ndet")
                out[k, jd - 1] += ccsf[k, icsf] * c
    return out


def read_det_states(path, nelec):
    """.det file with optional csf / csfmap sections (read_csf_file,
    read_csfmap_file): returns (cdet_states [nstates][ndet], iworbd).  Without
    a csf section the file's determinant coefficients are the one state."""
    cdet, iworbd = read_det(path, nelec)
    ln = [l.split() for l in _lines(path) if l.strip() and not l.strip().startswith("#")]
    heads = {t[0].lower(): i for i, t in enumerate(ln)}
    if "csf" not in heads:
        return cdet[None, :], iworbd
    i = heads["csf"]
    ncsf, nstates = int(ln[i][1]), int(ln[i][2])
    ccsf = np.array([[float(v) for v in ln[i + 1 + k][:ncsf]] for k in range(nstates)])
    if "csfmap" not in heads:                    # one determinant per CSF, in order
        return expand_csf(ccsf, [[(j + 1, 1.0)] for j in range(ncsf)], len(cdet)), iworbd
    i = heads["csfmap"]
    ncsf_m, ndet_m, nmap = int(ln[i][1]), int(ln[i][2]), int(ln[i][3])
    if ndet_m != len(cdet) or ncsf_m != ncsf:
        raise ValueError("CSFMAP: wrong number of determinants or csf")
    p = i + 1
    csfmap = []
    for _ in range(ncsf):
        nterm = int(ln[p][0])
        csfmap.append([(int(ln[p + 1 + t][0]), float(ln[p + 1 + t][1])) for t in range(nterm)])
        p += 1 + nterm
    if sum(len(t) for t in csfmap) != nmap:
        raise ValueError("Error in CSFMAP:: not enough nmaps / file is corrupt")
    return expand_csf(ccsf, csfmap, len(cdet)), iworbd


def read_jastrow(path, nctype, nspin2b=1):
    ln = [l for l in _lines(path) if l.strip()]
    assert ln[0].split()[0] == "jastrow_parameter"
    norda, nordb, nordc = (int(v) for v in ln[1].split()[:3])
    scalek = float(ln[2].split()[0])
    k = 3
    na, nb, nc = 2 + max(0, norda - 1), 2 + max(0, nordb - 1), nterms4(nordc)

    def take(n):
        nonlocal k
        vals = []
        while len(vals) < n:
            toks = ln[k].split()
            for t in toks:
                try:
                    vals.append(float(t))
                except ValueError:
                    break
                if len(vals) == n:
                    break
            k += 1
        return vals

    a4 = np.array([take(na) for _ in range(nctype)])
    b = np.array([take(nb) for _ in range(nspin2b)])
    c = np.array([take(nc) for _ in range(nctype)]) if nc > 0 else np.zeros((nctype, 0))
    return dict(norda=norda, nordb=nordb, nordc=nordc, scalek=scalek, a4=a4, b=b, c=c)


def read_gauss_ecp(path):
    ln = [l for l in _lines(path)]
    lpot = int(ln[1].split()[0])
    k = 2
    nterm = np.zeros(CW_MPS_L, np.int32)
    power = np.zeros((CW_MPS_L, CW_MGAUSS), np.int32)
    expo = np.zeros((CW_MPS_L, CW_MGAUSS))
    coef = np.zeros((CW_MPS_L, CW_MGAUSS))
    for l in range(1, lpot + 1):
        idx = lpot if l == 1 else l - 1
        n = int(ln[k].split()[0])
        k += 1
        nterm[idx - 1] = n
        for i in range(n):
            p = ln[k].split()
            coef[idx - 1, i] = float(p[0])
            power[idx - 1, i] = int(float(p[1]))
            expo[idx - 1, i] = float(p[2])
            k += 1
    return lpot, nterm, power, expo, coef


def load_champ(name, xyz, bfinfo, basis_dir, basis_id, lcao, det, jastrow, nelec, nup, nloc=0,
               pp_dir=None, pp_id=None, nquad=6, znuc=None):
    """Assemble a System from CHAMP input files."""
    labels, cent = read_xyz(xyz)
    types = []
    for lab in labels:
        if lab not in types:
            types.append(lab)
    iwctype = np.array([types.index(l) for l in labels], np.int32)
    bf = read_bfinfo(bfinfo, len(types))
    zn = np.array([znuc[t] for t in types], float)
    tdefs = []
    for it, t in enumerate(types):
        g = read_basis_grid(os.path.join(basis_dir, f"{basis_id}.basis.{t}"), nloc)
        prep = prepare_radial(g["x"], g["rwf"], g["igrid"], g["arg"], g["r0"], zn[it], nloc,
                              g["lvals"], g["icusp"])
        aos = list(zip(bf[it]["iwlbas"], bf[it]["iwrwf"]))
        tdefs.append(dict(prep=prep, aos=aos, igrid=g["igrid"]))
    basis = assemble_basis(tdefs)
    coef = read_lcao(lcao)
    cdet, iworbd = read_det(det, nelec)
    jas = read_jastrow(jastrow, len(types))
    sysd = dict(name=name, nelec=nelec, nup=nup, iwctype=iwctype, cent=cent, znuc=zn, coef=coef,
                iworbd=iworbd, cdet=cdet, **jas, **basis)
    if nloc:
        lpot = np.zeros(len(types), np.int32)
        nt = np.zeros((len(types), CW_MPS_L), np.int32)
        pw = np.zeros((len(types), CW_MPS_L, CW_MGAUSS), np.int32)
        ex = np.zeros((len(types), CW_MPS_L, CW_MGAUSS))
        co = np.zeros((len(types), CW_MPS_L, CW_MGAUSS))
        for it, t in enumerate(types):
            lpot[it], nt[it], pw[it], ex[it], co[it] = read_gauss_ecp(
                os.path.join(pp_dir, f"{pp_id}.gauss_ecp.dat.{t}"))
        xq, yq, zq, wq = gesqua(nquad)
        sysd.update(nloc=nloc, lpot=lpot, necp_term=nt, necp_power=pw, ecp_exponent=ex, ecp_coef=co,
                    nquad=nquad, xq0=xq, yq0=yq, zq0=zq, wq=wq)
    return System(**sysd)


def save_npz(system: System, path):
    d = {k: getattr(system, k) for k in system.__dataclass_fields__ if not k.startswith("_")}
    d = {k: (np.asarray(v) if v is not None else np.zeros(0)) for k, v in d.items()}
    np.savez_compressed(path, **d)


def load_npz(path) -> System:
    z = np.load(path, allow_pickle=False)
    kw = {}
    for k in System.__dataclass_fields__:
        if k.startswith("_") or k not in z:
            continue
        v = z[k]
        if v.ndim == 0:
            v = v.item()
        elif v.size == 0 and k in ("lpot", "necp_term", "necp_power", "ecp_exponent", "ecp_coef",
                                   "xq0", "yq0", "zq0", "wq"):
            v = None
        kw[k] = v
    if isinstance(kw.get("name"), bytes):
        kw["name"] = kw["name"].decode()
    return System(**kw)
