"""Real-space lattice, neighbour shells and Slater-Koster hoppings.

Host-side restatement of the reference's model set-up; it produces the
neighbour table (cell vector, basis index, per-site hopping blocks t0i) that
the H(k) Fourier sum consumes:

* ``read_basis``         -- source/mod_polyBasis.F90:23-170
* ``generate_neighbors`` -- source/Lattice.F90:40-157 (shells within relTol)
* ``sort_neighbors``     -- source/Lattice.F90:159-233
* ``read_element``       -- source/TightBinding.F90:221-653 (SK mode)
* ``intd``               -- source/TightBinding.F90:655-783 (two-centre table)
* ``sk_hoppings``        -- source/TightBinding.F90:93-219 (geometric mixing,
                            Andersen scaling law, orbital selection)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

DEFAULT_ORBS = ["s", "px", "py", "pz", "dxy", "dyz", "dzx", "dx2", "dz2"]
SQ3 = math.sqrt(3.0)


def _floats(line: str, n: int):
    out = []
    for tok in line.replace(",", " ").split():
        if tok.startswith("!"):
            break
        try:
            out.append(float(tok.replace("d", "e").replace("D", "e")))
        except ValueError:
            break
        if len(out) == n:
            break
    return out


def _is_numeric(tok: str) -> bool:
    try:
        float(tok.replace("d", "e").replace("D", "e"))
        return True
    except ValueError:
        return False


@dataclass
class Basis:
    name: str
    a0: float
    a1: np.ndarray
    a2: np.ndarray
    a3: np.ndarray
    type_names: list
    atom_type: list          # 0-based type index per atom
    positions: np.ndarray    # [nAtoms, 3]
    sysdim: int = 3


def read_basis(path: str, read_sysdim: bool = False) -> Basis:
    """Read a reference-format 'basis' file (mod_polyBasis.F90:23-170)."""
    with open(path) as f:
        lines = [l.rstrip("\n") for l in f]
    it = iter(lines)
    name = next(it).strip()
    a0 = _floats(next(it), 1)[0]
    a1 = np.array(_floats(next(it), 3)) * a0
    a2 = np.array(_floats(next(it), 3)) * a0
    a3 = np.array(_floats(next(it), 3)) * a0
    names = []
    for tok in next(it).split():
        if tok.startswith("!"):
            break
        names.append(tok)
    counts = [int(x) for x in next(it).split()[:len(names)]]
    coord = next(it).split()[0]
    types, pos = [], []
    for t, c in enumerate(counts):
        for _ in range(c):
            line = ""
            while len(line.strip()) == 0:
                line = next(it)
            p = np.array(_floats(line, 3))
            if coord in ("C", "c", "K", "k"):
                p = p * a0
            else:
                p = p[0] * a1 + p[1] * a2 + p[2] * a3
            types.append(t)
            pos.append(p)
    sysdim = 3
    if read_sysdim:
        sysdim = int(_floats(next(it), 1)[0])
    return Basis(name, a0, a1, a2, a3, names, types, np.array(pos), sysdim)


@dataclass
class Element:
    """Parameters of one element file (TightBinding.F90:221-653, tbmode = 1)."""
    name: str
    lattice_constant: float
    a: np.ndarray                 # [3, 3] Bravais vectors (columns a1,a2,a3) times a0
    sub_types: list
    lelement: np.ndarray          # which atoms of the element file are this element
    positions: np.ndarray
    sysdim: int
    orbs: list                    # 1-based default orbital indices (1..9)
    fermi: float
    occ: tuple
    Un: float
    Um: float
    lambda_p: float
    lambda_d: float
    onsite: np.ndarray            # [nOrb, nOrb]
    hopping: np.ndarray           # [10, nStages]
    stage: np.ndarray = field(default=None)  # [nStages, nAtomsFile]


def _orbital_list(tokens):
    orbs = []
    for t in tokens:
        if t.startswith("!"):
            break
        if _is_numeric(t):
            orbs.append(int(float(t)))
        else:
            orbs.append(DEFAULT_ORBS.index(t[:3].strip()) + 1)
    return orbs


def read_element(path: str, name: str, n_stages: int, rel_tol: float, sys_orbs,
                 soc: bool = True, socscale: float = 1.0) -> Element:
    """Read an SK element file and compute its neighbour stage distances."""
    with open(path) as f:
        raw = [l.rstrip("\n") for l in f]
    # next_line skips empty lines and comment lines
    lines = [l for l in raw[1:] if l.strip() and not l.strip().startswith("!")]
    it = iter(lines)
    a0 = _floats(next(it), 1)[0]
    brav = np.zeros((3, 3))
    for j in range(3):
        brav[:, j] = _floats(next(it), 3)
    brav = brav * a0
    sub = []
    for tok in next(it).split():
        if tok.startswith("!"):
            break
        sub.append(tok)
    counts = [int(float(x)) for x in next(it).split()[:len(sub)]]
    coord = next(it).split()[0]
    lel, pos = [], []
    for t, c in enumerate(counts):
        for _ in range(c):
            p = np.array(_floats(next(it), 3))
            if coord in ("C", "c", "K", "k"):
                p = p * a0
            else:
                p = p[0] * brav[:, 0] + p[1] * brav[:, 1] + p[2] * brav[:, 2]
            lel.append(sub[t].strip() == name)
            pos.append(p)
    sysdim = int(_floats(next(it), 1)[0])
    line = next(it)
    first = line.split()[0]
    if _is_numeric(first):
        orbs = list(sys_orbs)
        fermi = _floats(line, 1)[0]
    else:
        orbs = _orbital_list(line.split()[1:])
        fermi = _floats(next(it), 1)[0]
    occ = tuple(_floats(next(it), 3))
    utoks = [t for t in next(it).split()]
    uvals = []
    for t in utoks[:2]:
        if t.startswith("!"):
            break
        uvals.append(float(t))
    Un = uvals[0]
    Um = uvals[1] if len(uvals) > 1 else uvals[0]
    lam = _floats(next(it), 2)
    if not soc:
        socscale = 0.0
    lam_p, lam_d = socscale * lam[0], socscale * lam[1]
    next(it)  # superconducting parameter (unused on this path)
    nn_stages = int(_floats(next(it), 1)[0])
    on_site = np.zeros(9)
    w = next(it).split()
    on_site[0] = float(w[2])
    w = next(it).split()
    if w[3] == "2":
        on_site[1:4] = float(w[2])
    else:
        on_site[1:4] = [float(w[j]) for j in range(2, 5)]
    w = next(it).split()
    if w[3] == "3":
        on_site[4:7] = float(w[2])
    else:
        on_site[4:7] = [float(w[j]) for j in range(2, 5)]
    w = next(it).split()
    if w[3] == "4":
        on_site[7:9] = float(w[2])
    else:
        on_site[7:9] = [float(w[j]) for j in range(2, 4)]
    norb = len(orbs)
    onsite = np.zeros((norb, norb))
    for j in range(norb):
        onsite[j, j] = on_site[orbs[j] - 1]
    hop = np.zeros((10, n_stages))
    for j in range(nn_stages):
        for k in range(10):
            w = next(it).split()
            if j >= n_stages:
                continue
            hop[k, j] = float(w[3])
    el = Element(name, a0, brav, sub, np.array(lel), np.array(pos), sysdim, orbs, fermi, occ,
                 Un, Um, lam_p, lam_d, onsite, hop)
    el.stage = _element_stages(el, n_stages, rel_tol)
    return el


def _cells(n_stages: int, sysdim: int):
    m = 2 * n_stages + 1
    ncell = m ** sysdim
    out = []
    for i in range(ncell):
        c1 = (i % m) - n_stages
        c2 = ((i // m) % m) - n_stages if sysdim >= 2 else 0
        c3 = ((i // (m * m)) % m) - n_stages if sysdim >= 3 else 0
        out.append((c1, c2, c3))
    return out


def _element_stages(el: Element, n_stages: int, rel_tol: float):
    """Stage distances of the element's own lattice (TightBinding.F90:585-650)."""
    nat = el.positions.shape[0]
    dists = [[] for _ in range(nat)]
    for c in _cells(n_stages, el.sysdim):
        cv = c[0] * el.a[:, 0] + c[1] * el.a[:, 1] + c[2] * el.a[:, 2]
        for j in range(nat):
            p = el.positions[j] + cv
            for k in range(nat):
                d = p - el.positions[k]
                dist = math.sqrt(float(np.dot(d, d)))
                if dist <= 1.0e-9:
                    continue
                dists[k].append(dist)
    stage = np.full((n_stages, nat), 1.0e12)
    for k in range(nat):
        ld = sorted(dists[k])
        stage[0, k] = ld[0]
        l = 0
        for d in ld[1:]:
            if abs(d - stage[l, k]) < stage[0, k] * rel_tol:
                continue
            l += 1
            if l >= n_stages:
                break
            stage[l, k] = d
    return stage


@dataclass
class Neighbor:
    cell: tuple
    cell_vector: np.ndarray
    basis_index: int              # 0-based atom of the unit cell this site is a copy of
    position: np.ndarray
    distance: np.ndarray          # [nAtoms] distance to each atom of cell 0
    dircos: np.ndarray            # [nAtoms, 3]
    matched: np.ndarray           # [nAtoms] stage (0-based) or -1


def generate_neighbors(basis: Basis, n_stages: int, rel_tol: float, sysdim: int):
    """Neighbour shells of every basis atom (Lattice.F90:40-233)."""
    nat = basis.positions.shape[0]
    sites = []
    for c in _cells(n_stages, sysdim):
        cv = c[0] * basis.a1 + c[1] * basis.a2 + c[2] * basis.a3
        for j in range(nat):
            p = basis.positions[j] + cv
            dist = np.zeros(nat)
            dc = np.zeros((nat, 3))
            for k in range(nat):
                d = p - basis.positions[k]
                dist[k] = math.sqrt(float(np.dot(d, d)))
                if dist[k] <= 1.0e-9:
                    continue
                dc[k] = (p - basis.positions[k]) / dist[k]
            sites.append(Neighbor(c, cv, j, p, dist, dc, np.full(nat, -1)))
    # stage distances per basis atom (self-distances excluded, as the reference
    # only inserts distances above 1e-9 into its sorted list)
    stages = np.full((n_stages, nat), 1.0e12)
    for k in range(nat):
        ld = sorted(s.distance[k] for s in sites if s.distance[k] > 1.0e-9)
        stages[0, k] = ld[0]
        l = 0
        for d in ld[1:]:
            if abs(d - stages[l, k]) < stages[0, k] * rel_tol:
                continue
            l += 1
            if l >= n_stages:
                break
            stages[l, k] = d
    out = []
    for s in sites:
        found = False
        for j in range(nat):
            for k in range(n_stages):
                if abs(s.distance[j] - stages[k, j]) < stages[0, j] * rel_tol:
                    found = True
                    s.matched[j] = k
                    break
        if found:
            out.append(s)
    return out, stages


def intd(sss, pps, ppp, dds, ddp, ddd, sps, sds, pds, pdp, w):
    """Slater-Koster two-centre table b(9,9) for direction cosines w.

    Restates TightBinding.F90:655-783 (same matrix entries; orbital order
    s, px, py, pz, dxy, dyz, dzx, dx2-y2, dz2).
    """
    x, y, z = float(w[0]), float(w[1]), float(w[2])
    xx, xy, yy, yz, zz, zx = x * x, x * y, y * y, y * z, z * z, z * x
    xxyy, yyzz, zzxx = xx * yy, yy * zz, zz * xx
    r3 = SQ3
    f1 = xx + yy
    f2 = xx - yy
    f3 = zz - .5 * f1
    f8 = 3.0 * zz - 1.0
    f4 = .5 * r3 * f2 * pds
    f5 = .5 * f8 * pds
    g1 = 1.5 * f2 * dds
    g2 = r3 * f3 * dds
    aux = pps - ppp
    aux1 = r3 * sds
    aux2 = r3 * xx * pds + (1.0 - 2.0 * xx) * pdp
    aux3 = (r3 * yy * pds + (1.0 - 2.0 * yy) * pdp)
    aux4 = r3 * zz * pds + (1.0 - 2.0 * zz) * pdp
    b = np.zeros((9, 9))
    b[0, 0] = sss
    b[0, 1] = x * sps
    b[0, 2] = y * sps
    b[0, 3] = z * sps
    b[0, 4] = xy * aux1
    b[0, 5] = yz * aux1
    b[0, 6] = zx * aux1
    b[0, 7] = .5 * f2 * aux1
    b[0, 8] = .5 * f8 * sds
    b[1, 0] = -b[0, 1]
    b[1, 1] = xx * pps + (1.0 - xx) * ppp
    b[1, 2] = xy * aux
    b[1, 3] = zx * aux
    b[1, 4] = aux2 * y
    b[1, 5] = (r3 * pds - 2.0 * pdp) * xy * z
    b[1, 6] = aux2 * z
    b[1, 7] = (f4 + (1.0 - f2) * pdp) * x
    b[1, 8] = (f5 - r3 * zz * pdp) * x
    b[2, 0] = -b[0, 2]
    b[2, 1] = b[1, 2]
    b[2, 2] = yy * pps + (1.0 - yy) * ppp
    b[2, 3] = yz * aux
    b[2, 4] = aux3 * x
    b[2, 5] = aux3 * z
    b[2, 6] = b[1, 5]
    b[2, 7] = (f4 - (1.0 + f2) * pdp) * y
    b[2, 8] = (f5 - r3 * zz * pdp) * y
    b[3, 0] = -b[0, 3]
    b[3, 1] = b[1, 3]
    b[3, 2] = b[2, 3]
    b[3, 3] = zz * pps + (1.0 - zz) * ppp
    b[3, 4] = b[1, 5]
    b[3, 5] = aux4 * y
    b[3, 6] = aux4 * x
    b[3, 7] = (f4 - f2 * pdp) * z
    b[3, 8] = (f5 + r3 * f1 * pdp) * z
    b[4, 0] = b[0, 4]
    b[4, 1] = -b[1, 4]
    b[4, 2] = -b[2, 4]
    b[4, 3] = -b[3, 4]
    b[4, 4] = 3.0 * xxyy * dds + (f1 - 4.0 * xxyy) * ddp + (zz + xxyy) * ddd
    b[4, 5] = (3.0 * yy * dds + (1.0 - 4.0 * yy) * ddp + (yy - 1.0) * ddd) * zx
    b[4, 6] = (3.0 * xx * dds + (1.0 - 4.0 * xx) * ddp + (xx - 1.0) * ddd) * yz
    b[4, 7] = (g1 - 2.0 * f2 * ddp + .5 * f2 * ddd) * xy
    b[4, 8] = (g2 - 2.0 * r3 * zz * ddp + .5 * r3 * (1.0 + zz) * ddd) * xy
    b[5, 0] = b[0, 5]
    b[5, 1] = -b[1, 5]
    b[5, 2] = -b[2, 5]
    b[5, 3] = -b[3, 5]
    b[5, 4] = b[4, 5]
    b[5, 5] = 3.0 * yyzz * dds + (yy + zz - 4.0 * yyzz) * ddp + (xx + yyzz) * ddd
    b[5, 6] = (3.0 * zz * dds + (1.0 - 4.0 * zz) * ddp + (zz - 1.0) * ddd) * xy
    b[5, 7] = (g1 - (1.0 + 2.0 * f2) * ddp + (1.0 + .5 * f2) * ddd) * yz
    b[5, 8] = (g2 + r3 * (f1 - zz) * ddp - .5 * r3 * f1 * ddd) * yz
    b[6, 0] = b[0, 6]
    b[6, 1] = -b[1, 6]
    b[6, 2] = -b[2, 6]
    b[6, 3] = -b[3, 6]
    b[6, 4] = b[4, 6]
    b[6, 5] = b[5, 6]
    b[6, 6] = 3.0 * zzxx * dds + (zz + xx - 4.0 * zzxx) * ddp + (yy + zzxx) * ddd
    b[6, 7] = (g1 + (1.0 - 2.0 * f2) * ddp - (1.0 - .5 * f2) * ddd) * zx
    b[6, 8] = (g2 + r3 * (f1 - zz) * ddp - .5 * r3 * f1 * ddd) * zx
    b[7, 0] = b[0, 7]
    b[7, 1] = -b[1, 7]
    b[7, 2] = -b[2, 7]
    b[7, 3] = -b[3, 7]
    b[7, 4] = b[4, 7]
    b[7, 5] = b[5, 7]
    b[7, 6] = b[6, 7]
    b[7, 7] = .75 * f2 * f2 * dds + (f1 - f2 * f2) * ddp + (zz + .25 * f2 * f2) * ddd
    b[7, 8] = .5 * f2 * g2 - r3 * zz * f2 * ddp + .25 * r3 * (1.0 + zz) * f2 * ddd
    b[8, 0] = b[0, 8]
    b[8, 1] = -b[1, 8]
    b[8, 2] = -b[2, 8]
    b[8, 3] = -b[3, 8]
    b[8, 4] = b[4, 8]
    b[8, 5] = b[5, 8]
    b[8, 6] = b[6, 8]
    b[8, 7] = b[7, 8]
    b[8, 8] = f3 * f3 * dds + 3.0 * zz * f1 * ddp + .75 * f1 * f1 * ddd
    return b


# Andersen scaling exponents of the 10 two-centre integrals (TightBinding.F90:104)
EXPON = [1.0, 3.0, 3.0, 5.0, 5.0, 5.0, 2.0, 3.0, 4.0, 4.0]


def _sign(a, b):
    return abs(a) if b >= 0.0 else -abs(a)


def sk_hoppings(neighbors, stages, atom_type, elements, n_stages: int, simple_mix: bool = False):
    """Hopping blocks t0i(nOrb_j, nOrb_i) per (neighbour, site i) (TightBinding.F90:93-219).

    Returns ``{(neighbor_index, i): t0i}`` for every neighbour within the
    shells of atom i; t0i rows run over the neighbour's orbitals (atom j =
    basis_index) and columns over atom i's orbitals.
    """
    nat = len(atom_type)
    # The reference iterates Basis(i)%NeighborList(k,j) linked lists; the set of
    # (neighbour, i) pairs is exactly those with matched[i] >= 0.
    t = {}
    for nidx, nb in enumerate(neighbors):
        for i in range(nat):
            k = int(nb.matched[i])
            if k < 0:
                continue
            j = nb.basis_index
            ei = elements[atom_type[i]]
            ej = elements[atom_type[j]]
            sf = [0.0, 0.0]
            for l in range(ei.stage.shape[1]):
                if not ei.lelement[l]:
                    continue
                temp = ei.stage[k, l] / nb.distance[i]
                if abs(temp - 1.0) < abs(sf[0] - 1.0):
                    sf[0] = temp
            for l in range(ej.stage.shape[1]):
                if not ej.lelement[l]:
                    continue
                temp = ej.stage[k, l] / nb.distance[i]
                if abs(temp - 1.0) < abs(sf[1] - 1.0):
                    sf[1] = temp
            mix1 = [ei.hopping[l, k] * sf[0] ** EXPON[l] for l in range(10)]
            mix2 = [ej.hopping[l, k] * sf[1] ** EXPON[l] for l in range(10)]
            if simple_mix:
                mix = [0.5 * (mix1[l] + mix2[l]) for l in range(10)]
            else:
                mix = [_sign(math.sqrt(abs(mix1[l]) * abs(mix2[l])), mix1[l] + mix2[l]) for l in range(10)]
            # argument order of intd at TightBinding.F90:210
            bp = intd(mix[0], mix[1], mix[2], mix[3], mix[4], mix[5], mix[6], mix[7], mix[8], mix[9],
                      nb.dircos[i])
            oi = ei.orbs
            oj = ej.orbs
            blk = np.zeros((len(oj), len(oi)))
            for a in range(len(oi)):
                for b in range(len(oj)):
                    blk[b, a] = bp[oj[b] - 1, oi[a] - 1]
            t[(nidx, i)] = blk
    return t
