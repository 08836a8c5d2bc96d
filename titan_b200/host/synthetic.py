"""Seeded synthetic Slater-Koster models of the benchmark shapes.

Every workload is a seeded tight-binding model (no external data): two-centre
integrals (sss, pps, ppp, dds, ddp, ddd, sps, sds, pds, pdp -- the element-file
order of TightBinding.F90:559-568) uniform in [-1.5, 0.5] eV for the first
shell and 0.3x that for the second, on-site s, p, d uniform in [-2, 4] eV,
lambda_p = lambda_d = 0.06 eV, U = 1 eV on d (Un = Um), initial moment 2 muB
along z spread over the d orbitals.  Draw order per model: on-site (s, p, d),
then shell 1 (10 values), then shell 2 (10 values), all from
``numpy.random.default_rng(seed)``.

Shapes (n = dimH):

=========  =====================================  ===  ======================
name       lattice                                 n    default mesh
=========  =====================================  ===  ======================
bcc1       bcc bulk, 1 atom                        18   24^3 k, 64 imag
sq2        2D square monolayer, 2 atoms/cell       36   200^2 k, 128 imag + 64 real, 32 omega
slab5      bcc(001) slab, 5 layers                 90   adaptive 400^2 -> 16^2
bcc4       bcc bulk, 4 atoms/cell                  72   48^3 k, 96 imag
slab16     bcc(001) slab, 16 layers                288  128^2 k, 128 imag + 96 real, 64 omega
slabL      bcc(001) slab, L layers (any L >= 1)    18L  as slab5, uniform 32^2 k (test systems)
=========  =====================================  ===  ======================
"""
from __future__ import annotations

import math

import numpy as np

from . import lattice as L
from .deck import Deck
from .system import TBSystem

SHAPES = {
    # a1, a2, a3 (units of a0), positions (Cartesian, units of a0), sysdim, seed
    "bcc1": (np.array([[0.5, 0.5, -0.5], [0.5, -0.5, 0.5], [-0.5, 0.5, 0.5]]), np.zeros((1, 3)), 3, 1001),
    "sq2": (np.array([[1.0, 1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 0.0, 0.0]]),
            np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]]), 2, 1002),
    "slab5": (np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 0.0]]),
              np.array([[0.5 * (l % 2), 0.5 * (l % 2), 0.5 * l] for l in range(5)]), 2, 1003),
    "bcc4": (np.array([[2.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]),
             np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5], [1.0, 0.0, 0.0], [1.5, 0.5, 0.5]]), 3, 1004),
    "slab16": (np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 0.0]]),
               np.array([[0.5 * (l % 2), 0.5 * (l % 2), 0.5 * l] for l in range(16)]), 2, 1005),
}

A0 = 5.30   # lattice constant (bohr), the bcc Fe value of the reference example


def _shape(shape: str):
    """SHAPES entry; "slabL" for any other layer count L is the bcc(001) slab of L layers
    (seed 2000 + L)."""
    if shape in SHAPES:
        return SHAPES[shape]
    if shape.startswith("slab") and shape[4:].isdigit() and int(shape[4:]) >= 1:
        nl = int(shape[4:])
        return (np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 0.0]]),
                np.array([[0.5 * (l % 2), 0.5 * (l % 2), 0.5 * l] for l in range(nl)]), 2, 2000 + nl)
    raise KeyError(shape)


def _mesh_cfg(shape: str):
    if shape in DEFAULT_MESH:
        return DEFAULT_MESH[shape]
    return dict(nk=(32, 32, 1), parts=2, n1gl=32, parts3=1, n3gl=32, omegas=(0.0, 0.3, 4))


def draw_parameters(seed: int):
    rng = np.random.default_rng(seed)
    onsite = rng.uniform(-2.0, 4.0, size=3)
    shell1 = rng.uniform(-1.5, 0.5, size=10)
    shell2 = 0.3 * rng.uniform(-1.5, 0.5, size=10)
    return onsite, shell1, shell2


def make_element(name: str, a_cols: np.ndarray, positions: np.ndarray, sysdim: int, seed: int,
                 n_stages: int = 2, rel_tol: float = 0.05, orbs=None, U: float = 1.0,
                 lam: float = 0.06) -> L.Element:
    onsite, s1, s2 = draw_parameters(seed)
    orbs = list(range(1, 10)) if orbs is None else list(orbs)
    on9 = np.array([onsite[0]] + [onsite[1]] * 3 + [onsite[2]] * 5)
    norb = len(orbs)
    ons = np.zeros((norb, norb))
    for j in range(norb):
        ons[j, j] = on9[orbs[j] - 1]
    hop = np.zeros((10, n_stages))
    hop[:, 0] = s1
    if n_stages > 1:
        hop[:, 1] = s2
    fermi = float(onsite[2])   # centre of the d band
    el = L.Element(name, A0, a_cols * A0, [name], np.ones(positions.shape[0], bool), positions * A0,
                   sysdim, orbs, fermi, (1.0, 1.0, 6.0), U, U, lam, lam, ons, hop)
    el.stage = L._element_stages(el, n_stages, rel_tol)
    return el


def make_system(shape: str, seed: int | None = None, n_stages: int = 2, eta: float = 1.0e-3) -> TBSystem:
    a, pos, sysdim, default_seed = _shape(shape)
    seed = default_seed if seed is None else seed
    a1, a2, a3 = a[0] * A0, a[1] * A0, a[2] * A0
    basis = L.Basis(shape, A0, a1, a2, a3, [shape], [0] * pos.shape[0], pos * A0, sysdim)
    el = make_element(shape, np.stack([a1, a2, a3], axis=1) / A0, pos, sysdim, seed, n_stages)
    neighbors, _ = L.generate_neighbors(basis, n_stages, 0.05, sysdim)
    t0i = L.sk_hoppings(neighbors, None, basis.atom_type, [el], n_stages)
    return TBSystem(shape, sysdim, a1, a2, a3, list(basis.atom_type), [el], neighbors, t0i, el.fermi, eta, eta)


DEFAULT_MESH = {
    "bcc1": dict(nk=(24, 24, 24), parts=1, n1gl=64, parts3=1, n3gl=64, omegas=(0.0, 0.0, 1)),
    "sq2": dict(nk=(200, 200, 1), parts=2, n1gl=64, parts3=1, n3gl=64, omegas=(0.0, 0.5, 32)),
    "slab5": dict(nk=(400, 400, 1), parts=2, n1gl=64, parts3=1, n3gl=64, omegas=(0.0, 0.3, 16),
                  adaptive=(400 * 400, 16 * 16)),
    "bcc4": dict(nk=(48, 48, 48), parts=1, n1gl=96, parts3=1, n3gl=64, omegas=(0.0, 0.0, 1)),
    "slab16": dict(nk=(128, 128, 1), parts=2, n1gl=64, parts3=1, n3gl=96, omegas=(0.0, 0.3, 64)),
}


def make_deck(shape: str, seed: int | None = None, nk=None, parts=None, n1gl=None, parts3=None, n3gl=None,
              mesh: bool = True) -> Deck:
    """System + meshes; keyword overrides shrink the mesh for tests."""
    cfg = dict(_mesh_cfg(shape))
    sysm = make_system(shape, seed)
    nk = tuple(nk) if nk is not None else cfg["nk"]
    sd = sysm.sysdim
    kp = [1, 1, 1]
    kp[:sd] = nk[:sd]
    total = int(np.prod(kp[:sd]))
    p = dict(kp_in=tuple(kp), kptotal=total, minimumBZmesh=total,
             parts=parts or cfg["parts"], n1gl=n1gl or cfg["n1gl"],
             parts3=parts3 or cfg["parts3"], n3gl=n3gl or cfg["n3gl"])
    lo, hi, nw = cfg["omegas"]
    p["emin"], p["emax"], p["nEner"] = lo, hi, max(nw - 1, 0)
    if "adaptive" in cfg and nk == cfg["nk"]:
        from . import mesh as M
        y, _ = M.imag_energy_points(p["parts"], p["n1gl"])
        hi_n, lo_n = cfg["adaptive"]
        # log-uniform decay of the k count from the real axis (small y) outwards
        t = np.linspace(0.0, 1.0, len(y))
        p["nk_per_energy"] = np.rint(np.exp(math.log(hi_n) * (1 - t) + math.log(lo_n) * t)).astype(int)
    return Deck.from_system(sysm, p, mesh)
