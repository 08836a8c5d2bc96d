"""Tight-binding system description: the inputs of the Green-function hot path.

A ``TBSystem`` holds what the reference keeps in ``System_type`` plus the
module state the hot path reads (mod_System.F90:22-73, mod_parameters):
lattice, neighbour table with hopping blocks, on-site/SOC/Zeeman/Hubbard
ingredients of h0, Fermi level and the broadening eta.  ``neighbor_table``
flattens it into the arrays the C ABI takes; ``h0`` assembles the local
Hamiltonian for a magnetic state (mod_hamiltonian.F90:35-63 with the Hubbard
term of mod_U_matrix.F90:29-55).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import lattice as L
from . import mesh as M
from . import onsite as O


def read_input(path: str) -> dict:
    """Parse '-> key = value' lines of a reference input file (mod_input.F90:66-120)."""
    out = {}
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s.startswith("->"):
                continue
            s = s[2:]
            if "=" not in s:
                continue
            k, v = s.split("=", 1)
            v = v.split("!")[0].strip()
            out[k.strip()] = v
    return out


def _fnum(v: str) -> float:
    return float(v.replace("d", "e").replace("D", "e"))


@dataclass
class MagState:
    """Occupations and moments per (orbital, site): the self-consistent variables."""
    rho: np.ndarray   # [nAtoms, nOrb]
    mx: np.ndarray
    my: np.ndarray
    mz: np.ndarray
    Ef: float

    def d_totals(self, dorbs):
        """rhod, mxd, myd, mzd per site (mod_self_consistency.F90:375-384)."""
        nat = self.rho.shape[0]
        rd = np.array([sum(self.rho[i, m] for m in dorbs[i]) for i in range(nat)])
        xd = np.array([sum(self.mx[i, m] for m in dorbs[i]) for i in range(nat)])
        yd = np.array([sum(self.my[i, m] for m in dorbs[i]) for i in range(nat)])
        zd = np.array([sum(self.mz[i, m] for m in dorbs[i]) for i in range(nat)])
        return rd, xd, yd, zd


@dataclass
class TBSystem:
    name: str
    sysdim: int
    a1: np.ndarray
    a2: np.ndarray
    a3: np.ndarray
    atom_type: list
    elements: list                 # per type
    neighbors: list                # lattice.Neighbor
    t0i: dict                      # (neighbor_index, i) -> [nOrb_j, nOrb_i]
    Ef: float
    eta: float
    etap: float
    rho0: np.ndarray = field(default=None)   # [nAtoms, nOrb] reference occupations (Hubbard)
    rhod0: np.ndarray = field(default=None)
    mzd0: np.ndarray = field(default=None)
    mpd0: np.ndarray = field(default=None)
    hhw: np.ndarray = field(default=None)    # [nAtoms, 3] half external field (0 by default)

    # ---- sizes and index maps -------------------------------------------
    @property
    def n_atoms(self) -> int:
        return len(self.atom_type)

    @property
    def norbs(self):
        return [len(self.elements[t].orbs) for t in self.atom_type]

    @property
    def orbs(self):
        return [self.elements[t].orbs for t in self.atom_type]

    @property
    def dorbs(self):
        """Local indices of the d orbitals per site (Types%dOrbs)."""
        return [[a for a, o in enumerate(self.elements[t].orbs) if 5 <= o <= 9] for t in self.atom_type]

    @property
    def dimH(self) -> int:
        return 2 * sum(self.norbs)

    @property
    def dimens(self) -> int:
        return 4 * sum(n * n for n in self.norbs)

    def ia(self):
        return O.site_offsets(self.norbs)

    def sigmaimunu2i(self):
        """0-based chi row index map [4, nAtoms, nOrb, nOrb] (mod_System.F90:176-187)."""
        nmax = max(self.norbs)
        idx = np.full((4, self.n_atoms, nmax, nmax), -1, dtype=np.int64)
        k = 0
        for i, n in enumerate(self.norbs):
            for mu in range(n):
                for nu in range(n):
                    for s in range(4):
                        idx[s, i, mu, nu] = k
                        k += 1
        return idx

    # ---- Hamiltonian ingredients -------------------------------------------
    def neighbor_table(self):
        """Flattened hopping table for the C ABI and the oracle.

        Returns (cell_vec[nNeigh,3], basis_idx[nNeigh] (0-based), is_hopping
        [nNeigh, nAtoms] int32, t0i [nNeigh, nAtoms, nOrbMax, nOrbMax]
        complex128 with t0i[k, i, b, a] = t0i(b, a, i) of neighbour k).
        """
        nn = len(self.neighbors)
        nat = self.n_atoms
        nmax = max(self.norbs)
        cv = np.array([nb.cell_vector for nb in self.neighbors], float).reshape(nn, 3)
        bi = np.array([nb.basis_index for nb in self.neighbors], np.int32)
        ish = np.zeros((nn, nat), np.int32)
        t = np.zeros((nn, nat, nmax, nmax), complex)
        for (k, i), blk in self.t0i.items():
            ish[k, i] = 1
            t[k, i, :blk.shape[0], :blk.shape[1]] = blk
        return cv, bi, ish, t

    def local_blocks(self, state: MagState, soc_theta: float = 0.0, soc_phi: float = 0.0):
        """Per-site ls + sb + lb + hee (2nOrb x 2nOrb) for a magnetic state."""
        rd, xd, yd, zd = state.d_totals(self.dorbs)
        blocks = []
        for i, t in enumerate(self.atom_type):
            el = self.elements[t]
            n = len(el.orbs)
            blk = O.ls_matrix(el.orbs, el.lambda_p, el.lambda_d, soc_theta, soc_phi)
            hhw = np.zeros(3) if self.hhw is None else self.hhw[i]
            if np.any(hhw != 0):
                blk = blk + O.sb_matrix(n, hhw) + O.lb_matrix(el.orbs, hhw)
            rho0 = np.zeros(n) if self.rho0 is None else self.rho0[i]
            rhod0 = 0.0 if self.rhod0 is None else self.rhod0[i]
            mzd0 = 0.0 if self.mzd0 is None else self.mzd0[i]
            mpd0 = 0j if self.mpd0 is None else self.mpd0[i]
            blk = blk + O.hee_matrix(el.orbs, el.Un, el.Um, state.rho[i], rho0, rd[i], rhod0,
                                     zd[i], mzd0, complex(xd[i], yd[i]), mpd0)
            blocks.append(blk)
        return blocks

    def h0(self, state: MagState):
        """Local Hamiltonian h0 (dimH x dimH complex) for a magnetic state."""
        onsite = [self.elements[t].onsite.astype(complex) for t in self.atom_type]
        return O.assemble_h0(self.norbs, onsite, self.local_blocks(state))

    def linear_soc_split(self, state: MagState, soc_theta: float = 0.0, soc_phi: float = 0.0):
        """(h0 without the local SOC, V = the SOC blocks) with h0(state) = h0_0 + V, the split of
        hamiltklinearsoc (mod_hamiltonian.F90:304-396) for the linear-SOC susceptibility."""
        h0 = self.h0(state)
        V = np.zeros_like(h0)
        ia = O.site_offsets(self.norbs)
        for i, t in enumerate(self.atom_type):
            el = self.elements[t]
            b0, b3 = ia[i][0], ia[i][3]
            V[b0:b3, b0:b3] = O.ls_matrix(el.orbs, el.lambda_p, el.lambda_d, soc_theta, soc_phi)
        return h0 - V, V

    def Un(self):
        return np.array([self.elements[t].Un for t in self.atom_type])

    def Um(self):
        return np.array([self.elements[t].Um for t in self.atom_type])

    def total_occupation(self) -> float:
        return float(sum(sum(self.elements[t].occ) for t in self.atom_type))

    def reciprocal(self):
        return M.reciprocal_vectors(self.a1, self.a2, self.a3, self.sysdim)


def build_system(basis: L.Basis, element_paths: dict, params: dict) -> TBSystem:
    """Lattice + SK hoppings for a basis and element files (main.F90:94-141).

    ``params`` keys: sysdim, nn_stages, relTol, SOC, socscale, orbitals,
    fermi_layer, eta, etap, Ef (optional override).
    """
    sysdim = int(params.get("sysdim", 3))
    nst = int(params.get("nn_stages", 2))
    rel = float(params.get("relTol", 0.05))
    soc = params.get("SOC", True)
    socscale = float(params.get("socscale", 1.0))
    sys_orbs = params.get("orbitals", list(range(1, 10)))
    elements = []
    for nm in basis.type_names:
        elements.append(L.read_element(element_paths[nm], nm, nst, rel, sys_orbs, soc, socscale))
    neighbors, _ = L.generate_neighbors(basis, nst, rel, sysdim)
    t0i = L.sk_hoppings(neighbors, None, basis.atom_type, elements, nst,
                        simple_mix=bool(params.get("simplemix", False)))
    # common Fermi level (TightBinding.F90:111-116)
    fl = int(params.get("fermi_layer", 1)) - 1
    Ef = elements[fl].fermi
    for el in elements:
        for j in range(len(el.orbs)):
            el.onsite[j, j] = el.onsite[j, j] - el.fermi + Ef
    if "Ef" in params and params["Ef"] is not None:
        Ef = float(params["Ef"])
    eta = float(params.get("eta", 1e-3))
    etap = float(params.get("etap", eta))
    return TBSystem(basis.name, sysdim, basis.a1, basis.a2, basis.a3, list(basis.atom_type), elements,
                    neighbors, t0i, Ef, eta, etap)


def electric_field_vector(inp: dict, a1, a2, a3) -> np.ndarray:
    """ElectricFieldVector of a deck, unit length (mod_io.F90:296-325,
    ElectricField.F90:16-54): ebasis cartesian (3 components), bravais (2 integer
    coefficients of a1, a2) or spherical (theta, phi in degrees, the default)."""
    basis = inp.get("ebasis", "spherical").strip().lower()
    v = [_fnum(x) for x in inp.get("dirEfield", "90 0").split()]
    if basis == "cartesian":
        e = np.array(v[:3], float)
    elif basis == "bravais":
        e = v[0] * np.asarray(a1, float) + v[1] * np.asarray(a2, float)
    elif basis == "spherical":
        t, ph = math.radians(v[0]), math.radians(v[1])
        e = np.array([math.cos(ph) * math.sin(t), math.sin(ph) * math.sin(t), math.cos(t)])
    else:
        raise ValueError(f"ebasis = {basis}: field along atom directions is not implemented (as in the reference)")
    return e / np.linalg.norm(e)


def params_from_input(inp: dict) -> dict:
    """Translate a parsed reference input deck into build/mesh parameters (mod_io.F90:85-140)."""
    p = {}
    p["sysdim"] = int(inp.get("sysdim", "3"))
    p["nn_stages"] = int(inp.get("nn_stages", "2"))
    p["relTol"] = _fnum(inp.get("relTol", "0.05"))
    p["SOC"] = inp.get("SOC", "F").strip().upper().startswith("T")
    p["socscale"] = _fnum(inp.get("socscale", "1.0"))
    if "orbitals" in inp:
        p["orbitals"] = L._orbital_list(inp["orbitals"].split())
    p["fermi_layer"] = int(inp.get("fermi_layer", "1"))
    p["eta"] = _fnum(inp["eta"])
    p["etap"] = _fnum(inp.get("etap", inp["eta"]))
    if "Ef" in inp:
        p["Ef"] = _fnum(inp["Ef"])
    nk = [int(x) for x in inp["nkpt"].split()]
    sd = p["sysdim"]
    if len(nk) == sd:
        kp = [1, 1, 1]
        kp[:sd] = nk
        total = int(np.prod(kp[:sd]))
    else:
        total = nk[0]
        if sd == 3:
            n = int(math.ceil(float(total) ** 0.333333333333333))
            kp = [n, n, n]
            total = n ** 3
        elif sd == 2:
            n = int(math.ceil(float(total) ** 0.5))
            kp = [n, n, 1]
            total = n * n
        else:
            kp = [total, 1, 1]
    p["kp_in"] = tuple(kp)
    p["kptotal"] = total
    mb = int(inp.get("minimumBZmesh", "1000"))
    p["minimumBZmesh"] = min(mb, total)
    p["parts"] = int(inp.get("parts", "1"))
    p["n1gl"] = int(inp.get("n1gl", "64"))
    p["parts3"] = int(inp.get("parts3", "1"))
    p["n3gl"] = int(inp.get("n3gl", "64"))
    p["emin"] = _fnum(inp.get("emin", "0"))
    p["emax"] = _fnum(inp.get("emax", "0"))
    p["nEner"] = int(inp.get("nEner", "0"))
    p["options"] = inp.get("Options", "").split()
    return p


def read_initial_rho(path: str, norb: int):
    """Reference densities of an element with Un != 0: rho0(nOrb), then rhod0, mpd0 (re, im), mzd0,
    then Un, Um (the initialrho file of read_init_expecs, mod_initial_expectation.F90:473-534)."""
    with open(path) as f:
        vals = [float(x) for x in f.read().split()]
    rho0 = np.array(vals[:norb])
    rhod0, mpr, mpi, mzd0 = vals[norb:norb + 4]
    return {"rho0": rho0, "rhod0": rhod0, "mpd0": complex(mpr, mpi), "mzd0": mzd0,
            "Un": vals[norb + 4], "Um": vals[norb + 5]}


def set_reference_densities(system: "TBSystem", per_element: dict):
    """Per-site rho0 / rhod0 / mzd0 / mpd0 of the Hubbard term (mod_initial_expectation.F90:216-230) from
    reference densities keyed by element (type index); elements without an entry keep zero (the
    reference's Un = 0 case)."""
    nat, nmax = system.n_atoms, max(system.norbs)
    rho0 = np.zeros((nat, nmax))
    rhod0, mzd0 = np.zeros(nat), np.zeros(nat)
    mpd0 = np.zeros(nat, complex)
    for i, t in enumerate(system.atom_type):
        r = per_element.get(t)
        if r is None:
            continue
        rho0[i, :len(r["rho0"])] = r["rho0"]
        rhod0[i], mzd0[i], mpd0[i] = r["rhod0"], r["mzd0"], r["mpd0"]
    system.rho0, system.rhod0, system.mzd0, system.mpd0 = rho0, rhod0, mzd0, mpd0


def read_sc_file(path: str, norbs):
    """Self-consistency results file: n, mx, my, mz, delta per site, then Ef (mod_self_consistency.F90:341-389)."""
    vals = []
    with open(path) as f:
        lines = [l for l in f if l.strip() and not l.lstrip().startswith("!")]
    nat = len(norbs)
    rows = []
    for i in range(nat):
        rows.append([float(x) for x in lines[i].split()[:5 * norbs[i]]])
    Ef = float(lines[nat].split()[0])
    nmax = max(norbs)
    rho = np.zeros((nat, nmax))
    mx = np.zeros((nat, nmax))
    my = np.zeros((nat, nmax))
    mz = np.zeros((nat, nmax))
    for i, r in enumerate(rows):
        n = norbs[i]
        rho[i, :n] = r[0:n]
        mx[i, :n] = r[n:2 * n]
        my[i, :n] = r[2 * n:3 * n]
        mz[i, :n] = r[3 * n:4 * n]
    del vals
    return MagState(rho, mx, my, mz, Ef)


def initial_state(system: TBSystem, moment=(0.0, 0.0, 2.0)) -> MagState:
    """Starting magnetic state when no previous results exist (mod_self_consistency.F90:148-191).

    rho = rho0 and the moment is spread evenly over the d orbitals.
    """
    nat = system.n_atoms
    nmax = max(system.norbs)
    rho = np.zeros((nat, nmax)) if system.rho0 is None else system.rho0.copy()
    mx = np.zeros((nat, nmax))
    my = np.zeros((nat, nmax))
    mz = np.zeros((nat, nmax))
    for i, d in enumerate(system.dorbs):
        for m in d:
            mx[i, m] = moment[0] / len(d)
            my[i, m] = moment[1] / len(d)
            mz[i, m] = moment[2] / len(d)
    return MagState(rho, mx, my, mz, system.Ef)


def example_paths(root: str, name: str):
    d = os.path.join(root, name)
    return os.path.join(d, "input"), os.path.join(d, "basis"), d
