"""An input deck: system + integration meshes, as the reference sets them up.

``Deck.from_directory`` reads a reference-format example directory (input,
basis, element files) and builds everything the hot path consumes, in the
order of main.F90:94-180: lattice and neighbours, SK hoppings, energy points
(EnergyIntegration.F90:45-97), the real-axis BZ (realBZ, main.F90:160-164)
and the adaptive imaginary-axis (E, k) mesh (adaptiveMesh.F90:23-161).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from . import lattice as L
from . import mesh as M
from .system import (TBSystem, build_system, electric_field_vector, params_from_input, read_initial_rho, read_input,
                     set_reference_densities)


@dataclass
class Deck:
    system: TBSystem
    params: dict
    y: np.ndarray
    wght: np.ndarray
    ek: M.EKMesh
    real_kp: np.ndarray
    real_w: np.ndarray

    @classmethod
    def from_directory(cls, d: str, mesh: bool = True) -> "Deck":
        inp = read_input(os.path.join(d, "input"))
        p = params_from_input(inp)
        basis = L.read_basis(os.path.join(d, "basis"))
        elements = {nm: os.path.join(d, nm) for nm in basis.type_names}
        sysm = build_system(basis, elements, p)
        p["efield"] = electric_field_vector(inp, sysm.a1, sysm.a2, sysm.a3)
        # reference densities of elements with Un != 0 (the bulk run's initialrho_<element> file)
        init = {t: os.path.join(d, f"initialrho_{nm}.dat") for t, nm in enumerate(basis.type_names)}
        init = {t: f for t, f in init.items() if os.path.exists(f)}
        if init:
            set_reference_densities(sysm, {t: read_initial_rho(f, len(sysm.elements[t].orbs)) for t, f in init.items()})
        return cls.from_system(sysm, p, mesh)

    @classmethod
    def from_system(cls, sysm: TBSystem, p: dict, mesh: bool = True) -> "Deck":
        y, wght = M.imag_energy_points(p["parts"], p["n1gl"])
        if mesh:
            ek = M.adaptive_ek_mesh(sysm.a1, sysm.a2, sysm.a3, sysm.sysdim, y, wght, p["kptotal"],
                                    p["minimumBZmesh"], p.get("nk_per_energy"))
            rk, rw = M.bz_fraction(sysm.a1, sysm.a2, sysm.a3, sysm.sysdim, p["kp_in"])
        else:
            ek = None
            rk = rw = None
        return cls(sysm, p, y, wght, ek, rk, rw)

    def frequencies(self):
        """e = emin + deltae*(kount-1), kount = 1..nEner+1 (calculate_chi.F90:66-67, setLoops)."""
        n = self.params["nEner"]
        emin, emax = self.params["emin"], self.params["emax"]
        if n <= 0:
            return np.array([emin])
        de = (emax - emin) / n
        return np.array([emin + de * k for k in range(n + 1)])

    def real_points(self, e: float, Ef: float):
        return M.real_energy_points(Ef, e, self.params["parts3"], self.params["n3gl"])
