"""On-site potential / exchange-field perturbation and site observables.

The perturbation h0 -> h0 + sum_i P_i (V_i sigma_0 + B_i . sigma) acts on every
orbital of site i, in the reference's site-block layout [up orbitals | down
orbitals] (mod_System.F90:117-129).  The observables x_i = (n, mx, my, mz) of a
site are the orbital sums of expectation_values_greenfunction's outputs
(mod_expectation.F90:28-149).
"""
from __future__ import annotations

import numpy as np

PAULI = (np.eye(2, dtype=complex), np.array([[0, 1], [1, 0]], complex), np.array([[0, -1j], [1j, 0]]),
         np.diag([1.0 + 0j, -1.0]))


def vb_perturbation(system, V, B):
    """dimH x dimH complex matrix sum_i P_i (V_i sigma_0 + B_i . sigma)."""
    V = np.asarray(V, float)
    B = np.asarray(B, float).reshape(system.n_atoms, 3)
    n = system.dimH
    ia = system.ia()
    dh = np.zeros((n, n), complex)
    for i in range(system.n_atoms):
        ni = system.norbs[i]
        b = ia[i][0]
        M = V[i] * PAULI[0] + B[i, 0] * PAULI[1] + B[i, 1] * PAULI[2] + B[i, 2] * PAULI[3]
        o = np.arange(ni)
        for s in range(2):
            for t in range(2):
                dh[b + s * ni + o, b + t * ni + o] += M[s, t]
    return dh


def site_observables(system, rho, mx, my, mz):
    """x[i] = (n_i, mx_i, my_i, mz_i) summed over the orbitals of site i."""
    x = np.zeros((system.n_atoms, 4))
    for i in range(system.n_atoms):
        o = slice(0, system.norbs[i])
        x[i] = (rho[i, o].sum(), mx[i, o].sum(), my[i, o].sum(), mz[i, o].sum())
    return x
