"""Linear response to an electric field from the disturbance integral.

Host part of calculate_all (source/calculate_all.F90:117-420) around the GPU
energy integral tg_she (eintshe):

* ``prefactor``: (1 + chi_HF U)^-1 (calculate_all.F90:117-120);
* ``lp_matrix``: the orbital angular momentum in the local spin frame of each
  site (mod_magnet.F90:359-378);
* ``responses``: charge, spin and orbital disturbances, spin-orbit,
  exchange-correlation and external torques and the effective field
  (calculate_all.F90:279-420) from tchiorbiikl and the RPA susceptibility.

All of it is O(dimens^2) dense algebra on matrices that fit in cache and runs
once per frequency, after the (k, E) sums on the GPU.  Arrays use the numpy
[row, col] convention with rows in sigmaimunu2i order (spin channel fastest).
"""
from __future__ import annotations

import numpy as np

from .onsite import l_matrices


def prefactor(chi_hf, U):
    """(1 + chi_HF U)^-1, the renormalisation applied to the disturbance integral."""
    D = chi_hf.shape[0]
    return np.linalg.inv(np.eye(D, dtype=complex) + chi_hf @ U)


def type_lvec(orbs):
    """L_x, L_y, L_z restricted to a type's orbitals (1-based orbital codes), [3, n, n]."""
    idx = np.asarray(orbs, int) - 1
    return l_matrices()[:, idx][:, :, idx]


def lp_matrix(lvec, theta_deg, phi_deg):
    """L in the frame of a moment at polar angle theta and azimuth phi (degrees)."""
    t, p = np.deg2rad(theta_deg), np.deg2rad(phi_deg)
    ct, st, cp, sp = np.cos(t), np.sin(t), np.cos(p), np.sin(p)
    lx, ly, lz = lvec
    return np.stack([lx * ct * cp + ly * ct * sp - lz * st,
                     -lx * sp + ly * cp,
                     lx * st * cp + ly * st * sp + lz * ct])


def _site_rows(system):
    """idx[i] = sigmaimunu2i rows of site i as an array [4, n_i, n_i] (sigma, mu, nu)."""
    sidx = system.sigmaimunu2i()
    return [sidx[:, i, :n, :n] for i, n in enumerate(system.norbs)]


def site_reduced(system, chi):
    """sum over the diagonal orbitals mu = mu', nu = nu' of each site pair: [4 n_atoms, 4 n_atoms],
    index sigma * n_atoms + site (calculate_all.F90:266-277)."""
    nat = system.n_atoms
    R = np.zeros((4 * nat, system.dimens))
    for i, rows in enumerate(_site_rows(system)):
        for s in range(4):
            R[s * nat + i, np.diagonal(rows[s])] = 1.0
    return R @ chi @ R.T


def responses(system, tchi, chiorb, lvec, lpvec, lambda_p, lambda_d, porbs, dorbs, Um, mvec=None, hhw=None):
    """Disturbances (7, n_atoms), torques (3, 3, n_atoms) and Beff_cart (4, n_atoms) with their site sums.

    tchi: tchiorbiikl [dimens, 4]; chiorb: RPA susceptibility (prefactor chi_HF) [dimens, dimens];
    lvec / lpvec: per site [3, n, n] in the global / local frame; lambda_p, lambda_d, porbs, dorbs,
    Um: per site; mvec: per site cartesian moments (None: zero); hhw: per site field (None: no field).
    """
    nat = system.n_atoms
    # A[s][mu, nu] = tchi(sigmaimunu2i(s, i, mu, nu), 2) + tchi(..., 3)  (sigma' = 2, 3 in 1-based order)
    A = [tchi[rows][..., 1] + tchi[rows][..., 2] for rows in _site_rows(system)]
    dist = np.zeros((7, nat), complex)
    torq = np.zeros((3, 3, nat), complex)
    for i in range(nat):
        a = A[i]
        charge, sz2 = a[1] + a[2], a[1] - a[2]
        plus, minus = a[0] + a[3], a[0] - a[3]
        dist[0, i] = np.trace(charge)
        dist[1, i] = np.trace(plus)
        dist[2, i] = np.trace(minus) / 1j
        dist[3, i] = np.trace(sz2)
        dist[4:7, i] = np.einsum("cmn,mn->c", lvec[i], charge)
        for lam, orbl in ((lambda_p[i], porbs[i]), (lambda_d[i], dorbs[i])):
            if not len(orbl):
                continue
            o = np.ix_(orbl, orbl)
            lp = lpvec[i][:, o[0], o[1]]
            sa, sb, sc = (sz2[o] * lp[1]).sum(), (minus[o] * lp[2]).sum(), (plus[o] * lp[2]).sum()
            torq[0, 0, i] += lam * (sa + 1j * sb)
            torq[0, 1, i] += lam * (sc - (sz2[o] * lp[0]).sum())
            torq[0, 2, i] += lam * (-1j * (minus[o] * lp[0]).sum() - (plus[o] * lp[1]).sum())
        torq[0, :, i] *= 0.5
        m = np.zeros(3) if mvec is None else np.asarray(mvec[i], float)
        d1, d2, d3 = dist[1, i], dist[2, i], dist[3, i]
        torq[1, :, i] = Um[i] * np.array([m[2] * d2 - m[1] * d3, m[0] * d3 - m[2] * d1, m[1] * d1 - m[0] * d2])
        if hhw is not None:
            h = np.asarray(hhw[i], float)
            torq[2, :, i] = 2.0 * np.array([h[1] * d3 - h[2] * d2, h[2] * d1 - h[0] * d3, h[0] * d2 - h[1] * d1])
    # spin disturbance vector in the (+, up, down, -) basis, then the halved spin components
    sd = np.concatenate([dist[1] + 1j * dist[2], dist[0] + dist[3], dist[0] - dist[3], dist[1] - 1j * dist[2]])
    dist[1:4] *= 0.5
    sd *= 0.5
    beff = np.linalg.solve(site_reduced(system, chiorb), sd)
    bp, bu, bd, bm = beff.reshape(4, nat)
    bc = np.stack([bu + bd, 0.5 * (bp + bm), -0.5j * (bp - bm), 0.5 * (bu - bd)])
    return {"disturbances": dist, "torques": torq, "beff": bc, "total_disturbances": dist.sum(axis=1),
            "total_torques": torq.sum(axis=2), "total_beff": bc.sum(axis=1)}


def site_parameters(system, theta_deg=None, phi_deg=None):
    """Per-site (lvec, lpvec, lambda_p, lambda_d, porbs, dorbs, Um) of a TBSystem; theta / phi are the
    moment angles in degrees per site (zero when None)."""
    nat = system.n_atoms
    th = np.zeros(nat) if theta_deg is None else np.asarray(theta_deg, float)
    ph = np.zeros(nat) if phi_deg is None else np.asarray(phi_deg, float)
    els = [system.elements[t] for t in system.atom_type]
    lvec = [type_lvec(el.orbs) for el in els]
    lpvec = [lp_matrix(lvec[i], th[i], ph[i]) for i in range(nat)]
    porbs = [[a for a, o in enumerate(el.orbs) if 2 <= o <= 4] for el in els]
    return (lvec, lpvec, [el.lambda_p for el in els], [el.lambda_d for el in els], porbs, system.dorbs,
            system.Um())
