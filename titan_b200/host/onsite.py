"""Local (k-independent) Hamiltonian h0: on-site, L.S, Zeeman and Hubbard terms.

Host-side restatement; the result is the ``h0`` the Green-function kernels add
to the Fourier sum:

* ``l_matrices``   -- source/mod_magnet.F90:295-354 (cubic-harmonic L)
* ``ls_matrix``    -- source/mod_SOC.F90:13-75 (lambda/2 L.sigma, rotated by
                      the quantisation angles; identity rotation for theta =
                      phi = 0, the default of mod_parameters.F90:47)
* ``sb_matrix``    -- source/mod_magnet.F90:266-293
* ``lb_matrix``    -- source/mod_magnet.F90:235-263
* ``hee_matrix``   -- source/mod_U_matrix.F90:29-55
* ``assemble_h0``  -- source/mod_hamiltonian.F90:35-63
"""
from __future__ import annotations

import math

import numpy as np

SQ3 = math.sqrt(3.0)

PAULI = {
    0: np.array([[1, 0], [0, 1]], dtype=complex),
    1: np.array([[0, 1], [1, 0]], dtype=complex),
    2: np.array([[0, -1j], [1j, 0]], dtype=complex),
    3: np.array([[1, 0], [0, -1]], dtype=complex),
}


def l_matrices():
    """L_x, L_y, L_z in the 9-orbital cubic basis, shape [3, 9, 9] (mod_magnet.F90:305-345)."""
    lz = np.zeros((9, 9), dtype=complex)
    lz[1, 2] = -1j
    lz[2, 1] = 1j
    lz[4, 7] = 2j
    lz[7, 4] = -2j
    lz[5, 6] = 1j
    lz[6, 5] = -1j
    lp = np.zeros((9, 9), dtype=complex)
    lp[1, 3] = -1
    lp[2, 3] = -1j
    lp[3, 1] = 1
    lp[3, 2] = 1j
    lp[4, 5] = -1
    lp[4, 6] = -1j
    lp[5, 4] = 1
    lp[5, 7] = -1j
    lp[5, 8] = -SQ3 * 1j
    lp[6, 4] = 1j
    lp[6, 7] = 1
    lp[6, 8] = -SQ3
    lp[7, 5] = 1j
    lp[7, 6] = -1
    lp[8, 5] = SQ3 * 1j
    lp[8, 6] = SQ3
    lm = lp.conj().T
    lx = 0.5 * (lp + lm)
    ly = -0.5j * (lp - lm)
    return np.stack([lx, ly, lz])


def _rot_y(theta_deg):
    t = math.radians(theta_deg)
    return np.array([[math.cos(t), 0, math.sin(t)], [0, 1, 0], [-math.sin(t), 0, math.cos(t)]])


def _rot_z(phi_deg):
    p = math.radians(phi_deg)
    return np.array([[math.cos(p), -math.sin(p), 0], [math.sin(p), math.cos(p), 0], [0, 0, 1]])


def ls_matrix(orbs, lambda_p: float, lambda_d: float, theta: float = 0.0, phi: float = 0.0):
    """Spin-orbit block (2nOrb x 2nOrb) of one site (mod_SOC.F90:13-75).

    ls = 1/2 sum_{m,n} lambda_l L_m R_{mn} sigma_n on the p and d sub-blocks,
    R = Rz(phi) Ry(theta); rows/cols are [up orbitals, down orbitals].
    """
    L = l_matrices()
    norb = len(orbs)
    rzy = _rot_z(phi) @ _rot_y(theta)
    ls = np.zeros((2 * norb, 2 * norb), dtype=complex)
    p_idx = [a for a, o in enumerate(orbs) if 2 <= o <= 4]
    d_idx = [a for a, o in enumerate(orbs) if 5 <= o <= 9]
    for n in range(3):
        for m in range(3):
            sig = PAULI[n + 1]
            for lam, idx in ((lambda_p, p_idx), (lambda_d, d_idx)):
                for nu in idx:
                    for mu in idx:
                        l_el = L[m, orbs[mu] - 1, orbs[nu] - 1]
                        c = lam * l_el * rzy[m, n]
                        ls[mu, nu] += c * sig[0, 0]
                        ls[mu, nu + norb] += c * sig[0, 1]
                        ls[mu + norb, nu] += c * sig[1, 0]
                        ls[mu + norb, nu + norb] += c * sig[1, 1]
    return 0.5 * ls


def sb_matrix(norb: int, b):
    """Spin Zeeman block for half-field b (mod_magnet.F90:266-293)."""
    sb = np.zeros((2 * norb, 2 * norb), dtype=complex)
    for mu in range(norb):
        nu = mu + norb
        sb[mu, mu] = b[2]
        sb[nu, nu] = -b[2]
        sb[nu, mu] = b[0] + 1j * b[1]
        sb[mu, nu] = b[0] - 1j * b[1]
    return sb


def lb_matrix(orbs, hhw):
    """Orbital Zeeman block L.hhw (mod_magnet.F90:235-263)."""
    L = l_matrices()
    norb = len(orbs)
    lb = np.zeros((2 * norb, 2 * norb), dtype=complex)
    for nu in range(norb):
        for mu in range(norb):
            v = sum(L[s, orbs[mu] - 1, orbs[nu] - 1] * hhw[s] for s in range(3))
            lb[mu, nu] = v
            lb[mu + norb, nu + norb] = v
    return lb


def hee_matrix(orbs, Un: float, Um: float, rho, rho0, rhod: float, rhod0: float,
               mzd: float, mzd0: float, mpd: complex, mpd0: complex):
    """Hubbard block of one site (mod_U_matrix.F90:29-55); only d orbitals carry it."""
    norb = len(orbs)
    hee = np.zeros((2 * norb, 2 * norb), dtype=complex)
    for mud in [a for a, o in enumerate(orbs) if 5 <= o <= 9]:
        nud = mud + norb
        charge = Un * (rho[mud] - rho0[mud]) + 0.5 * Un * (-rhod + rhod0)
        hee[mud, mud] = charge + 0.5 * Um * (-mzd + mzd0)
        hee[nud, nud] = charge + 0.5 * Um * (mzd - mzd0)
        hee[mud, nud] = -0.5 * Um * np.conj(mpd - mpd0)
        hee[nud, mud] = -0.5 * Um * (mpd - mpd0)
    return hee


def site_offsets(norbs):
    """ia(4, nAtoms) as 0-based [up_begin, up_end+1, down_begin, down_end+1] (mod_System.F90:101-135)."""
    ia = []
    pos = 0
    for n in norbs:
        ia.append((pos, pos + n, pos + n, pos + 2 * n))
        pos += 2 * n
    return ia


def assemble_h0(norbs, onsite_blocks, local_blocks):
    """h0 = sum_i [onsite (both spins) + lb + sb + hee + ls] on site blocks (mod_hamiltonian.F90:35-63)."""
    ia = site_offsets(norbs)
    n = ia[-1][3]
    h0 = np.zeros((n, n), dtype=complex)
    for i, (b0, b1, b2, b3) in enumerate(ia):
        h0[b0:b1, b0:b1] = onsite_blocks[i]
        h0[b2:b3, b2:b3] = onsite_blocks[i]
        h0[b0:b3, b0:b3] += local_blocks[i]
    return h0
