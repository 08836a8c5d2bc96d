"""Sum rule of the static transverse susceptibility (source/mod_sumrule.F90:10-160).

For a self-consistent state the q = 0, omega = 0 HF susceptibility and the on-site spin
density S (calcSmunu, on the GPU as tg_smunu) satisfy, per site i and orbital pair
(mu, nu),
    sum_k eps_mnk S^k_{mu nu}  =  2 sum_{j, gamma, xi} sum_{q, p} eps_nqp chi^{m p}_{(i mu nu),(j gamma xi)} B^q_{(j gamma xi)}
with chi in the cartesian spin basis and B the effective field of the exchange, SOC and
external field terms (Beffective).  The reference prints whether sum |lhs - rhs| < 1e-5.
Host algebra on dimens-sized matrices; rows in sigmaimunu2i order.
"""
from __future__ import annotations

import numpy as np

# cartesian (0, x, y, z) <- spin (+, up, down, -) and back (mod_constants.F90:34-44), row index first
SPIN_TO_CART = np.array([[0, 1, 1, 0], [0.5, 0, 0, 0.5], [-0.5j, 0, 0, 0.5j], [0, 0.5, -0.5, 0]], dtype=complex)
CART_TO_SPIN = np.array([[0, 1, 1j, 0], [0.5, 0, 0, 1], [0.5, 0, 0, -1], [0, 1, -1j, 0]], dtype=complex)


def _eps():
    e = np.zeros((3, 3, 3))
    for a, b, c in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):
        e[a, b, c], e[a, c, b] = 1.0, -1.0
    return e


def pair_rows(system):
    """[group, 4] sigmaimunu2i rows of every on-site orbital pair (i, mu, nu), groups in row order."""
    sidx = system.sigmaimunu2i()
    rows = []
    for i, n in enumerate(system.norbs):
        blk = sidx[:, i, :n, :n].reshape(4, -1).T
        rows.append(blk)
    return np.concatenate(rows, axis=0)


def effective_field(system, mvec, lvec, lambda_p, lambda_d, porbs, dorbs, Um, hhw=None):
    """Beff[dimens]: -Um m / 2 on the d diagonals, the external field on all diagonals, lambda L / 2 on
    the p and d blocks, on the cartesian rows (Beffective, mod_sumrule.F90:111-160)."""
    sidx = system.sigmaimunu2i()
    B = np.zeros(system.dimens, dtype=complex)
    for i in range(system.n_atoms):
        m = np.asarray(mvec[i], float)
        for c in range(3):
            d = np.asarray(dorbs[i], int)
            B[sidx[c + 1, i, d, d]] -= 0.5 * Um[i] * m[c]
            if hhw is not None:
                n = system.norbs[i]
                B[sidx[c + 1, i, np.arange(n), np.arange(n)]] += hhw[i][c]
            for lam, orbl in ((lambda_p[i], porbs[i]), (lambda_d[i], dorbs[i])):
                o = np.asarray(orbl, int)
                if o.size:
                    B[sidx[c + 1, i][np.ix_(o, o)]] += 0.5 * lam * lvec[i][c][np.ix_(o, o)]
    return B


def check(system, chi_hf, S, B):
    """(lhs, rhs, sum |lhs - rhs|); lhs / rhs [group, m, n] with S[i, k, mu, nu] from tg_smunu."""
    P = pair_rows(system)
    cart = np.einsum('pr,grht,tq->gphq', SPIN_TO_CART, chi_hf[P[:, :, None, None], P[None, None, :, :]], CART_TO_SPIN)
    eps = _eps()
    Sg = np.concatenate([S[i, :, :n, :n].reshape(3, -1).T for i, n in enumerate(system.norbs)], axis=0)
    lhs = np.einsum('mnk,gk->gmn', eps, Sg)
    rhs = 2.0 * np.einsum('nqp,gmhp,hq->gmn', eps, cart[:, 1:, :, 1:], B[P][:, 1:])
    return lhs, rhs, float(np.sum(np.abs(lhs - rhs)))
