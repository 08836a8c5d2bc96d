"""Ground-state orbital moments from the on-site orbital density (calculate_L,
mod_expectation.F90:984-1009), the host algebra after tg_gs_orbital.

gupgd[i, a, b] is the reference's gupgd(a, b, i) (tg_gs_orbital); lvec / lpvec per site
are L (3, n, n) in the global and the local frame (titan_b200.host.response.site_parameters).
"""
from __future__ import annotations

import numpy as np


def calculate_l(system, gupgd, lvec, lpvec):
    """(lxm, lym, lzm, lxpm, lypm, lzpm) per site: Re sum_{mu,nu} L(mu, nu, c) gupgd(mu, nu, i)."""
    nat = system.n_atoms
    lm = np.zeros((3, nat))
    lpm = np.zeros((3, nat))
    for i in range(nat):
        n = system.norbs[i]
        P = gupgd[i, :n, :n]
        lm[:, i] = np.einsum("cmn,mn->c", lvec[i], P).real
        lpm[:, i] = np.einsum("cmn,mn->c", lpvec[i], P).real
    return lm[0], lm[1], lm[2], lpm[0], lpm[1], lpm[2]
