"""Error of a chi against a reference chi, normwise per 4 x 4 spin block.

chi rows and columns are (sigma, i, mu, nu) with sigma fastest (sigmaimunu2i,
mod_System.F90:176-187), so rows 4b .. 4b + 3 form the spin block of one
(i, mu, nu); block (a, b) is the 4 x 4 matrix of one row group and one column
group.
"""
from __future__ import annotations

import numpy as np


def spin_block_errors(chi, ref, significant=1e-6):
    """(max over blocks of ||chi_b - ref_b||_F / ||ref_b||_F over blocks with a non-zero
    reference norm, the same max over blocks holding at least `significant` of the largest
    block norm, the whole-matrix Frobenius error, the number of non-zero blocks)."""
    D = ref.shape[0]
    nb = D // 4
    f = np.asarray(ref).reshape(nb, 4, nb, 4)
    d = (np.asarray(chi) - np.asarray(ref)).reshape(nb, 4, nb, 4)
    fn = np.sqrt(np.einsum("iajb,iajb->ij", np.abs(f), np.abs(f)))
    dn = np.sqrt(np.einsum("iajb,iajb->ij", np.abs(d), np.abs(d)))
    nz = fn > 0
    rel = np.where(nz, dn / np.where(nz, fn, 1.0), 0.0)
    big = fn >= significant * fn.max()
    return (float(rel[nz].max()), float(rel[big].max()),
            float(np.linalg.norm(chi - ref) / np.linalg.norm(ref)), int(nz.sum()))


def spin_block_table(chi, ref, thresholds=(1e-2, 1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8)):
    """{threshold: (blocks holding >= threshold of the largest block norm, max normwise error
    over them)} for the 4 x 4 spin blocks of chi against ref."""
    D = ref.shape[0]
    nb = D // 4
    f = np.asarray(ref).reshape(nb, 4, nb, 4)
    d = (np.asarray(chi) - np.asarray(ref)).reshape(nb, 4, nb, 4)
    fn = np.sqrt(np.einsum("iajb,iajb->ij", np.abs(f), np.abs(f)))
    dn = np.sqrt(np.einsum("iajb,iajb->ij", np.abs(d), np.abs(d)))
    out = {}
    for t in thresholds:
        sel = fn >= t * fn.max()
        out[f"{t:.0e}"] = (int(sel.sum()), float(np.max(dn[sel] / fn[sel])))
    return out
