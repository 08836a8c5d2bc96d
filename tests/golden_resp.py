"""Readers of the reference's golden decks and outputs shared by the CPU and GPU tests: the
calculate_all output files (disturbances, torques and effective fields per site and their
totals) in tests/golden/<deck>/resp, and the Nb(100) monolayer deck with its LDOS files."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


RESP_KINDS = {"Cd": ("disturbances", 0), "Sx": ("disturbances", 1), "Sy": ("disturbances", 2),
              "Sz": ("disturbances", 3), "Lx": ("disturbances", 4), "Ly": ("disturbances", 5),
              "Lz": ("disturbances", 6), "SOTx": ("torques", (0, 0)), "SOTy": ("torques", (0, 1)),
              "SOTz": ("torques", (0, 2)), "XCTx": ("torques", (1, 0)), "XCTy": ("torques", (1, 1)),
              "XCTz": ("torques", (1, 2)), "Beff0": ("beff", 0), "Beffx": ("beff", 1), "Beffy": ("beff", 2),
              "Beffz": ("beff", 3)}


def resp_golden(name, kind, pos):
    """(amplitude, real, imag) of the first frequency of a calculate_all output file."""
    tag = "total" if pos is None else f"pos={pos}"
    f = os.path.join(GOLDEN, name, "resp", f"{kind}_{tag}.dat")
    row = [l for l in open(f) if not l.strip().startswith("#")][0].split()
    return float(row[1]), float(row[2]), float(row[3])


def check_responses(name, out, n_atoms, rtol=1e-8):
    """Compare a responses dict (disturbances / torques / beff per site and totals) with the
    golden files: every site value within rtol of the largest site amplitude of its kind, the
    sums over sites (which cancel to far below the site values for some kinds) within 5 rtol."""
    for kind, (key, c) in RESP_KINDS.items():
        arr = out[key]
        site = [arr[c][i] if isinstance(c, int) else arr[c[0], c[1], i] for i in range(n_atoms)]
        gold = [resp_golden(name, kind, i + 1) for i in range(n_atoms)]
        scale = max(max(g[0] for g in gold), 1e-300)
        tot = out["total_" + key][c] if isinstance(c, int) else out["total_" + key][c[0], c[1]]
        for k, (v, g) in enumerate(zip(site + [tot], gold + [resp_golden(name, kind, None)])):
            if g[0] == 0.0 and scale <= 1e-300:
                assert abs(v) <= 1e-14, (kind, v)
                continue
            tol = rtol * scale * (5.0 if k == n_atoms else 1.0)
            assert abs(abs(v) - g[0]) <= tol, (kind, k, abs(v), g[0])
            assert abs(v.real - g[1]) <= tol, (kind, k, v.real, g[1])
            assert abs(v.imag - g[2]) <= tol, (kind, k, v.imag, g[2])


def nb_ldos_golden(name):
    f = os.path.join(GOLDEN, "Nb_100_Monolayer", name)
    return np.array([[float(x) for x in l.split()] for l in open(f) if not l.startswith("#")])


def nb_monolayer():
    """The reference's Nb(100) monolayer deck (9 orbitals, SOC, Un = Um != 0 with the bulk
    reference densities of its initialrho file) at its golden self-consistent state."""
    from titan_b200.host.deck import Deck
    from titan_b200.host.system import read_sc_file
    d = Deck.from_directory(os.path.join(GOLDEN, "Nb_100_Monolayer"))
    st = read_sc_file(os.path.join(GOLDEN, "Nb_100_Monolayer", "selfconsistency.dat"), d.system.norbs)
    d.system.Ef = st.Ef
    return d, st
