"""The (V, B) adjoint formula against central finite differences of the
oracle's expectation values, on the CPU (checks signs and conventions of
the perturbation and of the Pauli contraction used by tg_adjoint_vb)."""
import numpy as np

from oracle import titan_oracle as O
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state
from titan_b200.host.vb import PAULI, site_observables, vb_perturbation
from gg_numpy import gg_tensor_numpy


def adjoint_from_T(T):
    nat = T.shape[0]
    A = np.zeros((4 * nat, 4 * nat))
    for i in range(nat):
        for j in range(nat):
            for a in range(4):
                for b in range(4):
                    v = 0.0
                    for q in range(16):
                        sp, t, tp, s = q & 1, (q >> 1) & 1, (q >> 2) & 1, (q >> 3) & 1
                        v += (PAULI[a][s, sp] * PAULI[b][t, tp] * T[i, j, 0, 0, q]).real
                    A[a + 4 * i, b + 4 * j] = v / np.pi
    return A


def test_adjoint_matches_finite_differences():
    deck = synthetic.make_deck("sq2", nk=(3, 3, 1), n1gl=6, parts=1, n3gl=4)
    s = deck.system
    h0 = s.h0(initial_state(s))
    ek = deck.ek
    Ef, eta = s.Ef, s.eta
    rng = np.random.default_rng(5)
    V0 = rng.normal(scale=0.05, size=s.n_atoms)
    B0 = rng.normal(scale=0.05, size=(s.n_atoms, 3))

    def x_of(V, B):
        m = O.Model(s, h0 + vb_perturbation(s, V, B))
        rho, mx, my, mz, _ = O.expectation(m, ek, Ef, eta)
        return site_observables(s, rho, mx, my, mz).reshape(-1)

    m0 = O.Model(s, h0 + vb_perturbation(s, V0, B0))
    G = m0.green(Ef + 1j * (ek.point_energy() + eta), ek.kp)
    A = adjoint_from_T(gg_tensor_numpy(s, G, ek.weight, resolved=False))
    h = 1e-5
    for j in range(s.n_atoms):
        for b in range(4):
            dV = np.zeros(s.n_atoms)
            dB = np.zeros((s.n_atoms, 3))
            if b == 0:
                dV[j] = h
            else:
                dB[j, b - 1] = h
            fd = (x_of(V0 + dV, B0 + dB) - x_of(V0 - dV, B0 - dB)) / (2 * h)
            assert np.max(np.abs(fd - A[:, b + 4 * j])) < 1e-7, (j, b)
