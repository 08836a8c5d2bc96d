"""Jacobian, GG tensor, (V, B) adjoint and Newton self-consistency on the GPU
against the oracle and finite differences (needs a B200)."""
import os

import numpy as np
import pytest

from oracle import titan_oracle as O
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state

from gg_numpy import fermi_column_numpy, gg_tensor_numpy

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def gpu():
    from titan_b200.native import GreenGPU
    g = GreenGPU(0)
    yield g
    g.close()


def small(shape):
    nk = (3, 3, 3) if shape == "bcc1" else (3, 3, 1)
    deck = synthetic.make_deck(shape, nk=nk, n1gl=6, parts=1, n3gl=4)
    s = deck.system
    h0 = s.h0(initial_state(s))
    return deck, s, h0


@pytest.mark.parametrize("shape", ["bcc1", "sq2"])
def test_gg_tensor_and_fermi_column_match_numpy(gpu, shape):
    deck, s, h0 = small(shape)
    gpu.setup(deck, h0)
    m = O.Model(s, h0)
    ek = deck.ek
    G = m.green(s.Ef + 1j * (ek.point_energy() + s.eta), ek.kp)
    for resolved in (True, False):
        T = gpu.gg_tensor(s.Ef, s.eta, resolved)
        Tr = gg_tensor_numpy(s, G, ek.weight, resolved)
        assert np.max(np.abs(T - Tr)) <= 1e-12 * np.max(np.abs(Tr))
    Gr = m.green(np.full(deck.real_kp.shape[0], s.Ef + 1j * s.eta), deck.real_kp)
    D = gpu.fermi_column(s.Ef, s.eta)
    Dr = fermi_column_numpy(s, Gr, deck.real_w)
    assert np.max(np.abs(D - Dr)) <= 1e-12 * np.max(np.abs(Dr))


@pytest.mark.parametrize("shape", ["bcc1", "sq2"])
@pytest.mark.parametrize("fixEf", [False, True])
def test_jacobian_matches_oracle(gpu, shape, fixEf):
    deck, s, h0 = small(shape)
    gpu.setup(deck, h0)
    J = gpu.jacobian(s.Ef, s.eta, fixEf)
    ref = O.jacobian(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), s.Ef, s.eta, fixEf)
    assert np.max(np.abs(J - ref)) <= 1e-11 * max(1.0, np.max(np.abs(ref)))


def test_adjoint_vb_matches_central_differences(gpu):
    """d(n, m)/d(V, B) from tg_adjoint_vb against central differences, h = 1e-5, to 1e-7."""
    from titan_b200.host.vb import site_observables, vb_perturbation
    deck, s, h0 = small("sq2")
    gpu.setup(deck, h0)
    rng = np.random.default_rng(7)
    V0 = rng.normal(scale=0.05, size=s.n_atoms)
    B0 = rng.normal(scale=0.05, size=(s.n_atoms, 3))

    def x_of(V, B):
        gpu.set_h0(h0 + vb_perturbation(s, V, B))
        rho, mx, my, mz, _ = gpu.expectation(s.Ef, s.eta)
        return site_observables(s, rho, mx, my, mz).reshape(-1)

    gpu.set_h0(h0 + vb_perturbation(s, V0, B0))
    A = gpu.adjoint_vb(s.Ef, s.eta)
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


@pytest.mark.parametrize("shape", ["sq2", "bcc4"])
def test_adjoint_matches_the_reference_jacobian_through_the_chain_rule(gpu, shape):
    """The d-shell (V, B) adjoint against the oracle's analytic Jacobian (calcJacobian_greenfunction,
    mod_self_consistency.F90:795-1205).  With Un = 0 the unknowns are the d-shell moments and
    update_Umatrix (mod_U_matrix.F90:29-55) sets the d-shell field B_i = -(Um_i / 2) m_i, so
    J_ref + 1 = -(Um / 2) A on the moment rows and columns (the reference subtracts the identity
    on the first neq - 1 unknowns only)."""
    nk = (2, 2, 2) if shape == "bcc4" else (3, 3, 1)
    deck = synthetic.make_deck(shape, nk=nk, n1gl=6, parts=1, n3gl=4)
    s = deck.system
    for el in s.elements:
        el.Un = 0.0
    h0 = s.h0(initial_state(s))
    gpu.setup(deck, h0)
    A = gpu.adjoint_vb_orbitals(s.Ef, s.eta, s.dorbs)
    J = O.jacobian(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), s.Ef, s.eta, fixEf=True)
    neq = J.shape[0]
    assert neq == 3 * s.n_atoms
    Jp = J + np.diag([1.0] * (neq - 1) + [0.0])
    Um = s.Um()
    pred = np.zeros_like(J)
    for i in range(s.n_atoms):
        for j in range(s.n_atoms):
            for a in range(3):
                for b in range(3):
                    pred[3 * i + a, 3 * j + b] = -0.5 * Um[j] * A[1 + a + 4 * i, 1 + b + 4 * j]
    assert np.max(np.abs(Jp - pred)) <= 1e-10 * max(1.0, np.max(np.abs(Jp)))


def test_autograd_function_uses_the_adjoint(gpu):
    import torch
    from titan_b200.autograd import expectation_vb
    deck, s, h0 = small("sq2")
    gpu.setup(deck, h0)
    V = torch.tensor([0.02, -0.01], dtype=torch.float64, requires_grad=True)
    B = torch.tensor([[0.01, 0.0, 0.03], [0.0, -0.02, 0.01]], dtype=torch.float64, requires_grad=True)
    x = expectation_vb(V, B, gpu, s, h0, s.Ef, s.eta)
    c = torch.arange(1.0, 1.0 + x.numel(), dtype=torch.float64).reshape(x.shape)
    (c * x).sum().backward()
    from titan_b200.host.vb import vb_perturbation
    gpu.set_h0(h0 + vb_perturbation(s, V.detach().numpy(), B.detach().numpy()))
    A = gpu.adjoint_vb(s.Ef, s.eta)
    g = (A.T @ c.numpy().reshape(-1)).reshape(s.n_atoms, 4)
    assert np.allclose(V.grad.numpy(), g[:, 0], rtol=0, atol=1e-12)
    assert np.allclose(B.grad.numpy(), g[:, 1:], rtol=0, atol=1e-12)


def test_newton_returns_to_the_fe_fixed_point(gpu, fe_deck):
    """GPU Newton (tg_expectation + tg_jacobian) from a perturbed state converges to
    the reference's Fe self-consistent state (scResult, TOL 1e-7)."""
    from titan_b200.host import scf
    from titan_b200.host.system import MagState
    s = fe_deck.system
    gold = fe_deck.state
    gpu.setup(fe_deck, s.h0(gold))
    d = sorted(s.dorbs[0])
    pert = MagState(gold.rho.copy(), gold.mx.copy(), gold.my.copy(), gold.mz.copy(), gold.Ef + 0.002)
    pert.rho[0, d] += 0.01 * np.linspace(-1, 1, len(d))
    pert.mz[0, d] *= 0.97
    res = scf.newton(gpu, s, pert, fixEf=False, tol=1e-12, maxit=20)
    assert res.converged and res.iterations <= 12
    x_gold = scf.unknowns_from_state(s, gold)
    assert np.max(np.abs(res.x - x_gold)) < 1e-7
    assert np.max(np.abs(res.residual)) < 1e-10
    lines = open(os.path.join(GOLDEN, "Fe_bulk_susc", "scResult")).read().split("\n")
    nd = float(lines[3].split("Nd=")[1].split()[0])
    mzs = float(lines[5].split("Mz=")[1].split()[0])
    assert abs(res.state.rho[0, d].sum() - nd) < 1e-7
    assert abs(res.state.mz[0].sum() - mzs) < 1e-7


def test_globalised_newton_converges_from_the_seeded_start(gpu):
    """bcc 4-atom cell (dimH 72): plain Newton diverges from the seeded initial state (E_F runs
    off); with the step capped and halved until |f| decreases (the role of dnsqe's trust region,
    mod_dnsqe.F90) the GPU iteration reaches max |f| <= 1e-10, and the oracle's residual at the
    result agrees that it is a fixed point."""
    from titan_b200.host import scf
    deck = synthetic.make_deck("bcc4", nk=(3, 3, 3), n1gl=12, parts=1, n3gl=4)
    s = deck.system
    st0 = initial_state(s)
    gpu.setup(deck, s.h0(st0))
    res = scf.newton(gpu, s, st0, max_step=0.5, ftol=1e-10, maxit=80)
    assert res.converged and np.max(np.abs(res.residual)) <= 1e-10
    f_ref, _, _ = O.sc_residual(s, lambda state: O.Model(s, s.h0(state)), deck.ek, res.x, st0)
    assert np.max(np.abs(f_ref)) < 1e-9
