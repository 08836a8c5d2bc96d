"""Host-side Jacobian assembly (tg_jacobian_assemble) against the oracle's
calcJacobian_greenfunction, with the GG tensor and Fermi column computed by
numpy on the CPU (no GPU needed)."""
import numpy as np
import pytest

from oracle import titan_oracle as O
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state

from gg_numpy import fermi_column_numpy, gg_tensor_numpy


@pytest.mark.parametrize("shape,nk", [("bcc1", (3, 3, 3)), ("sq2", (3, 3, 1))])
@pytest.mark.parametrize("fixEf", [False, True])
def test_assemble_matches_oracle(shape, nk, fixEf):
    from titan_b200.native import jacobian_assemble, jacobian_layout
    deck = synthetic.make_deck(shape, nk=nk, n1gl=4, parts=1, n3gl=4)
    s = deck.system
    st = initial_state(s)
    h0 = s.h0(st)
    m = O.Model(s, h0)
    Ef = s.Ef
    ek = deck.ek
    G = m.green(Ef + 1j * (ek.point_energy() + s.eta), ek.kp)
    T = gg_tensor_numpy(s, G, ek.weight)
    Gr = m.green(np.full(deck.real_kp.shape[0], Ef + 1j * s.eta), deck.real_kp)
    D = fermi_column_numpy(s, Gr, deck.real_w)
    J = jacobian_assemble(s, T, D, fixEf)
    ref = O.jacobian(m, ek, (deck.real_kp, deck.real_w), Ef, s.eta, fixEf)
    neq, per = jacobian_layout(s, fixEf)
    assert J.shape == ref.shape == (neq, neq)
    assert np.max(np.abs(J - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_layout_counts():
    from titan_b200.native import jacobian_layout
    s = synthetic.make_system("sq2")
    nd = [len(d) for d in s.dorbs]
    neq, per = jacobian_layout(s, False)
    assert neq == sum(nd) + 3 * s.n_atoms + 1          # Un = Um != 0 on every site
    assert list(per) == [0, nd[0] + 3, nd[0] + nd[1] + 6]
