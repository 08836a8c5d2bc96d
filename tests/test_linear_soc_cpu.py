"""The oracle's linear-SOC susceptibility (eintshechilinearsoc restated) is the first-order SOC
response: chi(H0 + t V) = chi(H0) + t chi_lsoc + O(t^2), checked by central differences
(the reference ships no golden file for this path)."""
import numpy as np

from oracle import titan_oracle as O
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state


def test_linear_soc_is_the_first_order_soc_response():
    deck = synthetic.make_deck("bcc1", nk=(3, 3, 3), n1gl=6, parts=1, n3gl=4)
    s = deck.system
    h00, V = s.linear_soc_split(initial_state(s))
    assert np.abs(V).max() > 0.0 and np.allclose(h00 + V, s.h0(initial_state(s)))
    e, q = 0.03, np.array([0.1, 0.0, 0.2])
    x2, p2 = deck.real_points(e, s.Ef)
    args = (deck.ek, (deck.real_kp, deck.real_w), q, e, s.Ef, s.eta, s.etap, x2, p2)
    chi0, lsoc = O.eintshechi_linear_soc(O.Model(s, h00), V, *args)
    assert np.abs(chi0 - O.eintshechi(O.Model(s, h00), *args)).max() == 0.0
    t = 1e-4
    fd = (O.eintshechi(O.Model(s, h00 + t * V), *args) - O.eintshechi(O.Model(s, h00 - t * V), *args)) / (2 * t)
    assert np.abs(fd - lsoc).max() < 1e-6 * np.abs(lsoc).max()
