"""The oracle's chi over an orbital subset (the d-only chi of the 16-layer slab) and the
exactness of the d-only RPA Dyson solve, on the CPU."""
import numpy as np

from oracle import titan_oracle as O
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state


def _sq2():
    deck = synthetic.make_deck("sq2", nk=(4, 4, 1), n1gl=4, parts=1, n3gl=4)
    s = deck.system
    return deck, s, O.Model(s, s.h0(initial_state(s)))


def test_subset_chi_is_the_sub_block_of_the_full_chi():
    deck, s, m = _sq2()
    e, q = 0.05, np.array([0.1, 0.0, 0.0])
    x2, p2 = deck.real_points(e, s.Ef)
    args = (m, deck.ek, (deck.real_kp, deck.real_w), q, e, s.Ef, s.eta, s.etap, x2, p2)
    full = O.eintshechi(*args)
    sel = [list(d) for d in s.dorbs]
    sub = O.eintshechi(*args, sel=sel)
    r = O.sel_rows(s, sel)
    assert sub.shape == (200, 200)
    assert np.max(np.abs(sub - full[np.ix_(r, r)])) < 1e-14 * np.max(np.abs(full))


def test_d_only_dyson_equals_the_dd_block_of_the_full_dyson():
    """U = P_d U P_d (mod_susceptibilities.F90:106-159), so by the Woodbury identity the d-d
    block of (1 + chi U)^-1 chi depends on chi_dd alone."""
    deck, s, m = _sq2()
    x2, p2 = deck.real_points(0.1, s.Ef)
    full = O.eintshechi(m, deck.ek, (deck.real_kp, deck.real_w), np.zeros(3), 0.1, s.Ef, s.eta, s.etap, x2, p2)
    U = O.umatrix(s)
    sel = [list(d) for d in s.dorbs]
    r = O.sel_rows(s, sel)
    rest = np.setdiff1d(np.arange(s.dimens), r)
    assert np.max(np.abs(U[rest])) == 0.0 and np.max(np.abs(U[:, rest])) == 0.0
    rpa_full = O.dyson(full, U)
    rpa_dd = O.dyson(full[np.ix_(r, r)], U[np.ix_(r, r)])
    ref = rpa_full[np.ix_(r, r)]
    assert np.linalg.norm(rpa_dd - ref) / np.linalg.norm(ref) < 1e-12
