"""Host-side set-up: meshes, index maps, Hamiltonian symmetries (no GPU)."""
import math

import numpy as np
import pytest

from titan_b200.host import mesh as M
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state
from oracle import titan_oracle as O


def test_gauleg_integrates_polynomials():
    x, w = M.gauleg(0.0, 2.0, 16)
    for p in range(0, 31):
        assert abs(np.sum(w * x ** p) - 2.0 ** (p + 1) / (p + 1)) < 1e-12 * 2.0 ** (p + 1)


def test_imag_points_sorted_and_weights_positive():
    y, w = M.imag_energy_points(2, 64)
    assert np.all(np.diff(y) > 0)
    assert np.all(w > 0)
    # integral of 1/(1+y)^2 over [0, inf) = 1
    assert abs(np.sum(w / (1 + y) ** 2) - 1.0) < 1e-10


@pytest.mark.parametrize("shape,nk", [("bcc1", (6, 6, 6)), ("sq2", (10, 10, 1)), ("bcc4", (3, 3, 3))])
def test_bz_weights_sum_to_one(shape, nk):
    s = synthetic.make_system(shape)
    kp, w = M.bz_fraction(s.a1, s.a2, s.a3, s.sysdim, nk)
    assert abs(w.sum() - 1.0) < 1e-12
    assert kp.shape[0] >= int(np.prod(nk[:s.sysdim]))


def test_sigmaimunu2i_is_a_permutation():
    s = synthetic.make_system("sq2")
    idx = s.sigmaimunu2i()
    flat = idx[idx >= 0]
    assert sorted(flat.tolist()) == list(range(s.dimens))
    # sigma fastest, then nu, then mu, then site (mod_System.F90:176-187)
    assert idx[1, 0, 0, 0] == 1 and idx[0, 0, 0, 1] == 4 and idx[0, 0, 1, 0] == 4 * 9


@pytest.mark.parametrize("shape", ["bcc1", "sq2", "slab5", "bcc4"])
def test_hk_hermitian_and_periodic(shape):
    s = synthetic.make_system(shape)
    h0 = s.h0(initial_state(s))
    m = O.Model(s, h0)
    k = np.array([[0.11, -0.23, 0.37]])
    H = m.hk(k)[0]
    assert np.max(np.abs(H - H.conj().T)) < 1e-13
    b = s.reciprocal()
    H2 = m.hk(k + b[0][None, :])[0]
    assert np.max(np.abs(H - H2)) < 1e-12


def test_green_resolvent_identity():
    s = synthetic.make_system("bcc1")
    m = O.Model(s, s.h0(initial_state(s)))
    k = np.array([[0.1, 0.2, 0.3], [0.0, 0.0, 0.0]])
    z = np.array([0.3 + 1e-3j, -1.0 + 0.5j])
    G = m.green(z, k)
    H = m.hk(k)
    for p in range(2):
        R = G[p] @ (z[p] * np.eye(s.dimH) - H[p])
        assert np.max(np.abs(R - np.eye(s.dimH))) < 1e-9
