"""Disturbance response (eintshe + calculate_all) on the GPU through the C ABI (needs a B200)."""
import os

import numpy as np
import pytest

from golden_resp import check_responses
from oracle import titan_oracle as O
from titan_b200.host import response as R
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
UE = np.array([1.0, 0.5, 0.2]) / np.linalg.norm([1.0, 0.5, 0.2])


@pytest.fixture(scope="module")
def gpu():
    from titan_b200.native import GreenGPU
    g = GreenGPU(0)
    yield g
    g.close()


def _nanoribbon():
    from titan_b200.host.deck import Deck
    from titan_b200.host.system import read_sc_file
    d = Deck.from_directory(os.path.join(GOLDEN, "nanoribbon"))
    s = d.system
    st = read_sc_file(os.path.join(GOLDEN, "nanoribbon", "selfconsistency.dat"), s.norbs)
    s.Ef = st.Ef
    return d, st


class _SubMesh:
    """A subset of an imaginary-axis (E, k) list with the EKMesh accessors the oracle reads."""

    def __init__(self, ek, sel):
        self.kp = ek.kp[sel]
        self.weight = ek.weight[sel]
        self.n_points = len(sel)
        self._y = ek.point_energy()[sel]

    def point_energy(self):
        return self._y


# dimH 18 and 36 (shared-memory operands), 72 and 90 (operands read from L2)
@pytest.mark.parametrize("shape,nk,e,q", [
    ("bcc1", (3, 3, 3), 0.0, (0, 0, 0)),
    ("bcc1", (3, 3, 3), 0.04, (0.1, 0.0, 0.2)),
    ("sq2", (4, 4, 1), 0.05, (0.05, 0.02, 0.0)),
    ("bcc4", (2, 2, 2), 0.03, (0.0, 0.1, 0.0)),
    ("slab5", (3, 3, 1), 0.02, (0.02, 0.0, 0.0)),
])
def test_she_matches_oracle(gpu, shape, nk, e, q):
    deck = synthetic.make_deck(shape, nk=nk, n1gl=6, parts=1, n3gl=4)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.setup(deck, h0)
    x2, p2 = deck.real_points(e, s.Ef)
    q = np.array(q, float)
    got = gpu.she(q, e, s.Ef, s.eta, s.etap, x2, p2, UE)
    ref = O.eintshe(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), q, e, s.Ef, s.eta, s.etap, x2, p2, UE)
    assert np.max(np.abs(got - ref)) <= 1e-10 * np.max(np.abs(ref)), shape


def test_she_nanoribbon_submesh_and_prefactor(gpu):
    """A random (E, k) subset of the nanoribbon mesh at q != 0; the prefactor multiplies the integral."""
    d, st = _nanoribbon()
    s = d.system
    h0 = s.h0(st)
    rng = np.random.default_rng(5)
    sub = _SubMesh(d.ek, np.sort(rng.choice(d.ek.n_points, 300, replace=False)))
    rsel = np.sort(rng.choice(len(d.real_w), 20, replace=False))
    gpu.set_system(s)
    gpu.set_h0(h0)
    gpu.set_imag_mesh_arrays(np.ascontiguousarray(sub.point_energy()), np.ascontiguousarray(sub.kp),
                             np.ascontiguousarray(sub.weight))
    gpu.set_real_mesh(d.real_kp[rsel], d.real_w[rsel])
    e = float(d.frequencies()[0])
    x2, p2 = d.real_points(e, s.Ef)
    q = np.array([0.01, 0.03, 0.0])
    ue = d.params["efield"]
    raw = gpu.she(q, e, s.Ef, s.eta, s.etap, x2, p2, ue)
    ref = O.eintshe(O.Model(s, h0), sub, (d.real_kp[rsel], d.real_w[rsel]), q, e, s.Ef, s.eta, s.etap, x2, p2, ue)
    assert np.max(np.abs(raw - ref)) <= 1e-11 * np.max(np.abs(ref))
    P = np.eye(s.dimens) + 0.01 * (rng.standard_normal((s.dimens, s.dimens))
                                   + 1j * rng.standard_normal((s.dimens, s.dimens)))
    pre = gpu.she(q, e, s.Ef, s.eta, s.etap, x2, p2, ue, prefactor=P)
    assert np.max(np.abs(pre - P @ raw)) <= 1e-12 * np.max(np.abs(P @ raw))


def test_she_nanoribbon_golden_through_gpu(gpu):
    """The reference's nanoribbon in an electric field along x: chi_HF and the disturbance
    integral on the GPU, the calculate_all algebra on the host, against every site and total of
    the reference's charge / spin / orbital disturbances, torques and effective fields."""
    d, st = _nanoribbon()
    s = d.system
    gpu.setup(d, s.h0(st))
    e = float(d.frequencies()[0])
    x2, p2 = d.real_points(e, s.Ef)
    chi = gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2, precision="fp64")
    U = O.umatrix(s)
    pref = R.prefactor(chi, U)
    tchi = gpu.she(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2, d.params["efield"], prefactor=pref)
    lvec, lpvec, lam_p, lam_d, porbs, dorbs, Um = R.site_parameters(s)
    out = R.responses(s, tchi, pref @ chi, lvec, lpvec, lam_p, lam_d, porbs, dorbs, Um)
    check_responses("nanoribbon", out, s.n_atoms)


@pytest.mark.parametrize("shape,e,q", [("bcc1", 0.04, (0.1, 0.0, 0.2)), ("sq2", 0.05, (0.0, 0.0, 0.0))])
def test_she_spectral_equals_gauss_jordan(gpu, shape, e, q):
    """The disturbance integral from spectral Green functions (uniform meshes, on request),
    from Gauss-Jordan per point and from the default (at dimH 36 the split: spectral for
    Im z >= 10 eta, Gauss-Jordan below) agree to 1e-12."""
    deck = synthetic.make_deck(shape, nk=(4, 4, 4) if shape == "bcc1" else (6, 6, 1), n1gl=6, parts=1, n3gl=4)
    s = deck.system
    gpu.setup(deck, s.h0(initial_state(s)))
    x2, p2 = deck.real_points(e, s.Ef)
    q = np.array(q, float)
    auto = gpu.she(q, e, s.Ef, s.eta, s.etap, x2, p2, UE)
    try:
        gpu.set_green_method("spectral")
        sp = gpu.she(q, e, s.Ef, s.eta, s.etap, x2, p2, UE)
        gpu.set_green_method("gauss-jordan")
        gj = gpu.she(q, e, s.Ef, s.eta, s.etap, x2, p2, UE)
    finally:
        gpu.set_green_method("auto")
    assert np.max(np.abs(sp - gj)) <= 1e-12 * np.max(np.abs(gj))
    assert np.max(np.abs(auto - gj)) <= 1e-12 * np.max(np.abs(gj))
