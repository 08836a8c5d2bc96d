"""Local density of states (ldos_energy) on the GPU through the C ABI (needs a B200)."""
import numpy as np
import pytest

from oracle import titan_oracle as O
from golden_resp import nb_ldos_golden, nb_monolayer
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from titan_b200.native import GreenGPU
    g = GreenGPU(0)
    yield g
    g.close()


@pytest.mark.parametrize("method", ["auto", "gauss-jordan"])
def test_nb_ldos_golden_through_gpu(gpu, method):
    """The reference's Nb(100) monolayer LDOS (per orbital, both spins, 101 energies) from the
    spectral path (default) and from Gauss-Jordan per (k, e)."""
    d, st = nb_monolayer()
    s = d.system
    gpu.setup(d, s.h0(st))
    mu, md = nb_ldos_golden("lmdosu_site=1.dat"), nb_ldos_golden("lmdosd_site=1.dat")
    try:
        gpu.set_green_method(method)
        up, dn = gpu.ldos(mu[:, 0], s.eta)
    finally:
        gpu.set_green_method("auto")
    np.testing.assert_allclose(up[:, 0], mu[:, 1:], rtol=2e-9, atol=0)
    np.testing.assert_allclose(dn[:, 0], md[:, 1:], rtol=2e-9, atol=0)


@pytest.mark.parametrize("shape", ["bcc1", "sq2", "bcc4"])
def test_ldos_matches_oracle(gpu, shape):
    """Spectral and Gauss-Jordan LDOS against the oracle on seeded cells (dimH 18, 36, 72),
    energies across the bands, eta = 1e-3."""
    deck = synthetic.make_deck(shape, nk=(6, 6, 6) if shape != "sq2" else (12, 12, 1), n1gl=4, parts=1, n3gl=4)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.setup(deck, h0)
    es = s.Ef + np.linspace(-1.5, 1.0, 23)
    ref_u, ref_d = O.ldos(O.Model(s, h0), (deck.real_kp, deck.real_w), es, s.eta)
    sp_u, sp_d = gpu.ldos(es, s.eta)
    try:
        gpu.set_green_method("gauss-jordan")
        gj_u, gj_d = gpu.ldos(es, s.eta)
    finally:
        gpu.set_green_method("auto")
    scale = max(np.abs(ref_u).max(), np.abs(ref_d).max())
    for got in (sp_u, gj_u):
        assert np.max(np.abs(got - ref_u)) <= 1e-11 * scale
    for got in (sp_d, gj_d):
        assert np.max(np.abs(got - ref_d)) <= 1e-11 * scale
