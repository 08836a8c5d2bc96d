"""Dimensions without a single-SM kernel and the d-only chi of the 16-layer slab, through
the C ABI (needs a B200).

dimH 108 (6-layer slab) lies outside the single-SM kernels' list and dimH 288 (16-layer
slab, the full workload's system) beyond it: both go through the thread-block-cluster
Gauss-Jordan kernel and the gathered chi0 operands.
"""
import numpy as np
import pytest

from oracle import titan_oracle as O
from titan_b200.host import synthetic
from titan_b200.host.accuracy import spin_block_errors
from titan_b200.host.system import initial_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from titan_b200.native import GreenGPU
    g = GreenGPU(0)
    yield g
    g.close()


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("shape", ["slab6", "slab16"])
def test_green_batch_general_dimension(gpu, shape):
    deck = synthetic.make_deck(shape, mesh=False)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.set_system(s)
    gpu.set_h0(h0)
    rng = np.random.default_rng(3)
    n = 11
    kp = rng.uniform(-2, 2, size=(n, 3))
    z = s.Ef + rng.uniform(-3, 3, n) + 1j * 10.0 ** rng.uniform(-3, 1, n)
    G = gpu.green_batch(z, kp)
    m = O.Model(s, h0)
    Gr = m.green(z, kp)
    for p in range(n):
        assert np.max(np.abs(G[p] - Gr[p])) <= 1e-12 * np.max(np.abs(Gr[p])) * s.dimH
    H = m.hk(kp)
    R = np.einsum("pab,pbc->pac", G, z[:, None, None] * np.eye(s.dimH)[None] - H)
    assert np.max(np.abs(R - np.eye(s.dimH)[None])) < 1e-9


def test_hamiltk_general_dimension(gpu):
    deck = synthetic.make_deck("slab6", mesh=False)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.set_system(s)
    gpu.set_h0(h0)
    kp = np.random.default_rng(1).uniform(-2, 2, size=(7, 3))
    Hr = O.Model(s, h0).hk(kp)
    assert np.max(np.abs(gpu.hamiltk_batch(kp) - Hr)) < 1e-13 * max(1.0, np.max(np.abs(Hr)))


def test_singular_point_general_dimension(gpu):
    """z - H exactly singular at the second point (no hoppings, h0 = 0, z = 0) -> status 2."""
    from titan_b200.native import TitanGPUError
    s_empty = synthetic.make_system("slab6")
    s_empty.neighbors = []
    s_empty.t0i = {}
    gpu.set_system(s_empty)
    gpu.set_h0(np.zeros((s_empty.dimH, s_empty.dimH), complex))
    z = np.array([1.0 + 1j, 0.0 + 0.0j, 2.0 + 0.5j])
    with pytest.raises(TitanGPUError) as ei:
        gpu.green_batch(z, np.zeros((3, 3)))
    assert ei.value.code == 2


def _chi_case(gpu, shape, sel_d, e, q):
    deck = synthetic.make_deck(shape, nk=(2, 2, 1), n1gl=4, parts=1, n3gl=3)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.setup(deck, h0)
    sel = [list(d) for d in s.dorbs] if sel_d else None
    gpu.set_chi_orbitals(sel)
    x2, p2 = deck.real_points(e, s.Ef)
    q = np.array(q, float)
    fp = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision="fp64")
    sp = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision="split")
    ref = O.eintshechi(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), q, e, s.Ef, s.eta, s.etap, x2, p2,
                       sel=sel)
    gpu.set_chi_orbitals(None)
    return fp, sp, ref


@pytest.mark.parametrize("e,q", [(0.0, (0, 0, 0)), (0.05, (0.1, 0.05, 0.0))])
def test_chi0_general_dimension_matches_oracle(gpu, e, q):
    fp, sp, ref = _chi_case(gpu, "slab6", False, e, q)
    assert rel(fp, ref) < 1e-10
    assert spin_block_errors(sp, fp)[1] < 1e-9
    assert rel(sp, ref) < 1e-9


@pytest.mark.parametrize("e,q", [(0.0, (0, 0, 0)), (0.05, (0.1, 0.0, 0.0))])
def test_chi0_d_only_slab16_matches_oracle(gpu, e, q):
    """The full workload's system (dimH 288) with the d-only chi of dimension 1600."""
    fp, sp, ref = _chi_case(gpu, "slab16", True, e, q)
    assert fp.shape == (1600, 1600)
    assert rel(fp, ref) < 1e-10
    assert spin_block_errors(sp, fp)[1] < 1e-9
    assert rel(sp, ref) < 1e-9


def test_d_only_rpa_is_the_dd_block_of_the_full_rpa(gpu):
    deck = synthetic.make_deck("sq2", nk=(4, 4, 1), n1gl=6, parts=1, n3gl=4)
    s = deck.system
    gpu.setup(deck, s.h0(initial_state(s)))
    e = 0.1
    x2, p2 = deck.real_points(e, s.Ef)
    full = gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2)
    sel = [list(d) for d in s.dorbs]
    gpu.set_chi_orbitals(sel)
    dd = gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2)
    gpu.set_chi_orbitals(None)
    r = O.sel_rows(s, sel)
    assert rel(dd, full[np.ix_(r, r)]) < 1e-12
    U = O.umatrix(s)
    rpa_full = gpu.dyson(full, U)
    rpa_dd = gpu.dyson(dd, U[np.ix_(r, r)])
    assert rel(rpa_dd, rpa_full[np.ix_(r, r)]) < 1e-10


def test_dyson_at_the_d_only_dimension_of_the_16_layer_slab(gpu):
    """tg_dyson at 1600 (the full workload's per-frequency solve) against numpy."""
    s = synthetic.make_system("slab16")
    gpu.set_system(s)
    sel = [list(d) for d in s.dorbs]
    r = O.sel_rows(s, sel)
    U = O.umatrix(s)[np.ix_(r, r)]
    rng = np.random.default_rng(5)
    D = 1600
    chi = 0.05 * (rng.standard_normal((D, D)) + 1j * rng.standard_normal((D, D))) / np.sqrt(D)
    got = gpu.dyson(chi, U)
    ref = O.dyson(chi, U)
    assert rel(got, ref) < 1e-10


@pytest.mark.parametrize("shape,sel_d,precision", [("slab6", False, "fp64"), ("slab16", True, "fp64"),
                                                   ("slab16", True, "split")])
def test_tridiagonal_resolvents_equal_gauss_jordan(gpu, shape, sel_d, precision):
    """Uniform meshes beyond the Jacobi kernel's dimensions: chi0 from G over the rows chi
    needs, formed from a Householder tridiagonalisation per k (the default there), equals the
    cluster Gauss-Jordan path, at q != 0 with the real axis."""
    deck = synthetic.make_deck(shape, nk=(3, 3, 1), n1gl=4, parts=1, n3gl=3)
    s = deck.system
    gpu.setup(deck, s.h0(initial_state(s)))
    gpu.set_chi_orbitals([list(d) for d in s.dorbs] if sel_d else None)
    e, q = 0.05, np.array([0.1, 0.0, 0.0])
    x2, p2 = deck.real_points(e, s.Ef)
    try:
        auto = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision=precision)
        gpu.set_green_method("gauss-jordan")
        gj = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision=precision)
    finally:
        gpu.set_green_method("auto")
        gpu.set_chi_orbitals(None)
    assert rel(auto, gj) < (1e-12 if precision == "fp64" else 1e-9)


@pytest.mark.parametrize("sel_d", [False, True])
def test_tridiagonal_real_axis_of_its_own(gpu, sel_d):
    """A real-axis BZ that differs from the imaginary-axis k list gets tridiagonalisations of
    its own (H(k) and H(k + q) slots apart from the imaginary axis'): equal to Gauss-Jordan
    and to the oracle on the same meshes."""
    deck = synthetic.make_deck("slab6", nk=(3, 3, 1), n1gl=4, parts=1, n3gl=3)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.setup(deck, h0)
    rkp = deck.real_kp + np.array([0.013, -0.021, 0.0])   # another k list than the imaginary axis'
    gpu.set_real_mesh(rkp, deck.real_w)
    sel = [list(d) for d in s.dorbs] if sel_d else None
    gpu.set_chi_orbitals(sel)
    e, q = 0.05, np.array([0.1, 0.0, 0.0])
    x2, p2 = deck.real_points(e, s.Ef)
    try:
        auto = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision="fp64")
        gpu.set_green_method("gauss-jordan")
        gj = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision="fp64")
    finally:
        gpu.set_green_method("auto")
        gpu.set_chi_orbitals(None)
    assert rel(auto, gj) < 1e-12
    ref = O.eintshechi(O.Model(s, h0), deck.ek, (rkp, deck.real_w), q, e, s.Ef, s.eta, s.etap, x2, p2, sel=sel)
    assert rel(auto, ref) < 1e-10
