"""CUDA path vs the CPU oracle, through the C ABI (needs a B200)."""
import os

import numpy as np
import pytest

from oracle import titan_oracle as O
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def gpu():
    from titan_b200.native import GreenGPU
    g = GreenGPU(0)
    yield g
    g.close()


def _setup(gpu, deck, state=None):
    s = deck.system
    st = state if state is not None else initial_state(s)
    h0 = s.h0(st)
    gpu.setup(deck, h0)
    return s, h0


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("shape", ["bcc1", "sq2", "bcc4", "slab5"])
def test_hamiltk_matches_calchk(gpu, shape):
    deck = synthetic.make_deck(shape, mesh=False)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.set_system(s)
    gpu.set_h0(h0)
    kp = np.random.default_rng(1).uniform(-2, 2, size=(40, 3))
    H = gpu.hamiltk_batch(kp)
    Hr = O.Model(s, h0).hk(kp)
    assert np.max(np.abs(H - Hr)) < 1e-13 * max(1.0, np.max(np.abs(Hr)))


@pytest.mark.parametrize("shape", ["bcc1", "sq2", "bcc4", "slab5"])
def test_green_batch_matches_lapack_inverse(gpu, shape):
    deck = synthetic.make_deck(shape, mesh=False)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.set_system(s)
    gpu.set_h0(h0)
    rng = np.random.default_rng(2)
    n = 37
    kp = rng.uniform(-2, 2, size=(n, 3))
    # near the real axis (Im z = eta = 1e-3) up to far away
    z = s.Ef + rng.uniform(-3, 3, n) + 1j * 10.0 ** rng.uniform(-3, 1, n)
    G = gpu.green_batch(z, kp)
    m = O.Model(s, h0)
    Gr = m.green(z, kp)
    for p in range(n):
        assert np.max(np.abs(G[p] - Gr[p])) <= 1e-12 * np.max(np.abs(Gr[p])) * s.dimH
    H = m.hk(kp)
    R = np.einsum("pab,pbc->pac", G, z[:, None, None] * np.eye(s.dimH)[None] - H)
    assert np.max(np.abs(R - np.eye(s.dimH)[None])) < 1e-9


def test_singular_matrix_reports_point_index(gpu):
    """z - H exactly singular (H = 0, z = 0 at the third point) -> status 3."""
    from titan_b200.native import TitanGPUError
    deck = synthetic.make_deck("bcc1", mesh=False)
    s = deck.system
    s_empty = synthetic.make_system("bcc1")
    s_empty.neighbors = []
    s_empty.t0i = {}
    gpu.set_system(s_empty)
    gpu.set_h0(np.zeros((s.dimH, s.dimH), complex))
    z = np.array([1.0 + 1j, 2.0 + 0.5j, 0.0 + 0.0j, 3.0 + 0j])
    with pytest.raises(TitanGPUError) as ei:
        gpu.green_batch(z, np.zeros((4, 3)))
    assert ei.value.code == 3


@pytest.mark.parametrize("shape,nk,e,q", [
    ("bcc1", (4, 4, 4), 0.0, (0, 0, 0)),
    ("bcc1", (4, 4, 4), 0.05, (0, 0, 0)),
    ("bcc1", (3, 3, 3), 0.02, (0.1, 0.0, 0.2)),
    ("sq2", (6, 6, 1), 0.0, (0, 0, 0)),
    ("sq2", (5, 5, 1), 0.1, (0.05, 0.02, 0.0)),
])
def test_chi0_fp64_matches_oracle(gpu, shape, nk, e, q):
    deck = synthetic.make_deck(shape, nk=nk, n1gl=8, parts=1, n3gl=6)
    s, h0 = _setup(gpu, deck)
    x2, p2 = deck.real_points(e, s.Ef)
    chi = gpu.chi0(np.array(q, float), e, s.Ef, s.eta, s.etap, x2, p2)
    ref = O.eintshechi(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), np.array(q, float), e, s.Ef, s.eta,
                       s.etap, x2, p2)
    assert rel(chi, ref) < 1e-10


def test_chi0_batch_equals_single_calls(gpu):
    deck = synthetic.make_deck("bcc1", nk=(3, 3, 3), n1gl=6, parts=1, n3gl=4)
    s, h0 = _setup(gpu, deck)
    es = [0.0, 0.03, 0.07]
    xs = [deck.real_points(e, s.Ef) for e in es]
    batch = gpu.chi0_batch(np.zeros(3), es, s.Ef, s.eta, s.etap, [x[0] for x in xs], [x[1] for x in xs])
    for w, e in enumerate(es):
        single = gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, xs[w][0], xs[w][1])
        assert rel(batch[w], single) < 1e-13


def test_fe_golden_through_gpu(gpu, fe_deck, fe_chi_golden):
    """The reference's Fe_bulk_susc chi_HF / chi_RPA rows through the GPU path."""
    s = fe_deck.system
    h0 = s.h0(fe_deck.state)
    gpu.setup(fe_deck, h0)
    ghf, grpa = fe_chi_golden
    U = O.umatrix(s)
    for idx in (0, 1, 5):
        e = fe_deck.frequencies()[idx]
        x2, p2 = fe_deck.real_points(e, s.Ef)
        chi = gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2)
        rpa = gpu.dyson(chi, U)
        hf_row = O.golden_row(s, e, 0.0, O.site_reduce(s, chi), 0, 0)
        rpa_row = O.golden_row(s, e, 0.0, O.site_reduce(s, rpa), 0, 0)
        for a, b in zip(hf_row, ghf[idx]):
            if abs(b) > 1e-6:
                assert abs(a - b) <= 1e-8 * abs(b), (idx, a, b)
        for a, b in zip(rpa_row, grpa[idx]):
            if abs(b) > 1e-6:
                assert abs(a - b) <= 5e-8 * abs(b), (idx, a, b)


def test_expectation_matches_oracle_and_fe_fixed_point(gpu, fe_deck):
    s = fe_deck.system
    st = fe_deck.state
    h0 = s.h0(st)
    gpu.setup(fe_deck, h0)
    rho, mx, my, mz, mp = gpu.expectation(st.Ef, s.eta)
    assert np.max(np.abs(rho - st.rho)) < 1e-7
    assert np.max(np.abs(mz - st.mz)) < 1e-7
    r2, x2, y2, z2, mp2 = O.expectation(O.Model(s, h0), fe_deck.ek, st.Ef, s.eta)
    for a, b in ((rho, r2), (mx, x2), (my, y2), (mz, z2)):
        assert np.max(np.abs(a - b)) < 1e-12


def test_dyson_matches_numpy(gpu):
    rng = np.random.default_rng(3)
    n = 100
    chi = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    U = np.zeros((n, n), complex)
    U[np.arange(0, n, 3), np.arange(0, n, 3)] = 0.3
    out = gpu.dyson(chi, U)
    ref = O.dyson(chi, U)
    assert rel(out, ref) < 1e-12


def test_chi0_adaptive_mesh_matches_oracle(gpu):
    """Non-uniform (E, k) list: per-energy k counts decay (adaptiveMesh.F90:199-218)."""
    from titan_b200.host.deck import Deck
    base = synthetic.make_deck("bcc1", nk=(4, 4, 4), n1gl=6, parts=1, n3gl=4, mesh=False)
    p = dict(base.params)
    p["nk_per_energy"] = [64, 64, 27, 27, 8, 8]
    deck = Deck.from_system(base.system, p, True)
    s, h0 = _setup(gpu, deck)
    e = 0.04
    x2, p2 = deck.real_points(e, s.Ef)
    chi = gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2)
    ref = O.eintshechi(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), np.zeros(3), e, s.Ef, s.eta,
                       s.etap, x2, p2)
    assert rel(chi, ref) < 1e-10
    rho, mx, my, mz, mp = gpu.expectation(s.Ef, s.eta)
    r2, x2_, y2, z2, mp2 = O.expectation(O.Model(s, h0), deck.ek, s.Ef, s.eta)
    assert np.max(np.abs(rho - r2)) < 1e-12 and np.max(np.abs(mz - z2)) < 1e-12


@pytest.mark.parametrize("shape,nk,e,q", [
    ("bcc1", (4, 4, 4), 0.0, (0, 0, 0)),
    ("bcc1", (3, 3, 3), 0.02, (0.1, 0.0, 0.2)),
    ("sq2", (6, 6, 1), 0.0, (0, 0, 0)),
    ("sq2", (5, 5, 1), 0.1, (0.05, 0.02, 0.0)),
])
def test_chi0_split_matches_fp64_and_oracle(gpu, shape, nk, e, q):
    """int8-sliced tensor-core contraction: normwise relative error <= 1e-9, and within the
    format's error bound (tg_chi0_error_bound; FP64 rounding of either path on top)."""
    deck = synthetic.make_deck(shape, nk=nk, n1gl=8, parts=1, n3gl=6)
    s, h0 = _setup(gpu, deck)
    x2, p2 = deck.real_points(e, s.Ef)
    qv = np.array(q, float)
    sp = gpu.chi0(qv, e, s.Ef, s.eta, s.etap, x2, p2, precision="split")
    bound = gpu.error_bound(1)[0]
    fp = gpu.chi0(qv, e, s.Ef, s.eta, s.etap, x2, p2, precision="fp64")
    assert gpu.error_bound(1)[0] == 0.0
    assert rel(sp, fp) < 1e-9
    assert 0.0 < bound < 1e-6 and rel(sp, fp) <= bound + 1e-13, (bound, rel(sp, fp))
    ref = O.eintshechi(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), qv, e, s.Ef, s.eta, s.etap, x2, p2)
    assert rel(sp, ref) < 1e-9


def test_chi0_split_fe_golden(gpu, fe_deck, fe_chi_golden):
    """The reference's Fe_bulk_susc chi_HF rows through the split-precision path."""
    s = fe_deck.system
    gpu.setup(fe_deck, s.h0(fe_deck.state))
    ghf, _ = fe_chi_golden
    for idx in (0, 5):
        e = fe_deck.frequencies()[idx]
        x2, p2 = fe_deck.real_points(e, s.Ef)
        chi = gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2, precision="split")
        hf_row = O.golden_row(s, e, 0.0, O.site_reduce(s, chi), 0, 0)
        for a, b in zip(hf_row, ghf[idx]):
            if abs(b) > 1e-6:
                assert abs(a - b) <= 1e-8 * abs(b), (idx, a, b)


@pytest.mark.parametrize("shape,nk", [("bcc4", (2, 2, 2)), ("slab5", (3, 3, 1))])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("split", 1e-9)])
def test_chi0_larger_cells_match_oracle(gpu, shape, nk, precision, tol):
    """4-atom bcc (dimH 72) and 5-layer slab (dimH 90): 16 and 25 site pairs."""
    deck = synthetic.make_deck(shape, nk=nk, n1gl=4, parts=1, n3gl=4)
    s, h0 = _setup(gpu, deck)
    e = 0.05
    x2, p2 = deck.real_points(e, s.Ef)
    q = np.array([0.03, 0.0, 0.0])
    chi = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision=precision)
    ref = O.eintshechi(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), q, e, s.Ef, s.eta, s.etap, x2, p2)
    assert rel(chi, ref) < tol


def test_chi0_sharded_mesh_sums_to_full(gpu):
    """Two mesh shares (as two ranks would hold them) add up to the full chi0."""
    from titan_b200.host.sharding import shard_imag_mesh, shard_real_bz
    deck = synthetic.make_deck("sq2", nk=(6, 6, 1), n1gl=8, parts=1, n3gl=6)
    s, h0 = _setup(gpu, deck)
    e = 0.05
    x2, p2 = deck.real_points(e, s.Ef)
    full = gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2, precision="fp64")
    parts = []
    for r in range(2):
        gpu.set_imag_mesh(shard_imag_mesh(deck.ek, r, 2))
        gpu.set_real_mesh(*shard_real_bz(deck.real_kp, deck.real_w, r, 2))
        parts.append(gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2, precision="fp64"))
    assert rel(parts[0] + parts[1], full) < 1e-13


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_nanoribbon_golden_through_gpu(gpu, precision):
    """The reference's 10-site px/py nanoribbon: chi_HF and chi_RPA of all 100 site
    pairs at omega = 1e-6 through the GPU path (dimH 40, 100 pairs of 16 x 16)."""
    from titan_b200.host.deck import Deck
    from titan_b200.host.system import read_sc_file
    d = Deck.from_directory(os.path.join(GOLDEN, "nanoribbon"))
    s = d.system
    st = read_sc_file(os.path.join(GOLDEN, "nanoribbon", "selfconsistency.dat"), s.norbs)
    s.Ef = st.Ef
    gpu.setup(d, s.h0(st))
    e = float(d.frequencies()[0])
    x2, p2 = d.real_points(e, s.Ef)
    chi = gpu.chi0(np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2, precision=precision)
    rpa = gpu.dyson(chi, O.umatrix(s))
    schi, srpa = O.site_reduce(s, chi), O.site_reduce(s, rpa)
    for i in range(1, s.n_atoms + 1):
        for j in range(1, s.n_atoms + 1):
            for kind, sc in (("chihf", schi), ("chi", srpa)):
                f = os.path.join(GOLDEN, "nanoribbon", f"{kind}_{i}_{j}.dat")
                g = [[float(x) for x in l.split()] for l in open(f) if not l.strip().startswith("#")][0]
                r = O.golden_row(s, e, 0.0, sc, i - 1, j - 1)
                for a, b in zip(r, g):
                    if abs(b) > 1e-6:
                        assert abs(a - b) <= 1e-8 * abs(b), (kind, i, j, a, b)


@pytest.mark.parametrize("shape", ["bcc1", "sq2", "bcc4", "slab5"])
def test_eig_batch_matches_eigh(gpu, shape):
    """Jacobi eigendecomposition of H(k) behind the spectral Green functions (at dimH 90 on
    the packed upper triangle of the rotated matrix)."""
    deck = synthetic.make_deck(shape, mesh=False)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.set_system(s)
    gpu.set_h0(h0)
    kp = np.random.default_rng(3).uniform(-2, 2, size=(25, 3))
    lam, U = gpu.eig_batch(kp)
    H = O.Model(s, h0).hk(kp)
    for k in range(kp.shape[0]):
        ref = np.linalg.eigvalsh(H[k])
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(np.sort(lam[k]) - ref)) < 1e-13 * scale * s.dimH
        assert np.max(np.abs(U[k].conj().T @ U[k] - np.eye(s.dimH))) < 1e-13 * s.dimH
        rec = U[k] @ np.diag(lam[k]) @ U[k].conj().T
        assert np.max(np.abs(rec - H[k])) < 1e-14 * scale * s.dimH


@pytest.mark.parametrize("shape,nk,e,q,precision", [
    ("bcc1", (4, 4, 4), 0.0, (0, 0, 0), "fp64"),
    ("bcc1", (3, 3, 3), 0.03, (0.1, 0.0, 0.2), "fp64"),
    ("sq2", (5, 5, 1), 0.1, (0.05, 0.02, 0.0), "fp64"),
    ("sq2", (5, 5, 1), 0.1, (0.0, 0.0, 0.0), "split"),
    ("bcc4", (2, 2, 2), 0.05, (0.0, 0.1, 0.0), "fp64"),
    ("slab5", (3, 3, 1), 0.05, (0.1, 0.0, 0.0), "fp64"),
    ("slab5", (3, 3, 1), 0.05, (0.0, 0.0, 0.0), "split"),
])
def test_spectral_green_equals_gauss_jordan(gpu, shape, nk, e, q, precision):
    """chi0 with G from the eigendecomposition (default on uniform meshes up to dimH 72; at
    dimH 90 the default is the tridiagonalised path and the packed eigendecomposition runs on
    request) and from Gauss-Jordan per point agree to roundoff; both match the oracle."""
    deck = synthetic.make_deck(shape, nk=nk, n1gl=8, parts=1, n3gl=6)
    s, h0 = _setup(gpu, deck)
    x2, p2 = deck.real_points(e, s.Ef)
    q = np.array(q, float)
    try:
        gpu.set_green_method("gauss-jordan")
        gj = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision=precision)
        gpu.set_green_method("spectral")
        forced = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision=precision)
    finally:
        gpu.set_green_method("auto")
    sp = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision=precision)
    assert rel(sp, gj) < (1e-12 if precision == "fp64" else 1e-10)
    assert rel(forced, gj) < (1e-12 if precision == "fp64" else 1e-10)
    ref = O.eintshechi(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), q, e, s.Ef, s.eta, s.etap, x2, p2)
    assert rel(sp, ref) < (1e-10 if precision == "fp64" else 1e-9)


def test_smunu_and_sum_rule_on_fe_golden_state(gpu, fe_deck):
    """calcSmunu on the GPU against the oracle, and the sum rule with the GPU's chi_HF(0, 0)."""
    from titan_b200.host import response as R
    from titan_b200.host import sumrule as SR
    s = fe_deck.system
    st = fe_deck.state
    h0 = s.h0(st)
    gpu.setup(fe_deck, h0)
    S = gpu.smunu(s.Ef, s.eta)
    ref = O.smunu(O.Model(s, h0), fe_deck.ek, s.Ef, s.eta)
    assert np.max(np.abs(S - ref)) < 1e-12 * np.max(np.abs(ref))
    chi = gpu.chi0(np.zeros(3), 0.0, s.Ef, s.eta, s.etap)
    lvec, lpvec, lam_p, lam_d, porbs, dorbs, Um = R.site_parameters(s)
    mvec = [[st.mx[i][dorbs[i]].sum(), st.my[i][dorbs[i]].sum(), st.mz[i][dorbs[i]].sum()] for i in range(s.n_atoms)]
    B = SR.effective_field(s, mvec, lvec, lam_p, lam_d, porbs, dorbs, Um)
    lhs, rhs, diff = SR.check(s, chi, S, B)
    assert diff < 1e-9 * np.abs(lhs).max()


@pytest.mark.parametrize("shape,nk,e,q", [
    ("bcc1", (3, 3, 3), 0.0, (0, 0, 0)),
    ("bcc1", (3, 3, 3), 0.03, (0.1, 0.0, 0.2)),
    ("sq2", (4, 4, 1), 0.05, (0.05, 0.02, 0.0)),
])
def test_chi0_linear_soc_matches_oracle(gpu, shape, nk, e, q):
    """eintshechilinearsoc on the GPU: chi_HF of H0 and the linear-SOC correction vs the oracle."""
    deck = synthetic.make_deck(shape, nk=nk, n1gl=6, parts=1, n3gl=4)
    s = deck.system
    h00, V = s.linear_soc_split(initial_state(s))
    gpu.setup(deck, h00)
    x2, p2 = deck.real_points(e, s.Ef)
    q = np.array(q, float)
    chi, lsoc = gpu.chi0_linear_soc(q, e, s.Ef, s.eta, s.etap, x2, p2, V)
    rchi, rl = O.eintshechi_linear_soc(O.Model(s, h00), V, deck.ek, (deck.real_kp, deck.real_w), q, e, s.Ef, s.eta,
                                       s.etap, x2, p2)
    assert rel(chi, rchi) < 1e-10
    assert rel(lsoc, rl) < 1e-10


def _moment_directions(state, dorbs):
    m = np.array([[state.mx[i][d].sum(), state.my[i][d].sum(), state.mz[i][d].sum()] for i, d in enumerate(dorbs)])
    return m / np.linalg.norm(m, axis=1)[:, None]


@pytest.mark.parametrize("q", [(0.0, 0.0, 0.0), (0.2, 0.1, 0.0)])
def test_jij_on_fe_golden_state(gpu, fe_deck, q):
    """jij_energy on the GPU against the oracle at the golden Fe state, q = 0 and q != 0."""
    s = fe_deck.system
    st = fe_deck.state
    h0 = s.h0(st)
    gpu.setup(fe_deck, h0)
    evec = _moment_directions(st, s.dorbs)
    J = gpu.jij(np.array(q), s.Ef, s.eta, evec, s.Um())
    ref = O.jij(O.Model(s, h0), fe_deck.ek, np.array(q), s.Ef, s.eta, evec, s.Um(), s.dorbs)
    assert np.max(np.abs(J - ref)) < 1e-11 * np.max(np.abs(ref))


def test_jij_two_sites_tilted_moments(gpu):
    """Two-site cell with non-collinear moment directions (all 9 tensor components nonzero)."""
    deck = synthetic.make_deck("sq2", nk=(5, 5, 1), n1gl=6, parts=1)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.setup(deck, h0)
    evec = np.array([[0.0, 0.6, 0.8], [0.6, 0.0, 0.8]])
    q = np.array([0.1, 0.05, 0.0])
    J = gpu.jij(q, s.Ef, s.eta, evec, s.Um())
    ref = O.jij(O.Model(s, h0), deck.ek, q, s.Ef, s.eta, evec, s.Um(), s.dorbs)
    assert np.max(np.abs(J - ref)) < 1e-11 * np.max(np.abs(ref))


def test_spectral_expectation_on_request(gpu, fe_deck):
    """TG_GREEN_SPECTRAL: occupations and moments from one eigendecomposition per k (the energy
    sum folded per eigenvalue, eigenvectors re-orthonormalised, Rayleigh-quotient eigenvalues)
    equal the Gauss-Jordan ones to 1e-12 on the Fe golden state (5.2e-13 measured)."""
    s = fe_deck.system
    st = fe_deck.state
    gpu.setup(fe_deck, s.h0(st))
    gj = gpu.expectation(st.Ef, s.eta)
    try:
        gpu.set_green_method("spectral")
        sp = gpu.expectation(st.Ef, s.eta)
    finally:
        gpu.set_green_method("auto")
    dev = max(np.max(np.abs(a - b)) for a, b in zip(sp, gj))
    assert dev < 1e-12, dev


def test_gs_orbital_matches_oracle_and_fe_golden(gpu, fe_deck):
    """tg_gs_orbital (calc_GS_L_and_E_greenfunction's orbital density) against the oracle, and the
    orbital moment of the golden Fe state against scResult."""
    from titan_b200.host.orbital import calculate_l
    from titan_b200.host.response import site_parameters
    s = fe_deck.system
    h0 = s.h0(fe_deck.state)
    gpu.setup(fe_deck, h0)
    P = gpu.gs_orbital(s.Ef, s.eta)
    ref = O.gs_orbital(O.Model(s, h0), fe_deck.ek, s.Ef, s.eta)
    assert np.max(np.abs(P - ref)) <= 1e-12 * np.max(np.abs(ref))
    lvec, lpvec = site_parameters(s)[:2]
    lz = calculate_l(s, P, lvec, lpvec)[2][0]
    line = [l for l in open(os.path.join(GOLDEN, "Fe_bulk_susc", "scResult")) if "Lz=" in l][0]
    assert abs(lz - float(line.split("Lz=")[1].split()[0])) < 1e-7


def test_gs_orbital_multi_site(gpu):
    deck = synthetic.make_deck("sq2", nk=(5, 5, 1), n1gl=8, parts=1, n3gl=4)
    s, h0 = _setup(gpu, deck)
    P = gpu.gs_orbital(s.Ef, s.eta)
    ref = O.gs_orbital(O.Model(s, h0), deck.ek, s.Ef, s.eta)
    assert np.max(np.abs(P - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_chi0_qbatch_on_an_adaptive_mesh(gpu, precision):
    """tg_chi0_qbatch over three q (q = 0 among them) and two frequencies on a non-uniform
    (E, k) list, where one G2 per pass serves every (q, e): equal to one tg_chi0 call per
    (q, e) and to the oracle."""
    from titan_b200.host.deck import Deck
    base = synthetic.make_deck("bcc1", nk=(4, 4, 4), n1gl=6, parts=1, n3gl=4, mesh=False)
    p = dict(base.params)
    p["nk_per_energy"] = [64, 64, 27, 27, 8, 8]
    deck = Deck.from_system(base.system, p, True)
    s, h0 = _setup(gpu, deck)
    qs = np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.0], [0.05, 0.1, 0.2]])
    es = [0.0, 0.04]
    xs = [deck.real_points(e, s.Ef) for e in es]
    got = gpu.chi0_qbatch(qs, es, s.Ef, s.eta, s.etap, [x[0] for x in xs], [x[1] for x in xs], precision)
    bounds = gpu.error_bound(len(qs) * len(es)).reshape(len(qs), len(es))
    assert np.all(bounds == 0.0) if precision == "fp64" else np.all((bounds > 0.0) & (bounds < 1e-6))
    m = O.Model(s, h0)
    for iq, q in enumerate(qs):
        for w, e in enumerate(es):
            single = gpu.chi0(q, e, s.Ef, s.eta, s.etap, xs[w][0], xs[w][1], precision)
            ref = O.eintshechi(m, deck.ek, (deck.real_kp, deck.real_w), q, e, s.Ef, s.eta, s.etap, xs[w][0],
                               xs[w][1])
            assert rel(got[iq, w], single) < (1e-12 if precision == "fp64" else 1e-9)
            assert rel(got[iq, w], ref) < (1e-10 if precision == "fp64" else 1e-9)
            if precision == "split":   # the bound plus FP64 rounding of the sums
                assert rel(got[iq, w], ref) <= bounds[iq, w] + 1e-11


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_chi0_qbatch_adaptive_slab5_spectral_real_axis(gpu, precision):
    """dimH 90 on an adaptive imaginary axis: tg_chi0_qbatch inverts G2 once per pass for both
    q and takes the real axis from eigendecompositions of H(k) and H(k + q); equal to the
    same call with Gauss-Jordan everywhere and to the oracle."""
    from titan_b200.host.deck import Deck
    base = synthetic.make_deck("slab5", nk=(3, 3, 1), n1gl=4, parts=1, n3gl=4, mesh=False)
    p = dict(base.params)
    p["nk_per_energy"] = [9, 9, 4, 4]
    deck = Deck.from_system(base.system, p, True)
    s, h0 = _setup(gpu, deck)
    qs = np.array([[0.0, 0.0, 0.0], [0.1, 0.05, 0.0]])
    es = [0.03]
    xs = [deck.real_points(e, s.Ef) for e in es]
    x2, p2 = [x[0] for x in xs], [x[1] for x in xs]
    got = gpu.chi0_qbatch(qs, es, s.Ef, s.eta, s.etap, x2, p2, precision)
    try:
        gpu.set_green_method("gauss-jordan")
        gj = gpu.chi0_qbatch(qs, es, s.Ef, s.eta, s.etap, x2, p2, precision)
    finally:
        gpu.set_green_method("auto")
    m = O.Model(s, h0)
    for iq, q in enumerate(qs):
        ref = O.eintshechi(m, deck.ek, (deck.real_kp, deck.real_w), q, es[0], s.Ef, s.eta, s.etap, x2[0], p2[0])
        assert rel(got[iq, 0], gj[iq, 0]) < (1e-12 if precision == "fp64" else 1e-9)
        assert rel(got[iq, 0], ref) < (1e-10 if precision == "fp64" else 1e-9)
