"""Edge cases of the C ABI on the GPU: argument and call-order errors, an empty
imaginary-axis mesh, and chi0 calls that span several passes.

Errors follow the reference's invers/LAPACK convention plus negative codes for
argument (TG_ERR_ARG), call-order (TG_ERR_STATE) and CUDA problems; every one is
a return status, never a device fault.  Passes: tg_chi0_batch walks the (E, k)
list in passes of at most 6 GiB of FP64 operands (310 656 points at dimH = 36),
so a 200 x 200 k mesh with 9 energies takes two passes whose boundary falls
inside the energies of one k; the result must equal the sum over two mesh shares
that each fit in one pass.
"""
import numpy as np
import pytest

from titan_b200.host import synthetic
from titan_b200.host.mesh import EKMesh
from titan_b200.host.system import initial_state
from titan_b200.native import TG_ERR_ARG, TG_ERR_STATE, TitanGPUError, _p

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from titan_b200.native import GreenGPU
    g = GreenGPU(0)
    yield g
    g.close()


def _setup(gpu, deck):
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu.setup(deck, h0)
    return s, h0


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_argument_and_call_order_errors():
    from titan_b200.native import GreenGPU
    g = GreenGPU(0)
    try:
        deck = synthetic.make_deck("bcc1", nk=(3, 3, 3), n1gl=4, parts=1, n3gl=4)
        s = deck.system
        # chi0 and the occupations before the system is set: call-order errors
        rc = g.lib.tg_chi0(g.h, _p(np.zeros(3)), 0.0, s.Ef, s.eta, s.etap, 0, None, None, 0, 72,
                           _p(np.zeros(2 * 72 * 72)))
        assert rc == TG_ERR_STATE
        buf = [np.zeros(64) for _ in range(5)]
        assert g.lib.tg_expectation(g.h, s.Ef, s.eta, *[_p(b) for b in buf]) == TG_ERR_STATE
        with pytest.raises(TitanGPUError) as ex:
            g._check(g.lib.tg_expectation(g.h, s.Ef, s.eta, *[_p(b) for b in buf]))
        assert ex.value.code == TG_ERR_STATE and "set" in str(ex.value).lower()
        g.setup(deck, s.h0(initial_state(s)))
        D = g.dimens
        out = np.zeros(2 * D * D)
        q = np.zeros(3)
        # unknown precision, wrong dimens, null output
        assert g.lib.tg_chi0(g.h, _p(q), 0.0, s.Ef, s.eta, s.etap, 0, None, None, 7, D, _p(out)) == TG_ERR_ARG
        assert g.lib.tg_chi0(g.h, _p(q), 0.0, s.Ef, s.eta, s.etap, 0, None, None, 0, D + 1, _p(out)) == TG_ERR_ARG
        assert g.lib.tg_chi0(g.h, _p(q), 0.0, s.Ef, s.eta, s.etap, 0, None, None, 0, D, None) == TG_ERR_ARG
        # omega != 0 needs real-axis points
        assert g.lib.tg_chi0(g.h, _p(q), 0.05, s.Ef, s.eta, s.etap, 0, None, None, 0, D, _p(out)) == TG_ERR_ARG
        # a negative mesh size
        assert g.lib.tg_set_real_mesh(g.h, -1, None, None) == TG_ERR_ARG
        assert g.lib.tg_last_error(g.h)
        # the context still works after the errors
        chi = g.chi0(q, 0.0, s.Ef, s.eta, s.etap, precision="fp64")
        assert np.isfinite(chi).all() and np.abs(chi).max() > 0
    finally:
        g.close()


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_empty_imaginary_mesh_gives_zero(gpu, precision):
    deck = synthetic.make_deck("sq2", nk=(4, 4, 1), n1gl=4, parts=1, n3gl=4)
    s, _ = _setup(gpu, deck)
    ek = deck.ek
    gpu.set_imag_mesh(EKMesh(ek.y, ek.wght, ek.energy_index[:0], ek.kp[:0], ek.weight[:0]))
    chi = gpu.chi0(np.zeros(3), 0.0, s.Ef, s.eta, s.etap, precision=precision)
    assert chi.shape == (s.dimens, s.dimens)
    assert np.all(chi == 0)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("split", 1e-9)])
def test_two_pass_chi0_equals_single_pass_shards(gpu, precision, tol):
    from titan_b200.host.sharding import shard_imag_mesh, shard_real_bz
    deck = synthetic.make_deck("sq2", nk=(200, 200, 1), n1gl=9, parts=1, n3gl=2)
    s, _ = _setup(gpu, deck)
    n = deck.ek.n_points
    per_pass = (6 << 30) // (s.dimH * s.dimH * 16) // 64 * 64
    assert per_pass < n < 2 * per_pass and per_pass % 9 != 0   # two passes, boundary inside a k
    e = 0.05
    x2, p2 = deck.real_points(e, s.Ef)
    q = np.array([0.01, 0.0, 0.0])
    full = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision=precision)
    parts = []
    for r in range(2):
        gpu.set_imag_mesh(shard_imag_mesh(deck.ek, r, 2))
        gpu.set_real_mesh(*shard_real_bz(deck.real_kp, deck.real_w, r, 2))
        parts.append(gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision=precision))
    assert rel(parts[0] + parts[1], full) < tol
    if precision == "split":
        gpu.setup(deck, s.h0(initial_state(s)))
        ref = gpu.chi0(q, e, s.Ef, s.eta, s.etap, x2, p2, precision="fp64")
        assert rel(full, ref) < 1e-9
