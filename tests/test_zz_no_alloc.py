"""tg_expectation_noalloc through the C ABI against tg_expectation (needs a B200).

Collected last (file name), so it runs both alone and after the other GPU tests;
each system is checked on a fresh context with the no-alloc call first (the call
that performs the per-device scratch lookup), twice in a row.
"""
import ctypes as C

import numpy as np
import pytest

from titan_b200.host import synthetic
from titan_b200.host.system import initial_state

pytestmark = pytest.mark.gpu


def _call_noalloc(gpu, Ef, eta):
    nat, nmax = gpu.system.n_atoms, gpu.nmax
    out = [np.zeros((nat, nmax)) for _ in range(4)]
    mp = np.zeros((nat, nmax), np.complex128)
    dp = C.POINTER(C.c_double)
    rc = gpu.lib.tg_expectation_noalloc(gpu.h, Ef, eta, *[o.ctypes.data_as(dp) for o in out],
                                        mp.view(np.float64).ctypes.data_as(dp))
    assert rc == 0, gpu.lib.tg_last_error(gpu.h)
    return out + [mp]


@pytest.mark.parametrize("shape,nk", [("bcc1", (4, 4, 4)), ("sq2", (6, 6, 1))])
def test_noalloc_expectation_matches_tg_expectation(shape, nk):
    from titan_b200.native import GreenGPU
    deck = synthetic.make_deck(shape, nk=nk, n1gl=8, parts=1, n3gl=4)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu = GreenGPU(0)
    try:
        gpu.setup(deck, h0)
        first = _call_noalloc(gpu, s.Ef, s.eta)
        second = _call_noalloc(gpu, s.Ef, s.eta)
        ref = list(gpu.expectation(s.Ef, s.eta))
        for got in (first, second):
            for a, b in zip(got, ref):
                assert np.max(np.abs(a - b)) < 1e-12
    finally:
        gpu.close()


def test_noalloc_ignores_the_spectral_method():
    """Under TG_GREEN_SPECTRAL tg_expectation diagonalises H(k); the no-alloc call still
    inverts per point, so it equals the default (Gauss-Jordan) tg_expectation."""
    from titan_b200.native import GreenGPU
    deck = synthetic.make_deck("sq2", nk=(6, 6, 1), n1gl=8, parts=1, n3gl=4)
    s = deck.system
    h0 = s.h0(initial_state(s))
    gpu = GreenGPU(0)
    try:
        gpu.setup(deck, h0)
        ref = list(gpu.expectation(s.Ef, s.eta))
        gpu.set_green_method("spectral")
        for _ in range(2):
            got = _call_noalloc(gpu, s.Ef, s.eta)
            for a, b in zip(got, ref):
                assert np.max(np.abs(a - b)) < 1e-12
    finally:
        gpu.close()


def test_noalloc_refuses_what_its_fixed_array_cannot_hold():
    """The 16-layer slab (dimH 288) needs the cluster Gauss-Jordan kernel, which keeps its
    Green functions in allocated memory: TG_ERR_ARG with a message, before any work, and
    the context stays usable."""
    from titan_b200.native import GreenGPU, TG_ERR_ARG
    deck = synthetic.make_deck("slab16", nk=(2, 2, 1), n1gl=4, parts=1, n3gl=4)
    s = deck.system
    gpu = GreenGPU(0)
    try:
        gpu.setup(deck, s.h0(initial_state(s)))
        nat, nmax = s.n_atoms, gpu.nmax
        out = [np.zeros((nat, nmax)) for _ in range(4)]
        mp = np.zeros((nat, nmax), np.complex128)
        dp = C.POINTER(C.c_double)
        rc = gpu.lib.tg_expectation_noalloc(gpu.h, s.Ef, s.eta, *[o.ctypes.data_as(dp) for o in out],
                                            mp.view(np.float64).ctypes.data_as(dp))
        assert rc == TG_ERR_ARG
        assert b"dimension" in gpu.lib.tg_last_error(gpu.h)
        green = gpu.green_batch(np.array([s.Ef + 0.1j]), np.zeros((1, 3)))
        assert np.all(np.isfinite(green))
    finally:
        gpu.close()
