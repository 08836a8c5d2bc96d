"""The pivot reciprocal of the Gauss-Jordan kernels and the FP64 peak probe (needs a B200)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rcp_newton_within_two_ulp_of_the_correctly_rounded_reciprocal():
    """rcp.approx.ftz.f64 plus three Newton-Raphson steps against numpy's 1/s (IEEE division,
    correctly rounded) over the range the pivots' |a|^2 take (1e-150 .. 1e150)."""
    from titan_b200.native import load_library
    lib = load_library()
    rng = np.random.default_rng(11)
    s = np.concatenate([10.0 ** rng.uniform(-150, 150, 200000), [1.0, 2.0, 3.0, 0.1, 1e-150, 1e150],
                        np.nextafter(1.0, 2.0) + np.arange(64) * 2.0 ** -52])
    r = np.empty_like(s)
    dp = C.POINTER(C.c_double)
    assert lib.tg_rcp_check(s.size, s.ctypes.data_as(dp), r.ctypes.data_as(dp)) == 0
    ref = 1.0 / s
    ulp = np.abs(r - ref) / np.spacing(ref)
    assert ulp.max() <= 2.0, ulp.max()


def test_fp64_peak_is_measured():
    from titan_b200.native import fp64_peak
    fma, mma = fp64_peak()
    # B200: 37 TFLOP/s nominal FP64; a working probe lands within a factor of two of it
    assert 10.0 < fma < 80.0 and 10.0 < mma < 80.0, (fma, mma)
