"""The C ABI without a GPU: the library loads, exports every entry point of
include/titan_gpu.h, the ctypes binding declares each of them, and the GPU
context refuses to start without a CUDA device (no CPU fallback)."""
import ctypes
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib_path():
    from titan_b200 import native
    if not os.path.exists(native.LIB_PATH):
        from titan_b200 import build as B
        B.build()
    return native.LIB_PATH


def test_library_exports_every_header_symbol():
    import __graft_entry__ as G
    h = ctypes.CDLL(_lib_path())
    syms = G.header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(h, s)]
    assert not missing, missing


def test_binding_declares_every_header_symbol():
    import __graft_entry__ as G
    from titan_b200 import native
    assert set(G.header_symbols()) <= set(native.SIGNATURES)


def test_context_requires_a_cuda_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    _lib_path()
    from titan_b200.native import GreenGPU, TitanGPUError
    with pytest.raises(TitanGPUError):
        GreenGPU(0)
