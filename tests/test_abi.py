"""C-ABI checks that need no GPU: the library loads and exports every declared symbol."""
import ctypes
import os

import pytest


def test_library_exports_every_declared_symbol(engine):
    from diffractiveopticalelement_b200 import _lib
    L = _lib.load_library()
    names = _lib.declared_functions()
    assert "doe_fft2d" in names and "doe_asm" in names and "doe_last_error" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"declared in include/doe_b200.h but not exported: {missing}"


def test_abi_version(engine):
    from diffractiveopticalelement_b200 import _lib
    assert _lib.load_library().doe_abi_version() == 1


def test_ctx_create_rejects_bad_arguments(engine):
    from diffractiveopticalelement_b200 import _lib
    L = _lib.load_library()
    assert L.doe_ctx_create(0, None) == _lib.DOE_ERR_BAD_ARG
    # without a GPU the context cannot be created; with one, device -1 is invalid
    h = ctypes.c_void_p()
    rc = L.doe_ctx_create(-1, ctypes.byref(h))
    assert rc in (_lib.DOE_ERR_BAD_ARG, _lib.DOE_ERR_NO_DEVICE)


def test_no_cpu_fallback_without_gpu(engine):
    """On a machine without a CUDA device the API refuses instead of computing on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import numpy as np
    from diffractiveopticalelement_b200 import EngineUnavailable, _lib
    _lib._ctx.clear()
    with pytest.raises(EngineUnavailable):
        engine.fft2d(np.zeros(16), np.zeros(16), 4, 4)


def test_input_validation_matches_reference_messages(engine):
    import numpy as np
    with pytest.raises(ValueError, match="grid must be power-of-two"):
        engine.ComplexField(6, 8)
    with pytest.raises(ValueError, match="does not match"):
        engine.fft2d(np.zeros(15), np.zeros(16), 4, 4)
