"""The allocation-free propagation entry point (doe_asm_c64_noalloc).

It exists for callers that may not allocate device memory themselves -- for
instance a host runtime that owns all device allocations through its own pool,
or a latency-critical loop that cannot afford the allocator's implicit
synchronisation. It runs the same angular-spectrum propagation as doe_asm using
a fixed scratch array compiled into the library, so its results must match the
ordinary entry point's within the tolerance every other GPU test uses, on
consecutive calls that reuse that scratch.

This file is named to be collected last, so that a failure here never hides the
rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _noalloc(engine, d_in, d_out, nx, ny, dx, dy, lam, z, bl, ev, se, stream):
    from diffractiveopticalelement_b200 import _lib
    L = _lib.load_library()
    err = ctypes.create_string_buffer(512)
    rc = L.doe_asm_c64_noalloc(d_in, d_out, nx, ny, dx, dy, lam, z, bl, ev, se, stream, err, 512)
    return rc, err.value.decode()


def test_noalloc_matches_doe_asm_on_consecutive_calls(engine):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    cases = [
        (256, 256, 8e-6, 8e-6, 532e-9, 0.03, 1, 1, 0.02),
        (512, 128, 6e-6, 8e-6, 633e-9, -0.02, 0, 1, 0.02),
        (256, 256, 8e-6, 8e-6, 450e-9, 0.045, 1, 1, 0.01),
    ]
    rng = np.random.default_rng(123)
    for nx, ny, dx, dy, lam, z, bl, ev, se in cases:
        u = (rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx))).astype(np.complex64)
        # existing entry point (doe_asm) on the same complex64 values held in FP64
        f = engine.ComplexField(nx, ny, dx, dy)
        f.re[:] = u.real.ravel().astype(np.float64)
        f.im[:] = u.imag.ravel().astype(np.float64)
        ref = engine.propagateAngularSpectrum(f, lam, z, {"bandLimit": bool(bl), "evanescent": bool(ev),
                                                          "softEdge": se})
        d_in = torch.from_numpy(u).cuda()
        d_out = torch.empty_like(d_in)
        rc, msg = _noalloc(engine, d_in.data_ptr(), d_out.data_ptr(), nx, ny, dx, dy, lam, z, bl, ev, se, stream)
        assert rc == 0, msg
        torch.cuda.synchronize()
        out = d_out.cpu().numpy().ravel()
        assert rel_l2(out, ref.re + 1j * ref.im) < TOL


def test_noalloc_rejects_grids_beyond_its_scratch(engine):
    rc, msg = _noalloc(engine, 1, 1, 1024, 1024, 8e-6, 8e-6, 532e-9, 0.03, 1, 1, 0.02, None)
    assert rc == 6 and "scratch limit" in msg  # DOE_ERR_UNSUPPORTED
    rc, msg = _noalloc(engine, 1, 1, 100, 64, 8e-6, 8e-6, 532e-9, 0.03, 1, 1, 0.02, None)
    assert rc == 1 and "power-of-two" in msg  # DOE_ERR_NOT_POW2
