"""The allocation-free propagation entry point (doe_asm_c64_noalloc).

It exists for callers that may not allocate device memory themselves -- for
instance a host runtime that owns all device allocations through its own pool,
or a latency-critical loop that cannot afford the allocator's implicit
synchronisation. It runs the same angular-spectrum propagation as doe_asm using
a fixed scratch array compiled into the library, so its results must match the
ordinary entry point's, and the FP64 oracle's, within the tolerance every other
GPU test uses, on consecutive calls that reuse that scratch: at the scratch limit
(512 x 512 samples), in place (input and output the same plane), on one-row and
one-column grids and at z = 0; and a warm call must leave the device's free
memory unchanged.

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


def _reference(engine, u, nx, ny, dx, dy, lam, z, bl, ev, se):
    f = engine.ComplexField(nx, ny, dx, dy)
    f.re[:] = u.real.ravel().astype(np.float64)
    f.im[:] = u.imag.ravel().astype(np.float64)
    ref = engine.propagateAngularSpectrum(f, lam, z, {"bandLimit": bool(bl), "evanescent": bool(ev), "softEdge": se})
    return ref.re + 1j * ref.im


CASES = [
    (256, 256, 8e-6, 8e-6, 532e-9, 0.03, 1, 1, 0.02),
    (512, 128, 6e-6, 8e-6, 633e-9, -0.02, 0, 1, 0.02),
    (512, 512, 8e-6, 8e-6, 450e-9, 0.045, 1, 1, 0.01),   # exactly the scratch limit
    (4096, 1, 4e-6, 4e-6, 532e-9, 0.01, 1, 1, 0.02),     # one row
    (1, 2048, 4e-6, 4e-6, 532e-9, 0.01, 0, 0, 0.02),     # one column, evanescent band kept
]


def test_noalloc_matches_doe_asm_and_oracle_on_consecutive_calls(engine, oracle):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(123)
    for nx, ny, dx, dy, lam, z, bl, ev, se in CASES:
        u = (rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx))).astype(np.complex64)
        ref = _reference(engine, u, nx, ny, dx, dy, lam, z, bl, ev, se)
        src = u.astype(np.complex128).ravel()
        orr, oi = oracle.asm(src.real.copy(), src.imag.copy(), nx, ny, dx, dy, lam, z, bool(bl), bool(ev), se)
        d_in = torch.from_numpy(u).cuda()
        for inplace in (False, True):  # two calls in a row on the shared scratch; the second in place
            d_out = d_in.clone() if inplace else torch.empty_like(d_in)
            rc, msg = _noalloc(engine, d_out.data_ptr() if inplace else d_in.data_ptr(), d_out.data_ptr(), nx, ny,
                               dx, dy, lam, z, bl, ev, se, stream)
            assert rc == 0, msg
            torch.cuda.synchronize()
            out = d_out.cpu().numpy().ravel()
            assert rel_l2(out, ref) < TOL, (nx, ny, inplace)
            assert rel_l2(out, orr + 1j * oi) < TOL, (nx, ny, inplace)


def test_noalloc_zero_distance_is_the_field_itself(engine):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    u = (np.arange(64 * 32) * (1 + 0.5j)).astype(np.complex64).reshape(32, 64)
    d_in = torch.from_numpy(u).cuda()
    d_out = torch.zeros_like(d_in)
    assert _noalloc(engine, d_in.data_ptr(), d_out.data_ptr(), 64, 32, 8e-6, 8e-6, 532e-9, 0.0, 1, 1, 0.02,
                    stream)[0] == 0
    rc, _ = _noalloc(engine, d_in.data_ptr(), d_in.data_ptr(), 64, 32, 8e-6, 8e-6, 532e-9, 0.0, 1, 1, 0.02, stream)
    torch.cuda.synchronize()
    assert rc == 0
    assert np.array_equal(d_out.cpu().numpy(), u) and np.array_equal(d_in.cpu().numpy(), u)


def test_noalloc_warm_calls_leave_device_memory_unchanged(engine):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    n = 512
    u = np.ones((n, n), np.complex64)
    d_in = torch.from_numpy(u).cuda()
    d_out = torch.empty_like(d_in)
    args = (d_in.data_ptr(), d_out.data_ptr(), n, n, 8e-6, 8e-6, 532e-9, 0.03, 1, 1, 0.02, stream)
    assert _noalloc(engine, *args)[0] == 0  # first use on this device: set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _noalloc(engine, *args)[0] == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_grids_beyond_its_scratch(engine):
    rc, msg = _noalloc(engine, 1, 1, 1024, 1024, 8e-6, 8e-6, 532e-9, 0.03, 1, 1, 0.02, None)
    assert rc == 6 and "scratch limit" in msg  # DOE_ERR_UNSUPPORTED
    rc, msg = _noalloc(engine, 1, 1, 1024, 512, 8e-6, 8e-6, 532e-9, 0.03, 1, 1, 0.02, None)
    assert rc == 6 and "scratch limit" in msg  # one sample beyond the limit in each direction of 512^2
    rc, msg = _noalloc(engine, 1, 1, 100, 64, 8e-6, 8e-6, 532e-9, 0.03, 1, 1, 0.02, None)
    assert rc == 1 and "power-of-two" in msg  # DOE_ERR_NOT_POW2
