"""GPU parity of the transforms and propagators against the FP64 oracle.

Tolerance: 1e-5 relative L2 against the FP64 oracle for every field (the
engine computes in FP32 with an FP64-reduced transfer-function phase).
"""
import math

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5
LAMBDA = 532e-9


def rand_planes(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) - 0.1, rng.standard_normal(n) + 0.2


@pytest.mark.parametrize("nx,ny", [(1, 1), (2, 2), (1, 8), (8, 1), (8, 8), (16, 4), (32, 64), (64, 64),
                                   (128, 256), (256, 256), (512, 128), (1024, 1024), (2048, 64),
                                   (64, 4096), (8192, 2)])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft2d_matches_oracle(engine, oracle, nx, ny, inverse):
    re, im = rand_planes(nx * ny, nx * 31 + ny)
    r, i = re.copy(), im.copy()
    engine.fft2d(r, i, nx, ny, inverse)
    orr, oi = oracle.fft2d(re, im, nx, ny, inverse)
    assert rel_l2(r + 1j * i, orr + 1j * oi) < TOL


def test_fft2d_matches_naive_dft(engine, oracle):
    re, im = rand_planes(64, 5)
    nr, ni = oracle.dft2d_naive(re, im, 8, 8)
    r, i = re.copy(), im.copy()
    engine.fft2d(r, i, 8, 8)
    assert rel_l2(r + 1j * i, nr + 1j * ni) < TOL
    engine.fft2d(r, i, 8, 8, True)
    assert rel_l2(r + 1j * i, re + 1j * im) < TOL


def test_fft2d_delta_is_flat(engine):
    re = np.zeros(32 * 32)
    im = np.zeros(32 * 32)
    re[0] = 1
    engine.fft2d(re, im, 32, 32)
    assert np.abs(np.hypot(re, im) - 1).max() < 1e-6


@pytest.mark.parametrize("n,dx,z,bl,ev,se", [
    (64, 8e-6, 25e-3, False, True, 0.02),
    (64, 8e-6, -25e-3, False, True, 0.02),
    (256, 8e-6, 30e-3, True, True, 0.02),
    (256, 8e-6, 30e-3, False, True, 0.02),
    (128, 8e-6, 0.05, True, True, 0.01),
    (1024, 4e-6, 48e-3, True, True, 0.02),
    (512, 0.3e-6, 2e-3, False, True, 0.02),   # evanescent band present
    (128, 0.2e-6, 1e-4, False, False, 0.02),  # evanescent kept (propagating correction)
    (32, 8e-6, 30e-3, True, True, 0.0),
])
def test_asm_matches_oracle(engine, oracle, n, dx, z, bl, ev, se):
    re, im = rand_planes(n * n, n + int(abs(z) * 1e6))
    f = engine.ComplexField(n, n, dx, dx)
    f.re[:], f.im[:] = re, im
    out = engine.propagateAngularSpectrum(f, LAMBDA, z, {"bandLimit": bl, "evanescent": ev, "softEdge": se})
    orr, oi = oracle.asm(re, im, n, n, dx, dx, LAMBDA, z, bl, ev, se)
    assert rel_l2(out.re + 1j * out.im, orr + 1j * oi) < TOL
    assert np.array_equal(f.re, re) and np.array_equal(f.im, im)  # clone semantics


@pytest.mark.parametrize("nx,ny,dx,dy", [(256, 64, 8e-6, 6e-6), (16, 1024, 4e-6, 4e-6), (1, 64, 8e-6, 8e-6),
                                         (128, 1, 8e-6, 8e-6), (1, 1, 8e-6, 8e-6)])
def test_asm_rectangular_grid(engine, oracle, nx, ny, dx, dy):
    re, im = rand_planes(nx * ny, 7)
    f = engine.ComplexField(nx, ny, dx, dy)
    f.re[:], f.im[:] = re, im
    engine.propagateAngularSpectrumInPlace(f, 633e-9, 0.02)
    orr, oi = oracle.asm(re, im, nx, ny, dx, dy, 633e-9, 0.02, True, True, 0.02)
    assert rel_l2(f.re + 1j * f.im, orr + 1j * oi) < TOL


def test_asm_zero_distance_is_identity(engine):
    re, im = rand_planes(64 * 64, 3)
    f = engine.ComplexField(64, 64, 8e-6)
    f.re[:], f.im[:] = re, im
    engine.propagateAngularSpectrumInPlace(f, LAMBDA, 0.0)
    assert np.array_equal(f.re, re) and np.array_equal(f.im, im)


def test_asm_unitary_round_trip(engine):
    n, dx, z = 64, 8e-6, 25e-3
    re, im = rand_planes(n * n, 11)
    f = engine.ComplexField(n, n, dx)
    f.re[:], f.im[:] = re, im
    fwd = engine.propagateAngularSpectrum(f, LAMBDA, z, {"bandLimit": False})
    back = engine.propagateAngularSpectrum(fwd, LAMBDA, -z, {"bandLimit": False})
    assert rel_l2(back.re + 1j * back.im, re + 1j * im) < TOL
    assert abs(fwd.power() / f.power() - 1) < 1e-6


@pytest.mark.parametrize("n,dx,z,bl,ev", [(128, 8e-6, 0.05, True, True), (64, 0.3e-6, 1e-3, False, True),
                                          (64, 0.2e-6, 1e-4, False, False), (256, 4e-6, 0.015, True, True)])
def test_transfer_function_matches_oracle(engine, oracle, n, dx, z, bl, ev):
    H = engine.angularSpectrumTransferFunction(n, n, dx, dx, LAMBDA, z, {"bandLimit": bl, "evanescent": ev})
    hr, hi, frac = oracle.asm_transfer(n, n, dx, dx, LAMBDA, z, bl, ev, 0.02)
    assert rel_l2(H["re"] + 1j * H["im"], hr + 1j * hi) < TOL
    assert H["propagatingFraction"] == frac


@pytest.mark.parametrize("n,f", [(64, 0.03), (256, 0.12), (1024, 0.02)])
def test_focal_plane_matches_oracle(engine, oracle, n, f):
    dx = 8e-6
    re, im = rand_planes(n * n, n)
    fld = engine.ComplexField(n, n, dx)
    fld.re[:], fld.im[:] = re, im
    out = engine.focalPlaneSpectrum(fld, LAMBDA, f)
    orr, oi, odx, ody = oracle.focal_plane(re, im, n, n, dx, dx, LAMBDA, f)
    assert rel_l2(out.re + 1j * out.im, orr + 1j * oi) < TOL
    assert out.dx == odx and out.dy == ody
    assert abs(out.power() / fld.power() - 1) < 1e-6


def test_focus_sweep_matches_oracle(engine, oracle):
    n, dx = 128, 8e-6
    re, im = rand_planes(n * n, 99)
    f = engine.ComplexField(n, n, dx)
    f.re[:], f.im[:] = re, im
    planes = engine.focusSweep(f, LAMBDA, 0.0, 0.04, 4)
    assert [p["z"] for p in planes] == [0.0, 0.01, 0.02, 0.03, 0.04]
    assert np.array_equal(planes[0]["field"].re, re)  # z == 0 leaves the field untouched
    for p in planes[1:]:
        orr, oi = oracle.asm(re, im, n, n, dx, dx, LAMBDA, p["z"], True, True, 0.02)
        assert rel_l2(p["field"].re + 1j * p["field"].im, orr + 1j * oi) < TOL


def test_device_sweep_matches_oracle(engine, oracle):
    """Device-resident batched sweep (complex64 in HBM), several fields and distances."""
    import torch
    nx = ny = 256
    dx = 4e-6
    nf, nz = 3, 5
    rng = np.random.default_rng(4)
    fields = (rng.standard_normal((nf, ny, nx)) + 1j * rng.standard_normal((nf, ny, nx))).astype(np.complex64)
    lam = np.array([450e-9, 532e-9, 633e-9])
    z = rng.uniform(15e-3, 48e-3, nf * nz)
    z[3] = 0.0
    d_in = torch.from_numpy(fields).cuda()
    d_out = torch.empty((nf * nz, ny, nx), dtype=torch.complex64, device="cuda")
    c = engine.context()
    c.check(c.lib.doe_asm_sweep_dev(c.h, d_in.data_ptr(), nf, nx, ny, dx, dx, lam.ctypes.data_as(
        __import__("ctypes").POINTER(__import__("ctypes").c_double)), z.ctypes.data_as(
        __import__("ctypes").POINTER(__import__("ctypes").c_double)), nz, 1, 1, 0.02, d_out.data_ptr()))
    c.synchronize()
    out = d_out.cpu().numpy()
    for f in range(nf):
        src = fields[f].astype(np.complex128).ravel()
        for k in range(nz):
            g = f * nz + k
            if z[g] == 0.0:
                assert np.array_equal(out[g], fields[f])
                continue
            orr, oi = oracle.asm(src.real.copy(), src.imag.copy(), nx, ny, dx, dx, lam[f], z[g], True, True, 0.02)
            assert rel_l2(out[g].ravel(), orr + 1j * oi) < TOL


def test_errors_use_reference_wording(engine):
    from diffractiveopticalelement_b200 import DOEError
    c = engine.context()
    re = np.zeros(12)
    with pytest.raises(DOEError, match="power-of-two"):
        c.check(c.lib.doe_fft2d(c.h, re.ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_double)),
                                re.ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_double)),
                                3, 4, 0))
    with pytest.raises(DOEError, match="not supported"):
        c.check(c.lib.doe_fft2d(c.h, None, None, 16384, 1, 0))


# ------------------------------------------------------------------ single-FFT Fresnel
def gaussian_phase_field(engine, nx, ny, d, seed):
    rng = np.random.default_rng(seed)
    i = (np.arange(nx) - nx / 2) * d
    j = (np.arange(ny) - ny / 2) * d
    X, Y = np.meshgrid(i, j)
    w = 0.2 * nx * d
    amp = np.exp(-(X ** 2 + Y ** 2) / w ** 2)
    ph = 3.0 * rng.standard_normal() * (X / (nx * d)) + 5.0 * (X ** 2 + Y ** 2) / (nx * d) ** 2
    f = engine.ComplexField(nx, ny, d, d)
    f.re = (amp * np.cos(ph)).ravel().copy()
    f.im = (amp * np.sin(ph)).ravel().copy()
    return f


@pytest.mark.parametrize("nx,ny,z", [(64, 64, 0.05), (256, 256, 0.03), (128, 64, 0.2), (512, 512, -0.04),
                                     (32, 128, 0.01)])
def test_fresnel_matches_oracle(engine, oracle, nx, ny, z):
    d = 8e-6
    f = gaussian_phase_field(engine, nx, ny, d, nx + ny)
    r = engine.propagateFresnelFFT(f, LAMBDA, z)
    orr, oi, dux, duy = oracle.fresnel(f.re, f.im, nx, ny, d, d, LAMBDA, z)
    assert rel_l2(r["field"].re + 1j * r["field"].im, orr + 1j * oi) < TOL
    assert r["dx"] == pytest.approx(dux, rel=1e-15) and r["dy"] == pytest.approx(duy, rel=1e-15)
    assert r["zCritical"] == pytest.approx(nx * d * d / LAMBDA)
    assert r["undersampled"] == (abs(z) < r["zCritical"])
    b = engine.propagateFresnelFFTInverse(r["field"], LAMBDA, z, {"dx": d, "dy": d})
    br, bi = oracle.fresnel_inverse(orr, oi, nx, ny, dux, duy, LAMBDA, z, d, d)
    assert rel_l2(b.re + 1j * b.im, br + 1j * bi) < TOL
    # round trip (test/propagate.test.js:137-146)
    assert rel_l2(b.re + 1j * b.im, f.re + 1j * f.im) < TOL


def test_fresnel_argument_errors(engine):
    f = engine.ComplexField(64, 64, 8e-6, 8e-6)
    with pytest.raises(ValueError, match="under-sampled"):
        engine.propagateFresnelFFT(f, LAMBDA, 1e-4, {"throwOnUndersampled": True})
    with pytest.raises(ValueError, match="DOE-plane pitch"):
        engine.propagateFresnelFFTInverse(f, LAMBDA, 0.05, {})
    from diffractiveopticalelement_b200 import DOEError
    with pytest.raises(DOEError, match="non-zero"):
        engine.propagateFresnelFFT(f, LAMBDA, 0.0)
    g = engine.propagate(gaussian_phase_field(engine, 64, 64, 8e-6, 1), LAMBDA, 0.05, {"method": "fresnel"})
    assert g.dx == pytest.approx(LAMBDA * 0.05 / (64 * 8e-6))


def test_repeated_device_sweep_replays_graph_bitwise(engine):
    """A device sweep repeated with identical arguments is captured into a CUDA graph
    on its second call and replayed afterwards; every call gives the same planes."""
    import ctypes as C
    import torch
    ctx = engine.Context(0)
    L = ctx.lib
    n, nf, nz = 128, 3, 10
    rng = np.random.default_rng(3)
    fields = torch.tensor((rng.standard_normal((nf, n, n)) + 1j * rng.standard_normal((nf, n, n))).astype(np.complex64),
                          device="cuda")
    lam = np.array([450e-9, 532e-9, 633e-9])
    zs = np.linspace(0.01, 0.05, nf * nz)
    dp = C.POINTER(C.c_double)
    outs = []
    for graph in (0, 1, 1, 1, 1):
        ctx.check(L.doe_ctx_set_tuning(ctx.h, b"sweep_graph", graph))
        ctx.check(L.doe_ctx_set_tuning(ctx.h, b"sweep_group", 4))
        out = torch.zeros((nf * nz, n, n), dtype=torch.complex64, device="cuda")
        for _ in range(3 if graph else 1):
            out.zero_()
            ctx.check(L.doe_asm_sweep_dev(ctx.h, fields.data_ptr(), nf, n, n, 4e-6, 4e-6, lam.ctypes.data_as(dp),
                                          zs.ctypes.data_as(dp), nz, 1, 1, 0.02, out.data_ptr()))
        ctx.synchronize()
        outs.append(out.cpu())
    for o in outs[1:]:
        assert torch.equal(o, outs[0])
    ctx.close()
