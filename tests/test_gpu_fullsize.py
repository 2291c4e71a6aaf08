"""Parity at the benchmark sizes: the 1024^2 band-limited focus sweep and the
4 x 2048^2 three-plane design.

The FP64 oracle is too slow for whole benchmark steps, so these tests combine a
few oracle spot checks at full size with size-independent properties over the rest:
agreement of two independent engine paths (the batched sweep against one
propagation per distance), linearity of the sweep in the field, the z / -z round
trip, and batch == single for the multi-plane designs. Tolerances: 1e-5 relative
L2 against the oracle per propagation (as every GPU parity test), 3e-5 for one
multi-plane iteration (six chained propagations), 1e-6 between engine paths.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
LAMBDA = 532e-9


def smooth_field(n, dx, seed):
    """Gaussian beam with a smooth low-order phase screen (the sweep workload's kind of input)."""
    rng = np.random.default_rng(seed)
    x = (np.arange(n) - n / 2) * dx
    X, Y = np.meshgrid(x, x)
    R = 0.5 * n * dx
    w = rng.uniform(0.2, 0.8) * 1e-3
    u, v = X / R, Y / R
    ph = sum(rng.normal() * rng.uniform(0, 1.5) * t for t in (u, v, u * u + v * v, u * v, u * u - v * v,
                                                                u ** 3, v ** 3))
    f = np.exp(-(X ** 2 + Y ** 2) / w ** 2) * np.exp(1j * ph)
    return f.astype(np.complex64)


def dev_sweep(engine, ctx, fields, lam, zs, n, dx):
    import torch
    nf, nz = fields.shape[0], zs.size // fields.shape[0]
    d_in = torch.from_numpy(np.ascontiguousarray(fields)).cuda()
    out = torch.empty((nf * nz, n, n), dtype=torch.complex64, device="cuda")
    dp = C.POINTER(C.c_double)
    ctx.check(ctx.lib.doe_asm_sweep_dev(ctx.h, d_in.data_ptr(), nf, n, n, dx, dx,
                                        np.ascontiguousarray(lam, dtype=np.float64).ctypes.data_as(dp),
                                        np.ascontiguousarray(zs, dtype=np.float64).ctypes.data_as(dp), nz, 1, 1, 0.02,
                                        out.data_ptr()))
    ctx.synchronize()
    return out.cpu().numpy()


def test_full_size_sweep_against_oracle_and_single_propagations(engine, oracle):
    n, dx, nz = 1024, 4e-6, 64
    ctx = engine.context()
    f = smooth_field(n, dx, 3)
    rng = np.random.default_rng(5)
    zs = rng.uniform(15e-3, 48e-3, nz)
    out = dev_sweep(engine, ctx, f[None], np.array([LAMBDA]), zs, n, dx)
    src = f.astype(np.complex128).ravel()
    for k in (0, 41):  # oracle spot checks (FP64, ~0.5 s each)
        orr, oi = oracle.asm(src.real.copy(), src.imag.copy(), n, n, dx, dx, LAMBDA, zs[k], True, True, 0.02)
        assert rel_l2(out[k].ravel(), orr + 1j * oi) < 1e-5
    g = engine.ComplexField(n, n, dx)
    for k in range(0, nz, 7):  # the single-propagation path (other kernels) agrees plane by plane
        g.re[:], g.im[:] = src.real, src.imag
        engine.propagateAngularSpectrumInPlace(g, LAMBDA, zs[k])
        assert rel_l2(out[k].ravel(), g.re + 1j * g.im) < 1e-6


def test_full_size_sweep_is_linear_and_round_trips(engine):
    n, dx, nz = 1024, 4e-6, 16
    ctx = engine.context()
    f1, f2 = smooth_field(n, dx, 11), smooth_field(n, dx, 12)
    a, b = 0.7 - 0.2j, -1.3 + 0.4j
    f3 = (a * f1.astype(np.complex128) + b * f2.astype(np.complex128)).astype(np.complex64)
    zs = np.tile(np.linspace(15e-3, 48e-3, nz), 3)
    out = dev_sweep(engine, ctx, np.stack([f1, f2, f3]), np.full(3, LAMBDA), zs, n, dx)
    lin = a * out[:nz].astype(np.complex128) + b * out[nz:2 * nz].astype(np.complex128)
    for k in range(nz):
        assert rel_l2(out[2 * nz + k].ravel(), lin[k].ravel()) < 1e-6
    # z then -z without the band limit returns the field (the Gaussian has no evanescent content)
    g = engine.ComplexField(n, n, dx)
    g.re[:], g.im[:] = f1.real.ravel(), f1.imag.ravel()
    h = engine.propagateAngularSpectrum(g, LAMBDA, 0.03, bandLimit=False)
    back = engine.propagateAngularSpectrum(h, LAMBDA, -0.03, bandLimit=False)
    assert rel_l2(back.re + 1j * back.im, g.re + 1j * g.im) < 1e-5
    assert abs(h.power() / g.power() - 1) < 1e-5


def test_full_size_multiplane_design(engine, oracle):
    """4 x 2048^2, planes at 25/30/35 mm: one iteration against the oracle, and the
    batched device loop equal to the single-design host call, bitwise."""
    import torch
    from diffractiveopticalelement_b200 import batch
    n, dx, zs, B = 2048, 8e-6, [0.025, 0.03, 0.035], 4
    ill = oracle.disc_mask(n, n, dx, dx, 0.45 * n * dx, 2 * dx)
    i = np.arange(n)
    X, Y = np.meshgrid(i, i)

    def rect(d, p):
        w = 100 + 40 * p + 20 * d
        return ((np.abs(X - n / 2 - 50 * (p - 1)) < w) & (np.abs(Y - n / 2 + 30 * d) < w // 2)).astype(np.float64).ravel()

    tg = np.array([[oracle.prepare_target(rect(d, p), ill) for p in range(3)] for d in range(B)])
    ph = np.array([oracle.random_phase(n, n, 80 + d) for d in range(B)])
    # one iteration of design 0 against the FP64 oracle (6 full-size propagations on the CPU)
    g1 = engine.gerchbergSaxtonMultiPlane(ill, [{"z": zs[p], "targetAmp": tg[0, p]} for p in range(3)],
                                          {"nx": n, "dx": dx, "lambda": LAMBDA, "iterations": 1, "initPhase": ph[0]})
    o1 = oracle.multiplane(ill, zs, list(tg[0]), None, None, nx=n, ny=n, dx=dx, lam=LAMBDA, iterations=1,
                           init_phase=ph[0])
    # one iteration chains six 2048^2 propagations (three planes, forward and back), each
    # within a few 1e-6 of the FP64 oracle; their errors add up to the bound used here
    assert rel_l2(ill * np.exp(1j * g1["phase"]), ill * np.exp(1j * o1["phase"])) < 3e-5
    assert np.allclose(np.array(g1["perPlaneError"]), o1["perPlaneError"], rtol=1e-4)
    # the batched device loop (the benchmark's path) equals single designs bitwise
    it = 3
    f = lambda a: torch.tensor(np.asarray(a, dtype=np.float32), device="cuda").contiguous()
    got = batch.multiplane_batch(engine.context(), f(ill), f(tg).reshape(B * 3, -1), f(ph), zs, nx=n, ny=n, dx=dx,
                                 lam=LAMBDA, iterations=it)
    for d in (0, B - 1):
        one = engine.gerchbergSaxtonMultiPlane(
            ill, [{"z": zs[p], "targetAmp": tg[d, p].astype(np.float32).astype(np.float64)} for p in range(3)],
            {"nx": n, "dx": dx, "lambda": LAMBDA, "iterations": it,
             "initPhase": ph[d].astype(np.float32).astype(np.float64)})
        assert np.array_equal(got["phase"][d].cpu().numpy().astype(np.float64), one["phase"])
    err = got["error"].cpu().numpy()
    assert np.all(err[:, -1] < err[:, 0])
