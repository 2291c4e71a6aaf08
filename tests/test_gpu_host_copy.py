"""Staged host copies of the reference-facing calls: pageable caller planes of 1 MB
or more go through the context's pinned chunks on host threads ("host_copy_threads");
the results must be bitwise those of the driver's own pageable copies and of pinned
caller buffers, for sizes that are and are not whole numbers of chunks."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
dp = C.POINTER(C.c_double)


def _ctx(engine, threads):
    ctx = engine._lib.Context(0)
    ctx.check(ctx.lib.doe_ctx_set_tuning(ctx.h, b"host_copy_threads", threads))
    v = C.c_longlong(-1)
    ctx.check(ctx.lib.doe_ctx_get_tuning(ctx.h, b"host_copy_threads", C.byref(v)))
    assert v.value == threads
    return ctx


def _p(a):
    return a.ctypes.data_as(dp)


def test_fresnel_planes_through_staging_equal_plain_copies(engine, oracle):
    nx, ny, dx = 1024, 1024, 4e-6  # 8 MiB FP64 planes: two staging chunks each
    rng = np.random.default_rng(3)
    re, im = rng.standard_normal(nx * ny), rng.standard_normal(nx * ny)
    outs = {}
    for threads in (0, 1, 6):
        ctx = _ctx(engine, threads)
        ore, oim, od = np.empty(nx * ny), np.empty(nx * ny), np.empty(2)
        for _ in range(2):  # the second call reuses the staging chunks
            ctx.check(ctx.lib.doe_fresnel(ctx.h, _p(re), _p(im), nx, ny, dx, dx, 532e-9, 0.03, _p(ore), _p(oim),
                                          _p(od)))
        outs[threads] = (ore.copy(), oim.copy())
        ctx.close()
    for threads in (1, 6):
        assert np.array_equal(outs[threads][0], outs[0][0]) and np.array_equal(outs[threads][1], outs[0][1])
    wr, wi, _, _ = oracle.fresnel(re, im, nx, ny, dx, dx, 532e-9, 0.03)
    err = np.sqrt(np.sum((outs[6][0] - wr) ** 2 + (outs[6][1] - wi) ** 2) / np.sum(wr ** 2 + wi ** 2))
    assert err < 1e-5


def test_ragged_sizes_and_pinned_caller_buffers(engine, oracle):
    """13.3 MB in and out (not a whole number of 4 MiB chunks), once from pageable
    arrays and once from pinned ones (copied directly), bitwise the oracle's scan."""
    batch, n = 100, 129 * 129
    rng = np.random.default_rng(9)
    ph = rng.uniform(-7, 7, batch * n)
    want = [oracle.error_diffusion(ph[k * n:(k + 1) * n], 4) for k in (0, 57, 99)]
    ctx = _ctx(engine, 6)
    out = np.empty_like(ph)
    ctx.check(ctx.lib.doe_error_diffusion(ctx.h, batch, n, 4, 1, 1, _p(ph), _p(out)))
    for w, k in zip(want, (0, 57, 99)):
        assert np.array_equal(out[k * n:(k + 1) * n], w)
    hin, hout = C.c_void_p(), C.c_void_p()
    ctx.check(ctx.lib.doe_host_alloc(ctx.h, C.byref(hin), ph.nbytes))
    ctx.check(ctx.lib.doe_host_alloc(ctx.h, C.byref(hout), ph.nbytes))
    a_in = np.ctypeslib.as_array((C.c_double * ph.size).from_address(hin.value))
    a_out = np.ctypeslib.as_array((C.c_double * ph.size).from_address(hout.value))
    a_in[:] = ph
    ctx.check(ctx.lib.doe_error_diffusion(ctx.h, batch, n, 4, 1, 1, C.cast(hin.value, dp), C.cast(hout.value, dp)))
    assert np.array_equal(a_out, out)
    ctx.lib.doe_host_free(ctx.h, hin)
    ctx.lib.doe_host_free(ctx.h, hout)
    assert ctx.lib.doe_ctx_set_tuning(ctx.h, b"host_copy_threads", -1) != 0
    assert ctx.lib.doe_ctx_set_tuning(ctx.h, b"host_copy_threads", 65) != 0
    ctx.close()


def test_design_host_call_through_staging(engine):
    """designDOE on a 512^2 grid (2 MiB FP64 input and result planes, one staged copy
    each): the same design with and without staging, bitwise."""
    n = 512
    yy, xx = np.mgrid[0:n, 0:n]
    target = (((xx - n / 2) ** 2 + (yy - n / 2) ** 2) < (n / 6) ** 2).astype(np.float64).ravel()
    cfg = {"nx": n, "ny": n, "dx": 8e-6, "lambda": 532e-9, "z": 0.03, "iterations": 3, "target": target,
           "algorithm": "wgs"}
    runs = {}
    for threads in (0, 4):
        ctx = _ctx(engine, threads)
        r = engine.designDOE(dict(cfg), ctx=ctx)
        runs[threads] = (np.array(r["phase"]), np.array(r["error"]))
        ctx.close()
    assert np.array_equal(runs[0][0], runs[4][0]) and np.array_equal(runs[0][1], runs[4][1])
