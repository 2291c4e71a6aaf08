"""The tcgen05 tensor-core passes of the 1024^2 focus sweep (src/propagate.js:427-434,
transform src/fft.js:86-139) against the FP64 oracle and the FP32 CUDA-core passes.

The tensor-core passes split every operand into f16 hi + lo parts and scale the
input by a power of two taken from the spectrum maximum, so the tests cover: the
benchmark's kind of field, several wavelengths in one call, white noise (the whole
spectrum populated), fields scaled by 1e6 and 1e-12 (the scale must follow), the
all-zero field, z = 0 planes, the FP64 host entry point, that the tensor-core
kernels are the ones that ran, and that a repeated (graph-replayed) sweep stays
correct after another call has grown the context's scratch memory.
Tolerances: 1e-5 relative L2 against the oracle (every GPU parity test), 2e-6
between the tensor-core and CUDA-core paths (each is within ~5e-7 of FP64).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2
from test_gpu_fullsize import smooth_field

pytestmark = pytest.mark.gpu
N, DX = 1024, 4e-6
dp = C.POINTER(C.c_double)


def make_ctx(engine, tc=1, graph=1):
    ctx = engine._lib.Context(0)
    ctx.check(ctx.lib.doe_ctx_set_tuning(ctx.h, b"sweep_tc", tc))
    ctx.check(ctx.lib.doe_ctx_set_tuning(ctx.h, b"sweep_graph", graph))
    return ctx


def sweep(ctx, fields, lams, zs):
    import torch
    nf = fields.shape[0]
    nz = zs.size // nf
    d_in = torch.from_numpy(np.ascontiguousarray(fields.astype(np.complex64))).cuda()
    out = torch.empty((nf * nz, N, N), dtype=torch.complex64, device="cuda")
    ctx.check(ctx.lib.doe_asm_sweep_dev(ctx.h, d_in.data_ptr(), nf, N, N, DX, DX,
                                        np.ascontiguousarray(lams, dtype=np.float64).ctypes.data_as(dp),
                                        np.ascontiguousarray(zs, dtype=np.float64).ctypes.data_as(dp), nz, 1, 1,
                                        0.02, out.data_ptr()))
    ctx.synchronize()
    return out.cpu().numpy()


def oracle_plane(oracle, field, lam, z):
    src = field.astype(np.complex128).ravel()
    orr, oi = oracle.asm(src.real.copy(), src.imag.copy(), N, N, DX, DX, lam, z, True, True, 0.02)
    return orr + 1j * oi


def test_tc_sweep_matches_oracle_and_cuda_core_path(engine, oracle):
    lams = np.array([450e-9, 633e-9])
    rng = np.random.default_rng(21)
    zs = rng.uniform(15e-3, 48e-3, 2 * 8)
    f = np.stack([smooth_field(N, DX, 31), smooth_field(N, DX, 32)])
    tc, cc = make_ctx(engine, 1), make_ctx(engine, 0)
    out = sweep(tc, f, lams, zs)
    ref = sweep(cc, f, lams, zs)
    for fi, k in ((0, 0), (0, 5), (1, 3)):
        assert rel_l2(out[fi * 8 + k].ravel(), oracle_plane(oracle, f[fi], lams[fi], zs[fi * 8 + k])) < 1e-5
    for k in range(16):
        assert rel_l2(out[k], ref[k]) < 2e-6


def test_tc_sweep_white_noise_and_scale(engine, oracle):
    rng = np.random.default_rng(7)
    noise = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).astype(np.complex64)
    lam = np.array([532e-9] * 3)
    zs = np.tile(np.array([20e-3, 45e-3]), 3)
    fields = np.stack([noise, (noise.astype(np.complex128) * 1e6).astype(np.complex64),
                       (noise.astype(np.complex128) * 1e-12).astype(np.complex64)])
    ctx = make_ctx(engine, 1)
    out = sweep(ctx, fields, lam, zs)
    assert rel_l2(out[1].ravel(), oracle_plane(oracle, noise, 532e-9, 45e-3)) < 1e-5
    for k in range(2):  # a power-of-two input scale follows the field: results scale exactly with it
        assert rel_l2(out[2 + k].astype(np.complex128) / 1e6, out[k]) < 1e-6
        assert rel_l2(out[4 + k].astype(np.complex128) / 1e-12, out[k]) < 1e-6


def test_tc_sweep_zero_field_and_zero_distance(engine):
    f = smooth_field(N, DX, 5)
    fields = np.stack([np.zeros((N, N), np.complex64), f])
    zs = np.array([0.03, 0.0, 0.02, 0.0, 0.03, 0.04])  # field 0: 0.03, 0, 0.02; field 1: 0, 0.03, 0.04
    out = sweep(make_ctx(engine, 1), fields, np.array([532e-9, 532e-9]), zs)
    assert not np.any(out[:3])
    assert np.array_equal(out[3], f)  # z == 0 is the input field itself (src/propagate.js:113)
    assert np.isfinite(out).all() and np.any(out[4])


def test_tc_host_sweep_matches_oracle(engine, oracle):
    f = smooth_field(N, DX, 9).astype(np.complex128)
    zs = np.array([16e-3, 33e-3, 47e-3])
    re, im = np.ascontiguousarray(f.real.ravel()), np.ascontiguousarray(f.imag.ravel())
    ore, oim = np.zeros(3 * N * N), np.zeros(3 * N * N)
    ctx = make_ctx(engine, 1)
    ctx.check(ctx.lib.doe_asm_sweep(ctx.h, re.ctypes.data_as(dp), im.ctypes.data_as(dp), N, N, DX, DX, 633e-9,
                                    zs.ctypes.data_as(dp), 3, 1, 1, 0.02, ore.ctypes.data_as(dp),
                                    oim.ctypes.data_as(dp)))
    for k in (0, 2):
        got = ore[k * N * N:(k + 1) * N * N] + 1j * oim[k * N * N:(k + 1) * N * N]
        assert rel_l2(got, oracle_plane(oracle, f, 633e-9, zs[k])) < 1e-5


def test_tc_kernels_are_the_ones_that_ran(engine):
    ctx = make_ctx(engine, 1, graph=0)
    ctx.check(ctx.lib.doe_ctx_set_profiling(ctx.h, 1))
    sweep(ctx, smooth_field(N, DX, 1)[None], np.array([532e-9]), np.array([0.02, 0.03]))
    names = C.create_string_buffer(64 * 32)
    ms = (C.c_double * 32)()
    cnt = (C.c_ulonglong * 32)()
    n = ctx.lib.doe_ctx_profile_read(ctx.h, 32, names, 64, ms, cnt)
    labels = {names.raw[64 * k:64 * (k + 1)].split(b"\0")[0].decode() for k in range(n)}
    assert {"tc_sweep_col", "tc_sweep_row"} <= labels
    assert "asm_sweep_col" not in labels


def test_replayed_sweep_after_scratch_growth(engine):
    """A repeated device sweep is replayed from a captured CUDA graph. Another call
    that grows a scratch slot in between (a larger host propagation) must not leave
    the replay reading freed memory: the result stays equal to a direct run."""
    f = smooth_field(N, DX, 17)[None]
    zs = np.array([0.02, 0.03, 0.04])
    ctx = make_ctx(engine, 1, graph=1)
    first = sweep(ctx, f, np.array([532e-9]), zs)   # direct
    again = sweep(ctx, f, np.array([532e-9]), zs)   # captured and launched
    assert np.array_equal(first, again)
    big = 2048
    g = np.random.default_rng(0).standard_normal(2 * big * big)
    re, im = np.ascontiguousarray(g[:big * big]), np.ascontiguousarray(g[big * big:])
    ctx.check(ctx.lib.doe_asm(ctx.h, re.ctypes.data_as(dp), im.ctypes.data_as(dp), big, big, 4e-6, 4e-6, 532e-9,
                              0.03, 1, 1, 0.02))
    for _ in range(3):
        assert np.array_equal(sweep(ctx, f, np.array([532e-9]), zs), first)


def test_mirrored_row_transfer_function_form(engine, oracle):
    """The sweep column pass that evaluates H once per pair of mirrored rows
    (H(kx, ky) = H(kx, N - ky)), with per-element spectrum reads ("sweep_hsym" 1) or
    the CTA's spectrum tile staged by TMA (2), gives the plain pass's planes and the
    oracle's."""
    f = smooth_field(N, DX, 41)[None]
    zs = np.array([0.017, 0.029, 0.046])
    outs = {}
    for hsym in (0, 1, 2):
        ctx = make_ctx(engine, 0, graph=0)
        ctx.check(ctx.lib.doe_ctx_set_tuning(ctx.h, b"sweep_hsym", hsym))
        outs[hsym] = sweep(ctx, f, np.array([532e-9]), zs)
        ctx.close()
    print("mirrored-row forms bitwise equal to the plain form:", np.array_equal(outs[0], outs[1]),
          np.array_equal(outs[0], outs[2]))
    assert np.array_equal(outs[1], outs[0])  # the same factors, read from shared memory
    assert np.array_equal(outs[2], outs[0])  # ... and the spectrum staged by TMA
    for k in (0, 2):
        assert rel_l2(outs[2][k].ravel(), oracle_plane(oracle, f[0], 532e-9, zs[k])) < 1e-5


def test_spectrum_resident_multi_plane_form(engine, oracle):
    """The sweep column pass that keeps a CTA's spectrum tile in shared memory across
    K planes ("sweep_res" K; one TMA copy per tile) gives the one-plane-per-CTA pass's
    planes bitwise, including a last group shorter than K, and the oracle's."""
    f = smooth_field(N, DX, 43)[None]
    zs = np.array([0.013, 0.021, 0.034, 0.047, 0.058])
    outs = {}
    for res in (1, 2, 4, 8):
        ctx = make_ctx(engine, 0, graph=0)
        ctx.check(ctx.lib.doe_ctx_set_tuning(ctx.h, b"sweep_fused", 1))
        ctx.check(ctx.lib.doe_ctx_set_tuning(ctx.h, b"sweep_res", res))
        v = C.c_longlong(0)
        ctx.check(ctx.lib.doe_ctx_get_tuning(ctx.h, b"sweep_res", C.byref(v)))
        assert v.value == res
        outs[res] = sweep(ctx, f, np.array([532e-9]), zs)
        ctx.close()
    for res in (2, 4, 8):
        print(f"sweep_res {res} bitwise equal to one plane per CTA:", np.array_equal(outs[res], outs[1]))
        assert np.array_equal(outs[res], outs[1])
    for k in (0, 4):
        assert rel_l2(outs[4][k].ravel(), oracle_plane(oracle, f[0], 532e-9, zs[k])) < 1e-5
    ctx = make_ctx(engine, 0, graph=0)
    assert ctx.lib.doe_ctx_set_tuning(ctx.h, b"sweep_res", 0) != 0
    assert ctx.lib.doe_ctx_set_tuning(ctx.h, b"sweep_res", 65) != 0
    ctx.close()
