"""The engine against the committed golden fixtures (tests/golden/, FP64 oracle
outputs on seeded inputs). Tolerances: 1e-5 relative L2 for single transforms and
propagations; five design iterations compound FP32 rounding, so the DOE field is
held to 1e-4 and the error history to 1e-5 absolute; elementwise FP64 work
(error diffusion, hologram encoding, mode generation, modal sums) to 1e-12 or
bitwise; the FP64 screen metrics to 1e-9 relative."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LAM = 532e-9


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def field(engine, re, im, n, ny=None, dx=8e-6):
    f = engine.ComplexField(n, ny or n, dx)
    f.re[:], f.im[:] = re, im
    return f


def test_golden_fft2d(engine):
    g = load("fft2d_16x8")
    for inv, key in ((False, "fwd"), (True, "inv")):
        r, i = g["re"].copy(), g["im"].copy()
        engine.fft2d(r, i, 16, 8, inv)
        assert rel_l2(r + 1j * i, g[key + "_re"] + 1j * g[key + "_im"]) < 1e-5


def test_golden_asm(engine):
    g = load("asm_32")
    dx, lam, z1, z2 = g["params"]
    a = engine.propagateAngularSpectrum(field(engine, g["re"], g["im"], 32), lam, z1, bandLimit=True)
    assert rel_l2(a.re + 1j * a.im, g["bl_re"] + 1j * g["bl_im"]) < 1e-5
    b = engine.propagateAngularSpectrum(field(engine, g["re"], g["im"], 32), lam, z2, bandLimit=False)
    assert rel_l2(b.re + 1j * b.im, g["back_re"] + 1j * g["back_im"]) < 1e-5


def test_golden_lens_and_fresnel(engine):
    g = load("lens_fresnel_32")
    f = engine.focalPlaneSpectrum(field(engine, g["re"], g["im"], 32), LAM, 0.05)
    assert rel_l2(f.re + 1j * f.im, g["lens_re"] + 1j * g["lens_im"]) < 1e-5
    assert (f.dx, f.dy) == tuple(g["lens_d"])
    r = engine.propagateFresnelFFT(field(engine, g["re"], g["im"], 32), LAM, 0.2)
    out = r["field"]
    assert rel_l2(out.re + 1j * out.im, g["fres_re"] + 1j * g["fres_im"]) < 1e-5
    assert (out.dx, out.dy) == pytest.approx(tuple(g["fres_d"]), rel=1e-15)


@pytest.mark.parametrize("alg", ["gs", "wgs", "fourier"])
def test_golden_designs(engine, alg):
    g = load(f"design_{alg}_32")
    opts = {"nx": 32, "ny": 32, "dx": 8e-6, "lambda": LAM, "z": 0.03, "iterations": 5,
            "initPhase": g["init_phase"], "roi": g["roi"]}
    fn = {"gs": engine.gerchbergSaxton, "wgs": engine.weightedGerchbergSaxton, "fourier": engine.fourierCgh}[alg]
    r = fn(g["ill"], g["tgt"], opts)
    assert rel_l2(g["ill"] * np.exp(1j * r["phase"]), g["ill"] * np.exp(1j * g["phase"])) < 1e-4
    assert np.max(np.abs(np.asarray(r["error"]) - g["error"])) < 1e-5
    assert np.max(np.abs(np.asarray(r["efficiency"]) - g["efficiency"])) < 1e-5
    if alg == "wgs":
        assert abs(r["rmse"] - g["rmse"][0]) < 1e-5


def test_golden_multiplane(engine):
    g = load("multiplane_32")
    r = engine.gerchbergSaxtonMultiPlane(
        g["ill"], [{"z": 0.025, "targetAmp": g["t1"], "weight": 1.0}, {"z": 0.035, "targetAmp": g["t2"], "weight": 0.5}],
        {"nx": 32, "dx": 8e-6, "lambda": LAM, "iterations": 3, "initPhase": g["init_phase"]})
    assert rel_l2(g["ill"] * np.exp(1j * r["phase"]), g["ill"] * np.exp(1j * g["phase"])) < 1e-4
    assert np.allclose(np.asarray(r["perPlaneError"]), g["per_plane"], rtol=1e-4, atol=1e-7)


def test_golden_screen_metrics(engine):
    g = load("screen_metrics_32")
    c = engine.context()
    out = np.empty(18)
    dp = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))
    arrs = [np.ascontiguousarray(g[k], dtype=np.float64) for k in ("fre", "fim", "irr", "roi", "ill", "phase")]
    c.check(c.lib.doe_screen_metrics_full(c.h, dp(arrs[0]), dp(arrs[1]), 32, 32, 8e-6, 8e-6, dp(arrs[2]), dp(arrs[3]),
                                          dp(arrs[4]), dp(arrs[5]), 8e-6, 8e-6, 4, 4, dp(out)))
    ref = g["metrics"]
    for a, b in zip(out, ref):
        if np.isfinite(b):
            assert abs(a - b) <= 1e-9 * max(1.0, abs(b))


def test_golden_error_diffusion(engine):
    g = load("error_diffusion_32")
    assert np.array_equal(engine.errorDiffusionQuantize(g["phi"], 4), g["snake"])
    assert np.array_equal(engine.errorDiffusionQuantize(g["phi"], 3, {"snake": False}), g["raster"])


def test_golden_interference(engine):
    g = load("interference_32")
    h = engine.recordHologram(field(engine, g["obj_re"], g["obj_im"], 32), field(engine, g["ref_re"], g["ref_im"], 32),
                              {"encode": "phase", "levels": 4})
    assert np.array_equal(h["recorded"], g["recorded"])
    assert np.max(np.abs(h["plate"].re - g["plate_re"])) < 1e-12
    assert np.max(np.abs(h["plate"].im - g["plate_im"])) < 1e-12
    rc = engine.reconstructHologram(field(engine, g["plate_re"], g["plate_im"], 32),
                                    field(engine, g["ref_re"], g["ref_im"], 32), LAM, 0.004)
    assert rel_l2(rc["real"].re + 1j * rc["real"].im, g["real_re"] + 1j * g["real_im"]) < 1e-5
    assert rel_l2(rc["virtual"].re + 1j * rc["virtual"].im, g["virt_re"] + 1j * g["virt_im"]) < 1e-5
    modes = engine.partiallyCoherentModes(16, 16, 8e-6, 8e-6, {"modes": 3, "sigma": 24e-6, "waist": 50e-6, "seed": 5})
    for m in range(3):
        assert np.max(np.abs(modes[m].re - g["modes_re"][m])) < 1e-12
        assert np.max(np.abs(modes[m].im - g["modes_im"][m])) < 1e-12
    mi = engine.modalIntensity([field(engine, g["modes_re"][m], g["modes_im"][m], 16) for m in range(3)],
                               [1.0, 0.5, 2.0])
    assert np.array_equal(mi["intensity"], g["modal"])
