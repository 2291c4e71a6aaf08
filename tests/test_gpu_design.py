"""GPU parity of the phase-retrieval loops against the FP64 oracle.

Two kinds of checks:
  * field parity (1e-5 relative L2, the tolerance of every GPU test): one or two
    iterations from the same state give the same DOE field A exp(i phi) and the
    same target-plane amplitude as the oracle;
  * trajectory parity over full runs, where FP32 rounding compounds: the error and
    efficiency histories, the returned amplitude and the WGS RMSE stay within the
    bounds below of the oracle on well-conditioned designs (ROI given), and the
    reference's own known-answer assertions (test/doe.test.js) hold on GPU results.
"""
import math

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5
LAMBDA = 532e-9
DX = 8e-6


def disc(n, r):
    i = np.arange(n)
    X, Y = np.meshgrid(i, i)
    return (np.hypot(X - n / 2, Y - n / 2) <= r).astype(np.float64).ravel()


def setup(oracle, n, frac=0.3, seed=7):
    ill = oracle.disc_mask(n, n, DX, DX, 0.45 * n * DX, 2 * DX)
    tgt = oracle.prepare_target(disc(n, frac * n), ill)
    roi = oracle.auto_roi(disc(n, frac * n), n, n)
    ip = oracle.random_phase(n, n, seed)
    return ill, tgt, roi, ip


def doe_field(ill, phase):
    return ill * np.exp(1j * phase)


def run_gpu(engine, alg, ill, tgt, n, it, ip, roi=None, **kw):
    opts = {"nx": n, "ny": n, "dx": DX, "lambda": LAMBDA, "z": 0.03, "iterations": it, "initPhase": ip,
            "roi": roi, **kw}
    if alg == "gs":
        return engine.gerchbergSaxton(ill, tgt, opts)
    if alg == "wgs":
        return engine.weightedGerchbergSaxton(ill, tgt, opts)
    if alg == "fourier":
        return engine.fourierCgh(ill, tgt, opts)
    return engine.weightedGerchbergSaxton(ill, tgt, opts, engine.fourierCgh)


def run_orc(oracle, alg, ill, tgt, n, it, ip, roi=None, **kw):
    return oracle.design(alg, ill, tgt, nx=n, ny=n, dx=DX, lam=LAMBDA, z=0.03, iterations=it, init_phase=ip,
                         roi=roi, **kw)


# ------------------------------------------------------------------ field parity
@pytest.mark.parametrize("alg", ["gs", "wgs", "fourier", "wgs-fourier"])
@pytest.mark.parametrize("n,it", [(64, 1), (128, 2), (256, 1)])
@pytest.mark.parametrize("with_roi", [True, False])
def test_short_runs_match_oracle_fields(engine, oracle, alg, n, it, with_roi):
    ill, tgt, roi, ip = setup(oracle, n)
    r = roi if with_roi else None
    g = run_gpu(engine, alg, ill, tgt, n, it, ip, r)
    o = run_orc(oracle, alg, ill, tgt, n, it, ip, r)
    assert rel_l2(doe_field(ill, g["phase"]), doe_field(ill, o["phase"])) < TOL
    assert rel_l2(g["amplitude"], o["amplitude"]) < TOL
    assert np.allclose(g["error"], o["error"], rtol=TOL, atol=0)
    assert np.allclose(g["efficiency"], o["efficiency"], rtol=TOL, atol=1e-7)


def test_hio_feedback_matches_oracle(engine, oracle):
    n = 128
    ill, tgt, roi, ip = setup(oracle, n)
    g = run_gpu(engine, "gs", ill, tgt, n, 3, ip, roi, feedback=0.8, escape=1)
    o = run_orc(oracle, "gs", ill, tgt, n, 3, ip, roi, feedback=0.8, escape=1)
    assert rel_l2(doe_field(ill, g["phase"]), doe_field(ill, o["phase"])) < TOL
    assert np.allclose(g["error"], o["error"], rtol=TOL)


# ------------------------------------------------------------------ trajectory parity
@pytest.mark.parametrize("alg,n,it", [("gs", 64, 40), ("gs", 256, 100), ("wgs", 128, 40), ("wgs", 256, 100),
                                      ("fourier", 128, 40), ("fourier", 256, 100)])
def test_full_runs_track_oracle(engine, oracle, alg, n, it):
    ill, tgt, roi, ip = setup(oracle, n)
    g = run_gpu(engine, alg, ill, tgt, n, it, ip, roi)
    o = run_orc(oracle, alg, ill, tgt, n, it, ip, roi)
    assert np.max(np.abs(np.array(g["error"]) / np.array(o["error"]) - 1)) < 1e-4
    assert np.max(np.abs(np.array(g["efficiency"]) - np.array(o["efficiency"]))) < 1e-5
    assert rel_l2(g["amplitude"], o["amplitude"]) < 1e-3
    assert rel_l2(doe_field(ill, g["phase"]), doe_field(ill, o["phase"])) < 5e-3
    if alg == "wgs":
        assert abs(g["rmse"] / o["rmse"] - 1) < 1e-4
        assert rel_l2(g["weights"], o["weights"]) < 1e-3


def test_multiplane_tracks_oracle(engine, oracle):
    n, it = 128, 20
    ill = oracle.disc_mask(n, n, DX, DX, 0.45 * n * DX, 2 * DX)
    t1 = oracle.prepare_target(disc(n, 0.2 * n), ill)
    t2 = oracle.prepare_target(disc(n, 0.35 * n), ill)
    r1 = oracle.auto_roi(disc(n, 0.2 * n), n, n)
    r2 = oracle.auto_roi(disc(n, 0.35 * n), n, n)
    o = oracle.multiplane(ill, [0.025, 0.035], [t1, t2], [r1, r2], [1.0, 0.5], nx=n, ny=n, dx=DX, iterations=it)
    g = engine.gerchbergSaxtonMultiPlane(
        ill, [{"z": 0.025, "targetAmp": t1, "roi": r1, "weight": 1.0},
              {"z": 0.035, "targetAmp": t2, "roi": r2, "weight": 0.5}], {"nx": n, "dx": DX, "iterations": it})
    assert np.max(np.abs(np.array(g["error"]) - o["error"])) < 1e-5
    assert np.allclose(np.array(g["perPlaneError"]), o["perPlaneError"], rtol=1e-4)
    assert rel_l2(doe_field(ill, g["phase"]), doe_field(ill, o["phase"])) < 5e-3
    g1 = engine.gerchbergSaxtonMultiPlane(ill, [{"z": 0.025, "targetAmp": t1}], {"nx": n, "dx": DX, "iterations": 1})
    o1 = oracle.multiplane(ill, [0.025], [t1], None, None, nx=n, ny=n, dx=DX, iterations=1)
    assert rel_l2(doe_field(ill, g1["phase"]), doe_field(ill, o1["phase"])) < TOL


# ------------------------------------------------------------------ reference known answers on GPU results
N = 64


def tophat(engine):
    return engine.illuminationProfile("tophat", N, N, DX, DX, {"radius": 0.45 * N * DX})


def test_gs_reduces_error_on_gpu(engine):
    """test/doe.test.js:61-84."""
    ill = tophat(engine)
    t = np.sqrt(disc(N, 0.3 * N))
    tgt = t * math.sqrt(np.sum(ill * ill) / np.sum(t * t))
    r = engine.gerchbergSaxton(ill, tgt, {"nx": N, "ny": N, "dx": DX, "dy": DX, "lambda": LAMBDA, "z": 0.03,
                                          "iterations": 40, "seed": 5})
    assert len(r["error"]) == 40
    assert r["error"][39] < r["error"][0] and r["error"][39] < 0.5
    assert np.all(np.isfinite(r["phase"]))
    f = engine.ComplexField(N, N, DX, DX)
    f.setAmplitudePhase(ill, r["phase"])
    engine.propagateAngularSpectrumInPlace(f, LAMBDA, 0.03, {"bandLimit": False})
    irr = f.intensity()
    inroi = disc(N, 0.32 * N) > 0
    assert irr[inroi].sum() / irr.sum() > 0.5


def test_wgs_fits_signal_region_better_on_gpu(engine):
    """test/doe.test.js:86-126."""
    ill = tophat(engine)
    t = np.sqrt(disc(N, 0.3 * N))
    tgt = t * math.sqrt(np.sum(ill * ill) / np.sum(t * t))
    o = {"nx": N, "ny": N, "dx": DX, "dy": DX, "lambda": LAMBDA, "z": 0.03, "seed": 11, "iterations": 20}
    plain = engine.gerchbergSaxton(ill, tgt, o)
    weighted = engine.weightedGerchbergSaxton(ill, tgt, o)
    roi = disc(N, 0.32 * N)

    def roi_rms(amp):
        scale = math.sqrt(np.sum(amp * amp * roi) / np.sum(tgt * tgt * roi))
        m = roi != 0
        return math.sqrt(np.sum((amp[m] / scale - tgt[m]) ** 2) / np.sum(tgt[m] ** 2))

    assert roi_rms(weighted["amplitude"]) < roi_rms(plain["amplitude"])


def test_far_field_cgh_is_unitary_on_gpu(engine):
    """test/doe.test.js:128-159."""
    ill = tophat(engine)
    t = np.sqrt(disc(N, 0.25 * N))
    tgt = t * math.sqrt(np.sum(ill * ill) / np.sum(t * t))
    r = engine.fourierCgh(ill, tgt, {"nx": N, "ny": N, "dx": DX, "dy": DX, "lambda": LAMBDA, "z": 0.03,
                                     "iterations": 60, "seed": 3})
    assert r["error"][59] < r["error"][0]
    f = engine.ComplexField(N, N, DX, DX)
    f.setAmplitudePhase(ill, r["phase"])
    focal = engine.focalPlaneSpectrum(f, LAMBDA, 0.03)
    assert abs(focal.power() / f.power() - 1) < 1e-6
    meas = focal.amplitude()
    scale = math.sqrt(np.sum(meas ** 2) / np.sum(r["amplitude"] ** 2))
    assert math.sqrt(np.sum((meas / scale - r["amplitude"]) ** 2) / np.sum(r["amplitude"] ** 2)) < 0.35


def test_design_is_deterministic_and_batch_equals_single(engine):
    """test/doe.test.js:350-382 (bitwise here), and one batch == separate calls."""
    cfg = {"nx": 64, "ny": 64, "dx": DX, "lambda": LAMBDA, "z": 0.03, "iterations": 10,
           "target": disc(64, 20), "mode": "image-plane"}
    a = engine.designDOE(cfg)
    b = engine.designDOE(cfg)
    assert np.array_equal(a["phase"], b["phase"])
    assert np.all(np.abs(a["phase"]) <= math.pi + 1e-6)
    assert a["algorithm"] == "wgs" and a["mode"] == "image-plane" and 1 <= len(a["error"]) <= 10
    import ctypes as C
    from diffractiveopticalelement_b200 import _lib
    c = engine.context()
    n = 64 * 64
    ill = a["illumination"]
    descs, results, keep = (_lib.DesignDesc * 3)(), (_lib.DesignResult * 3)(), []
    singles = []
    for k in range(3):
        tgt = engine.prepareTargetAmp(disc(64, 12 + 4 * k), ill)
        ip = engine.randomPhase(64, 64, 100 + k)
        keep += [tgt, ip]
        descs[k] = _lib.DesignDesc(64, 64, DX, DX, LAMBDA, 0.03, _lib.DOE_ALG_WGS, 8, 0.0, 0, 0.9, 1.0,
                                   _lib.dp(ill), _lib.dp(tgt), None, _lib.dp(ip))
        ph = np.empty(n)
        keep.append(ph)
        results[k] = _lib.DesignResult(_lib.dp(ph), None, None, None, None, None, 0.0)
        singles.append(engine.weightedGerchbergSaxton(ill, tgt, {"nx": 64, "dx": DX, "lambda": LAMBDA, "z": 0.03,
                                                                 "iterations": 8, "initPhase": ip})["phase"])
    c.check(c.lib.doe_design_batch(c.h, 3, descs, results))
    for k in range(3):
        assert np.array_equal(np.ctypeslib.as_array(results[k].phase, shape=(n,)), singles[k])


def test_design_rejects_unsupported_grids(engine):
    from diffractiveopticalelement_b200 import DOEError
    with pytest.raises(DOEError, match="design grids"):
        engine.gerchbergSaxton(np.ones(16 * 16), np.ones(16 * 16), {"nx": 16, "iterations": 2})
    with pytest.raises(ValueError, match="no planes"):
        engine.gerchbergSaxtonMultiPlane(np.ones(64 * 64), [], {"nx": 64})
