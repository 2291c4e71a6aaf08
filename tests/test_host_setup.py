"""Host-side set-up that mirrors the reference's own host code (no GPU needed)."""
import numpy as np
import pytest


@pytest.mark.parametrize("kind,opts", [("disc", {}), ("ring", {}), ("checker", {}), ("lines", {}), ("zone", {}),
                                        ("dots", {"cols": 6, "rows": 5}), ("rects", {"seed": 3})])
@pytest.mark.parametrize("n", [64, 128])
def test_auto_roi_matches_oracle(engine, oracle, kind, opts, n):
    from diffractiveopticalelement_b200.projector import autoRoi, makeTarget
    t = makeTarget(kind, n, n, opts)
    ref = oracle.auto_roi(t["irradiance"], n, n)
    assert np.array_equal(t["roi"], ref) or np.max(np.abs(t["roi"] - ref)) < 1e-15
    for dil, soft in [(1, 0), (3, 1), (2, 3)]:
        a = autoRoi(t["irradiance"], n, n, {"dilate": dil, "soft": soft})
        b = oracle.auto_roi(t["irradiance"], n, n, dil, soft)
        assert np.max(np.abs(a - b)) < 1e-15


def test_rectangles_target_is_seeded_and_bounded(engine):
    from diffractiveopticalelement_b200.projector import rectangles_target
    a = rectangles_target(256, 256, 7)
    b = rectangles_target(256, 256, 7)
    c = rectangles_target(256, 256, 8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    m = a.reshape(256, 256)
    ys, xs = np.nonzero(m)
    assert xs.min() >= 64 and xs.max() < 192 and ys.min() >= 64 and ys.max() < 192
    assert set(np.unique(m)) <= {0.0, 1.0}


def test_target_power_match_matches_oracle(engine, oracle):
    ill = oracle.rect_mask(64, 64, 8e-6, 8e-6, 0.9 * 64 * 8e-6, 0.9 * 64 * 8e-6, 16e-6)
    irr = np.random.default_rng(0).random(64 * 64)
    assert np.max(np.abs(engine.prepareTargetAmp(irr, ill) / oracle.prepare_target(irr, ill) - 1)) < 1e-13


def test_projector_defaults_and_geometry(engine):
    P = engine.ProjectorSystem
    sys_ = P({"n": 128, "pitch": 8e-6, "lambda": 532e-9, "mode": "far-field"})
    assert abs(sys_.z - sys_.matchDistance()) < 1e-15  # src/projector.js:359-361
    assert P({"n": 128, "mode": "far-field", "distance": 0.02}).z == 0.02
    with pytest.raises(ValueError, match="unknown kind"):
        P({"n": 64, "target": {"kind": "spiral"}})


def test_design_doe_defaults_follow_the_reference_nullish_rule(engine, monkeypatch):
    """designDOE (src/doe.js:796-866) fills a default only where the option is
    missing or null (`??`): an explicit None takes the default, an explicit 0 is
    kept. The device loop is intercepted, so this runs without a GPU."""
    from diffractiveopticalelement_b200 import doe as D
    seen = {}

    def fake_run(algorithm, illumination, targetAmp, o, ctx=None):
        seen.update(o)
        n = int(o["nx"]) * int(o["ny"])
        return {"phase": np.zeros(n), "error": [], "efficiency": [], "amplitude": np.zeros(n),
                "intensity": np.zeros(n), "iterations": o["iterations"], "field": None, "rmse": 0.0,
                "weights": np.ones(n), "weightedIterations": o["iterations"]}

    monkeypatch.setattr(D, "_run", fake_run)
    r = D.designDOE({"nx": 32, "seed": None, "beta": None, "escape": 0, "iterations": 10, "progressEvery": None,
                     "z": 0.0})
    assert seen["seed"] == 12345 and seen["beta"] == 0.9 and seen["progressEvery"] == 10
    assert seen["escape"] == 0 and seen["z"] == 0.0 and r["z"] == 0.0  # explicit zeros are kept
    assert np.array_equal(r["illumination"], D.discMask(32, 32, 8e-6, 8e-6, (32 * 8e-6 / 2) * 0.95, soft=16e-6))
    D.designDOE({"nx": 32, "iterations": 10})
    assert seen["escape"] == 2  # Math.round(iterations * 0.2)
    assert np.array_equal(seen["initPhase"], D.randomPhase(32, 32, 12345))
