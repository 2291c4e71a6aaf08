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
