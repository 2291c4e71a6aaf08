"""GPU parity of simulate / screenMetrics and the reference's projector known answers."""
import math

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5
BASE = {"n": 128, "pitch": 8e-6, "lambda": 532e-9, "distance": 0.03, "iterations": 40, "seed": 12345}


@pytest.mark.parametrize("mode,pad,bl", [("image-plane", 1, False), ("image-plane", 2, False),
                                         ("image-plane", 1, True), ("far-field", 1, False)])
def test_simulate_matches_oracle(engine, oracle, mode, pad, bl):
    n, dx, lam, z = 128, 8e-6, 532e-9, 0.03
    ill = oracle.disc_mask(n, n, dx, dx, 0.45 * n * dx, 2 * dx)
    ph = oracle.random_phase(n, n, 5)
    sys_ = engine.ProjectorSystem({**BASE, "mode": mode})
    sys_.result = {"illumination": ill, "phase": ph}
    f = sys_.simulate({"pad": pad, "bandLimit": bl})
    er, ei = ill * np.cos(ph), ill * np.sin(ph)
    if mode == "far-field":
        orr, oi, odx, _ = oracle.focal_plane(er, ei, n, n, dx, dx, lam, z)
        assert f.dx == odx
    else:
        N = n * pad
        o = (N - n) // 2
        pr = np.zeros((N, N)); pi = np.zeros((N, N))
        pr[o:o + n, o:o + n] = er.reshape(n, n)
        pi[o:o + n, o:o + n] = ei.reshape(n, n)
        rr, ii = oracle.asm(pr.ravel(), pi.ravel(), N, N, dx, dx, lam, z, bl, True, 0.02)
        orr = rr.reshape(N, N)[o:o + n, o:o + n].ravel()
        oi = ii.reshape(N, N)[o:o + n, o:o + n].ravel()
    assert rel_l2(f.re + 1j * f.im, orr + 1j * oi) < TOL


def test_screen_metrics_match_oracle(engine, oracle):
    n = 128
    sys_ = engine.ProjectorSystem({**BASE, "target": {"kind": "disc"}})
    rng = np.random.default_rng(1)
    f = engine.ComplexField(n, n, 8e-6)
    f.re[:] = rng.standard_normal(n * n)
    f.im[:] = rng.standard_normal(n * n)
    ph = rng.uniform(-np.pi, np.pi, n * n)
    m = sys_.screenMetrics(f, {"phase": ph})
    o = oracle.screen_metrics(f.re, f.im, n, n, f.dx, f.dy, sys_.target["irradiance"], sys_.target["roi"],
                              sys_.illumination(), sys_.dx, sys_.dy)
    for k in ("rmse", "efficiency", "fluxFraction", "powerInSignal", "powerAtScreen", "powerIncident"):
        assert abs(m[k] / o[k] - 1) < 1e-6, k


@pytest.mark.parametrize("kind,extra", [("disc", {}), ("dots", {"cols": 6, "rows": 5}), ("ring", {})])
def test_full_screen_metrics_match_oracle(engine, oracle, kind, extra):
    """Every field of screenMetrics (regionStats, correlation, SSIM, spot uniformity,
    zero order, rms radius) against the FP64 restatement of src/metrics.js."""
    n = 128
    sys_ = engine.ProjectorSystem({**BASE, "target": {"kind": kind, **extra}})
    sys_.design({"iterations": 8})
    f = sys_.simulate()
    m = sys_.screenMetrics(f)
    o = oracle.screen_metrics_full(f.re, f.im, n, n, f.dx, f.dy, sys_.target["irradiance"], sys_.target["roi"],
                                   sys_.result["illumination"], sys_.result["phase"], sys_.dx, sys_.dy,
                                   sys_.target.get("grid"))
    assert set(m) == set(o)
    for k, v in o.items():
        if v is None or not np.isfinite(v):
            assert m[k] == v or (v is not None and not np.isfinite(m[k])), k
        else:
            assert abs(m[k] - v) <= 1e-9 * max(1.0, abs(v)), (k, m[k], v)


def test_projection_conserves_energy(engine):
    """test/projector.test.js:86-102."""
    sys_ = engine.ProjectorSystem({**BASE, "n": 64, "mode": "image-plane", "target": {"kind": "disc"}})
    sys_.design({"iterations": 10})
    field = sys_.simulate()
    screen = float(np.sum(field.intensity()))
    incident = float(np.sum(sys_.illumination() ** 2))
    assert abs(screen / incident - 1) < 1e-6
    assert field.nx == sys_.nx and abs(field.dx - sys_.dx) < 1e-18


def test_image_plane_design_beats_flat_element(engine):
    """test/projector.test.js:62-84 (radiometric part) on a disc target."""
    sys_ = engine.ProjectorSystem({**BASE, "mode": "image-plane", "target": {"kind": "disc"}})
    r = sys_.design()
    assert r["mode"] == "image-plane" and r["iterations"] == 40 and r["algorithm"] == "wgs"
    m = sys_.screenMetrics(sys_.simulate())
    flat = np.zeros(sys_.nx * sys_.ny)
    mf = sys_.screenMetrics(sys_.simulate({"phase": flat}))
    assert m["rmse"] < mf["rmse"]
    assert m["efficiency"] > 0.55 and m["fluxFraction"] > 0.55


def test_far_field_is_distance_invariant(engine):
    """test/projector.test.js:104-150 and :274-289 (scale-aware radiometry)."""
    sys_ = engine.ProjectorSystem({**BASE, "mode": "far-field", "target": {"kind": "disc"}})
    sys_.design({"iterations": 20})
    a = sys_.simulate({"z": 0.02})
    b = sys_.simulate({"z": 0.05})
    assert abs(a.dx - (sys_.lam * 0.02) / (sys_.nx * sys_.dx)) < 1e-18

    def norm(f):
        ir = f.intensity()
        return ir / ir.mean()
    na, nb = norm(a), norm(b)
    assert math.sqrt(np.sum((na - nb) ** 2) / np.sum(na * na)) < 1e-5
    assert abs(a.power() / b.power() - 1) < 1e-6
    m1 = sys_.screenMetrics(sys_.simulate({"z": 0.03}))
    m2 = sys_.screenMetrics(sys_.simulate({"z": 0.06}))
    assert abs(m1["efficiency"] - m2["efficiency"]) < 1e-6
    assert abs(m1["rmse"] - m2["rmse"]) < 1e-5


def test_auto_algorithm_per_mode(engine):
    """test/projector.test.js:152-180."""
    image = engine.ProjectorSystem({**BASE, "n": 64, "mode": "image-plane", "target": {"kind": "disc"}})
    far = engine.ProjectorSystem({**BASE, "n": 64, "mode": "far-field", "target": {"kind": "disc"}})
    ri = image.design({"iterations": 20})
    rf = far.design({"iterations": 20})
    assert ri["algorithm"] == "wgs" and rf["algorithm"] == "gs"
    mi = image.screenMetrics(image.simulate())
    mf = far.screenMetrics(far.simulate())
    assert mi["rmse"] < 0.1 and mf["rmse"] < 0.35
    assert np.max(np.abs(np.cos(ri["phase"]) - np.cos(rf["phase"]))) > 0.2


def test_multiplane_projector_runs(engine):
    sys_ = engine.ProjectorSystem({**BASE, "n": 64, "target": {"kind": "disc"}})
    r = sys_.designMultiPlane([{"kind": "disc", "z": 0.025}, {"kind": "ring", "z": 0.035, "weight": 0.5}],
                              {"iterations": 10})
    assert r["mode"] == "multi-plane" and len(r["error"]) == 10 and len(r["perPlaneError"]) == 2
    assert r["error"][-1] < r["error"][0]


@pytest.mark.parametrize("mode,pad,bl", [("image-plane", 2, False), ("image-plane", 1, True), ("far-field", 1, False)])
def test_simulate_many_equals_per_distance_simulate(engine, oracle, mode, pad, bl):
    """One engine call for many distances (shared forward transform) gives the
    planes of one simulate call per distance, z = 0 included in the near field."""
    n, dx = 128, 8e-6
    sys_ = engine.ProjectorSystem({**BASE, "mode": mode})
    sys_.result = {"illumination": oracle.disc_mask(n, n, dx, dx, 0.45 * n * dx, 2 * dx),
                   "phase": oracle.random_phase(n, n, 9)}
    zs = [0.012, 0.03, 0.047, 0.0211] + ([] if mode == "far-field" else [0.0, -0.02])
    many = sys_.simulateMany(zs, {"pad": pad, "bandLimit": bl})
    for z, f in zip(zs, many):
        one = sys_.simulate({"z": z, "pad": pad, "bandLimit": bl})
        assert (f.dx, f.dy) == (one.dx, one.dy)
        if mode == "far-field" or z == 0.0:
            assert np.array_equal(f.re, one.re) and np.array_equal(f.im, one.im)
        else:
            assert rel_l2(f.re + 1j * f.im, one.re + 1j * one.im) < 1e-6


@pytest.mark.parametrize("mode", ["image-plane", "far-field"])
def test_defocus_curve_and_focus_stack(engine, mode):
    """defocusCurve (src/projector.js:622-642) and focusStack (:645-653): distances,
    per-plane metrics equal to screenMetrics(simulate(z)), best focus at the design
    distance for the image-plane design."""
    sys_ = engine.ProjectorSystem({**BASE, "n": 64, "mode": mode, "target": {"kind": "disc"}})
    sys_.design()
    curve = sys_.defocusCurve({"points": 7, "span": 0.6})
    assert len(curve) == 7
    assert curve[3]["z"] == pytest.approx(sys_.z)
    for p in (curve[0], curve[3], curve[6]):
        m = sys_.screenMetrics(sys_.simulate({"z": p["z"], "pad": 2}))
        for k in ("rmse", "efficiency", "correlation", "ssim", "uniformity"):
            assert p[k] == pytest.approx(m[k], rel=1e-4, abs=1e-9)
    if mode == "image-plane":
        assert min(range(7), key=lambda i: curve[i]["rmse"]) == 3
    stack = sys_.focusStack({"points": 5})
    assert [round(s["z"] / sys_.z, 6) for s in stack] == [0.5, 0.75, 1.0, 1.25, 1.5]
    mid = sys_.simulate({"z": stack[2]["z"], "pad": 2}).intensity()
    assert rel_l2(stack[2]["intensity"], mid) < 1e-6
