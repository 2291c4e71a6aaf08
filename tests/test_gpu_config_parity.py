"""Parity of the benchmarked design configurations against the FP64 oracle.

C1 -- image-plane WGS exactly as the benchmark runs it (the reference's
ProjectorSystem.design path, src/doe.js:455-546 over :327-437): 256^2, pitch
8 um, 532 nm, z = 30 mm, 'rect' illumination (0.9 N dx square, raised-cosine
edge of 2 dx, src/doe.js:979-1000), a seeded target of 3-8 rectangles in the
central 128^2 window, ROI from autoRoi (src/projector.js:262-315), beta = 0.9,
seeded random initial phase, no band limit inside the loop.
  * one and two iterations: the DOE field A exp(i phi), the target-plane
    amplitude and the error / efficiency histories within 1e-5 of the oracle;
  * 100 iterations: the histories, the WGS RMSE and the screen metrics
    (projector.js:554-595) within the trajectory bounds below, and the drift of
    the DOE field against the oracle recorded per iteration count (printed; the
    FP32 loop leaves 1e-5 once rounding differences have been amplified by the
    phase retrieval's feedback, see the bound in test_c1_drift_curve).
C3 -- far-field designs (fourierCgh, src/doe.js:639-730) at the benchmark's two
largest sizes, 512^2 and 1024^2, on a seeded spot-array target: one or two
iterations within 1e-5.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5
N, DX, LAMBDA, Z = 256, 8e-6, 532e-9, 0.03


def c1_inputs(engine, seed):
    from diffractiveopticalelement_b200.projector import autoRoi, rectangles_target
    ill = engine.illuminationProfile("rect", N, N, DX, DX, {})
    irr = rectangles_target(N, N, seed)
    roi = autoRoi(irr, N, N)
    tgt = engine.prepareTargetAmp(irr, ill)
    ip = engine.randomPhase(N, N, seed)
    return ill, irr, roi, tgt, ip


def run_both(engine, oracle, seed, it):
    ill, irr, roi, tgt, ip = c1_inputs(engine, seed)
    g = engine.weightedGerchbergSaxton(ill, tgt, {"nx": N, "ny": N, "dx": DX, "lambda": LAMBDA, "z": Z,
                                                  "iterations": it, "initPhase": ip, "roi": roi, "beta": 0.9})
    o = oracle.design("wgs", ill, tgt, nx=N, ny=N, dx=DX, lam=LAMBDA, z=Z, iterations=it, init_phase=ip, roi=roi,
                      beta=0.9)
    return ill, irr, roi, g, o


def doe_field(ill, phase):
    return np.asarray(ill) * np.exp(1j * np.asarray(phase))


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("it", [1, 2])
def test_c1_short_runs_match_oracle(engine, oracle, seed, it):
    ill, irr, roi, g, o = run_both(engine, oracle, seed, it)
    assert rel_l2(doe_field(ill, g["phase"]), doe_field(ill, o["phase"])) < TOL
    assert rel_l2(g["amplitude"], o["amplitude"]) < TOL
    assert np.allclose(g["error"], o["error"], rtol=TOL, atol=0)
    assert np.allclose(g["efficiency"], o["efficiency"], rtol=TOL, atol=1e-7)


@pytest.mark.parametrize("seed", [1, 7])
def test_c1_full_run_tracks_oracle_and_meets_the_screen_goal(engine, oracle, seed):
    ill, irr, roi, g, o = run_both(engine, oracle, seed, 100)
    # histories and RMSE: the per-iteration errors of the two loops agree to 1e-4
    # relative, efficiencies to 1e-5 absolute over all 100 iterations
    assert np.max(np.abs(np.array(g["error"]) / np.array(o["error"]) - 1)) < 1e-4
    assert np.max(np.abs(np.array(g["efficiency"]) - np.array(o["efficiency"]))) < 1e-5
    assert abs(g["rmse"] / o["rmse"] - 1) < 1e-4
    # screen metrics of the returned amplitude (projector.js:554-595): RMSE and efficiency
    mg = oracle.screen_metrics(g["amplitude"], np.zeros(N * N), N, N, DX, DX, irr, roi, ill, DX, DX)
    mo = oracle.screen_metrics(o["amplitude"], np.zeros(N * N), N, N, DX, DX, irr, roi, ill, DX, DX)
    assert abs(mg["rmse"] - mo["rmse"]) < 1e-6  # 1e-4 of the 1 % goal (measured: 1.5e-7 at RMSE 0.135 %)
    assert abs(mg["efficiency"] - mo["efficiency"]) < 1e-5
    assert mg["rmse"] <= 0.01  # the benchmark's goal is reachable within 100 iterations
    # fields after 100 iterations: the drift stays within the trajectory bound
    assert rel_l2(g["amplitude"], o["amplitude"]) < 1e-3
    assert rel_l2(doe_field(ill, g["phase"]), doe_field(ill, o["phase"])) < 5e-3


def test_c1_drift_curve(engine, oracle):
    """Relative L2 distance of the DOE field A exp(i phi) between the FP32 loop and
    the FP64 oracle after k iterations of the C1 design (seed 1). Both start from
    the same state; the distance starts at FP32 rounding (~1e-7) and grows as the
    phase retrieval amplifies it. Asserted: below 1e-5 for the first iterations and
    never above the trajectory bound of the full-run tests."""
    curve = {}
    for k in (1, 2, 3, 5, 10, 20, 50, 100):
        ill, irr, roi, g, o = run_both(engine, oracle, 1, k)
        curve[k] = rel_l2(doe_field(ill, g["phase"]), doe_field(ill, o["phase"]))
    print("C1 drift (iterations: rel L2 of the DOE field vs the FP64 oracle):",
          ", ".join(f"{k}: {v:.2e}" for k, v in curve.items()))
    assert curve[1] < TOL and curve[2] < TOL
    assert all(v < 5e-3 for v in curve.values())


@pytest.mark.parametrize("n,it", [(512, 2), (1024, 1)])
def test_c3_farfield_sizes_match_oracle(engine, oracle, n, it):
    from diffractiveopticalelement_b200 import surrogate as S
    from diffractiveopticalelement_b200.projector import autoRoi
    ill = engine.discMask(n, n, DX, DX, (n * DX / 2) * 0.95, soft=2 * DX)
    irr = S.spot_array_target(n, 5000 + n)
    roi = autoRoi(irr, n, n)
    tgt = engine.prepareTargetAmp(irr, ill)
    ip = engine.randomPhase(n, n, 40 + n)
    z = n * DX * DX / LAMBDA
    g = engine.fourierCgh(ill, tgt, {"nx": n, "ny": n, "dx": DX, "lambda": LAMBDA, "z": z, "iterations": it,
                                     "initPhase": ip, "roi": roi})
    o = oracle.design("fourier", ill, tgt, nx=n, ny=n, dx=DX, lam=LAMBDA, z=z, iterations=it, init_phase=ip, roi=roi)
    assert rel_l2(doe_field(ill, g["phase"]), doe_field(ill, o["phase"])) < TOL
    assert rel_l2(g["amplitude"], o["amplitude"]) < TOL
    assert np.allclose(g["error"], o["error"], rtol=TOL, atol=0)
    assert np.allclose(g["efficiency"], o["efficiency"], rtol=TOL, atol=1e-7)
