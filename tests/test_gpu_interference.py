"""GPU parity of hologram record / reconstruct, modal intensity and the
partially coherent mode generator against the FP64 oracle.

Tolerances: the elementwise FP64 steps (record, unpropagated modal sum, box
smoothing) run with every product and sum rounded separately in the
reference's order, so they are bitwise equal; transcendental steps (atan2,
exp, sin, cos from CUDA's libdevice against glibc) agree to 1e-12 absolute;
propagated fields agree to 1e-5 relative L2 (FP32 transforms, FP64-reduced
transfer-function phase).
"""
import math

import numpy as np
import pytest

from conftest import rel_l2
from test_interference_oracle import DX, LAMBDA, N, hologram_inputs, visibility

pytestmark = pytest.mark.gpu
TOL = 1e-5


def field(E, re, im, nx, ny, dx):
    f = E.ComplexField(nx, ny, dx, dx)
    f.re[:] = re
    f.im[:] = im
    return f


@pytest.mark.parametrize("encode,levels", [("raw", 0), ("binary", 0), ("phase", 0), ("phase", 4), ("phase", 7),
                                           ("raw", 4)])
def test_record_hologram_matches_oracle(engine, oracle, encode, levels):
    ore, oim, rre, rim, _, _ = hologram_inputs()
    rng = np.random.default_rng(11)
    oim = 0.2 * rng.standard_normal(ore.size)
    h = engine.recordHologram(field(engine, ore, oim, N, N, DX), field(engine, rre, rim, N, N, DX),
                              {"encode": encode, "levels": levels})
    o = oracle.record_hologram(ore, oim, rre, rim, encode, levels)
    assert np.array_equal(h["recorded"], o["recorded"])
    assert np.array_equal(h["sum"].re, o["sum_re"]) and np.array_equal(h["sum"].im, o["sum_im"])
    if encode == "phase":
        assert np.max(np.abs(h["plate"].re - o["plate_re"])) < 1e-12
        assert np.max(np.abs(h["plate"].im - o["plate_im"])) < 1e-12
    else:
        assert np.array_equal(h["plate"].re, o["plate_re"]) and np.all(h["plate"].im == 0)


def test_record_hologram_rejects_bad_input(engine):
    a = engine.ComplexField(8, 8, DX)
    with pytest.raises(ValueError):
        engine.recordHologram(a, engine.ComplexField(16, 16, DX))
    with pytest.raises(ValueError):
        engine.recordHologram(a, a, {"encode": "hologram"})


@pytest.mark.parametrize("n,z,band_limit", [(128, 0.005, False), (256, 0.02, True), (64, 0.0, False)])
def test_reconstruct_hologram_matches_oracle(engine, oracle, n, z, band_limit):
    ore, oim, rre, rim, _, _ = hologram_inputs(n, DX)
    o = oracle.record_hologram(ore, oim, rre, rim, "phase", 8)
    plate = field(engine, o["plate_re"], o["plate_im"], n, n, DX)
    ref = field(engine, rre, rim, n, n, DX)
    r = engine.reconstructHologram(plate, ref, LAMBDA, z, {"bandLimit": band_limit})
    q = oracle.reconstruct_hologram(o["plate_re"], o["plate_im"], rre, rim, n, n, DX, DX, LAMBDA, z,
                                    band_limit=band_limit)
    assert np.array_equal(r["illumination"].re, q["illum_re"]) and np.array_equal(r["illumination"].im, q["illum_im"])
    assert rel_l2(r["real"].re + 1j * r["real"].im, q["real_re"] + 1j * q["real_im"]) < TOL
    assert rel_l2(r["virtual"].re + 1j * r["virtual"].im, q["virt_re"] + 1j * q["virt_im"]) < TOL


def test_reconstruct_hologram_default_band_limit_off(engine, oracle):
    ore, oim, rre, rim, _, _ = hologram_inputs()
    o = oracle.record_hologram(ore, oim, rre, rim, "raw")
    r = engine.reconstructHologram(field(engine, o["plate_re"], o["plate_im"], N, N, DX),
                                   field(engine, rre, rim, N, N, DX), LAMBDA, 0.05)
    q = oracle.reconstruct_hologram(o["plate_re"], o["plate_im"], rre, rim, N, N, DX, DX, LAMBDA, 0.05)
    assert rel_l2(r["real"].re + 1j * r["real"].im, q["real_re"] + 1j * q["real_im"]) < TOL


@pytest.mark.parametrize("M,weighted", [(1, False), (2, False), (6, True), (70, True)])
def test_modal_intensity_matches_oracle(engine, oracle, M, weighted):
    nx, ny = 64, 32
    rng = np.random.default_rng(M)
    re, im = rng.standard_normal((M, nx * ny)), rng.standard_normal((M, nx * ny))
    w = rng.uniform(0.1, 3.0, M) if weighted else None
    modes = [field(engine, re[m], im[m], nx, ny, DX) for m in range(M)]
    got = engine.modalIntensity(modes, w)
    assert got["modeCount"] == M and got["coherence"] == (1 if M == 1 else 0)
    assert np.array_equal(got["intensity"], oracle.modal_intensity(re, im, nx * ny, w))


@pytest.mark.parametrize("M", [3, 70])
def test_propagated_modal_intensity_matches_oracle(engine, oracle, M):
    re, im = oracle.partially_coherent_modes(N, N, DX, DX, modes=M, sigma=4 * DX, waist=0.3 * N * DX, seed=5)
    modes = [field(engine, re[m], im[m], N, N, DX) for m in range(M)]
    got = engine.propagatedModalIntensity(modes, LAMBDA, 0.05, None, {"bandLimit": False})
    pr, pi = [], []
    for m in range(M):
        a, b = oracle.asm(re[m], im[m], N, N, DX, DX, LAMBDA, 0.05, band_limit=False)
        pr.append(a)
        pi.append(b)
    exp = oracle.modal_intensity(np.concatenate(pr), np.concatenate(pi), N * N)
    assert rel_l2(got["intensity"], exp) < 2 * TOL


@pytest.mark.parametrize("nx,ny,modes,sigma", [(128, 128, 6, 4 * DX), (64, 32, 3, 0.2 * DX), (256, 64, 2, 40e-6)])
def test_partially_coherent_modes_match_oracle(engine, oracle, nx, ny, modes, sigma):
    got = engine.partiallyCoherentModes(nx, ny, DX, DX, {"modes": modes, "sigma": sigma, "waist": 0.3 * nx * DX,
                                                         "seed": 5})
    re, im = oracle.partially_coherent_modes(nx, ny, DX, DX, modes=modes, sigma=sigma, waist=0.3 * nx * DX, seed=5)
    assert len(got) == modes
    for m in range(modes):
        assert np.max(np.abs(got[m].re - re[m])) < 1e-12
        assert np.max(np.abs(got[m].im - im[m])) < 1e-12


def test_partial_coherence_reference_assertions_on_gpu(engine):
    """test/interference.test.js:89-117 through the engine end to end."""
    modes = engine.partiallyCoherentModes(N, N, DX, DX, modes=6, sigma=4 * DX, waist=0.3 * N * DX, seed=5)
    single = engine.propagateAngularSpectrum(modes[0], LAMBDA, 0.05, bandLimit=False).intensity()
    inc = engine.propagatedModalIntensity(modes, LAMBDA, 0.05, bandLimit=False)["intensity"]
    contrast = lambda v: math.sqrt(max(0.0, (v ** 2).mean() - v.mean() ** 2)) / v.mean()
    assert contrast(inc) < contrast(single)


def test_hologram_reference_assertions_on_gpu(engine):
    ore, oim, rre, rim, _, _ = hologram_inputs()
    h = engine.recordHologram(field(engine, ore, oim, N, N, DX), field(engine, rre, rim, N, N, DX))
    rec = h["recorded"]
    assert rec.min() >= 0 and abs(rec.max() - 1) < 1e-12
    assert np.all(h["plate"].im == 0)
    assert visibility(rec) > 0.3
