"""CPU pins of the oracle's holography / partial-coherence restatement.

The known answers are the reference's own assertions in
test/interference.test.js (partial coherence :64-87 and :89-117, hologram
record / reconstruct :119-248), checked on the oracle, plus independent NumPy
restatements of the elementwise steps.
"""
import math

import numpy as np

N = 128
DX = 8e-6
LAMBDA = 532e-9


def coords(n, d):
    return (np.arange(n) - n / 2) * d


def visibility(plane):
    """src/metrics.js:265-268 over samples > 0 (regionStats threshold 0)."""
    v = plane[plane > 0]
    mx, mn = v.max(), v.min()
    return (mx - mn) / (mx + mn) if mx + mn > 0 else 0.0


def test_incoherent_modes_wash_fringes_out(oracle):
    k = 2 * math.pi / LAMBDA
    x = np.tile(coords(N, DX), N)
    ph = k * math.sin(0.01) * x
    are, aim, bre, bim = np.cos(ph), np.sin(ph), np.cos(-ph), np.sin(-ph)
    coherent = (are + bre) ** 2 + (aim + bim) ** 2
    inc = oracle.modal_intensity(np.concatenate([are, bre]), np.concatenate([aim, bim]), N * N)
    assert visibility(coherent) > 0.9
    assert visibility(inc) < 0.05


def test_modal_intensity_matches_numpy(oracle):
    rng = np.random.default_rng(3)
    M, n = 5, 300
    re, im = rng.standard_normal((M, n)), rng.standard_normal((M, n))
    w = rng.uniform(0.2, 2.0, M)
    got = oracle.modal_intensity(re, im, n, w)
    ref = (w[:, None] * (re ** 2 + im ** 2)).sum(0) / w.sum()
    assert np.allclose(got, ref, rtol=1e-13, atol=0)
    got1 = oracle.modal_intensity(re, im, n)
    assert np.allclose(got1, (re ** 2 + im ** 2).mean(0), rtol=1e-13)
    # zero weight sum leaves the weighted sum undivided (src/interference.js:67)
    z = oracle.modal_intensity(re[:2], im[:2], n, np.array([1.0, -1.0]))
    assert np.allclose(z, (re[0] ** 2 + im[0] ** 2) - (re[1] ** 2 + im[1] ** 2), rtol=1e-12, atol=1e-12)


def _np_box(a, r):
    """Circular box mean of radius r along both axes."""
    out = np.zeros_like(a)
    for s in range(-r, r + 1):
        out += np.roll(a, -s, axis=1)
    tmp = out / (2 * r + 1)
    out = np.zeros_like(a)
    for s in range(-r, r + 1):
        out += np.roll(tmp, -s, axis=0)
    return out / (2 * r + 1)


def test_partially_coherent_modes_restatement(oracle):
    nx, ny, modes = 32, 16, 3
    dx = 8e-6
    re, im = oracle.partially_coherent_modes(nx, ny, dx, dx, modes=modes, sigma=3 * dx, waist=60e-6, seed=5)
    ph = np.array(oracle.random_phase(nx * ny * modes, 1, seed=5)).reshape(modes, ny, nx)
    x, y = coords(nx, dx), coords(ny, dx)
    env = np.exp(-(x[None, :] ** 2 + y[:, None] ** 2) / (60e-6) ** 2)
    for m in range(modes):
        sm = _np_box(ph[m], 3)
        exp = (env * np.exp(1j * sm)).ravel()
        assert np.max(np.abs(re[m] + 1j * im[m] - exp)) < 1e-12


def test_partially_coherent_modes_reduce_speckle(oracle):
    re, im = oracle.partially_coherent_modes(N, N, DX, DX, modes=6, sigma=4 * DX, waist=0.3 * N * DX, seed=5)
    pr, pi = [], []
    for m in range(6):
        a, b = oracle.asm(re[m], im[m], N, N, DX, DX, LAMBDA, 0.05, band_limit=False)
        pr.append(a)
        pi.append(b)
    inc = oracle.modal_intensity(np.concatenate(pr), np.concatenate(pi), N * N)
    single = pr[0] ** 2 + pi[0] ** 2
    contrast = lambda v: math.sqrt(max(0.0, (v ** 2).mean() - v.mean() ** 2)) / v.mean()
    assert contrast(inc) < contrast(single)


def hologram_inputs(n=N, dx=DX):
    carrier = 16
    sin_t = LAMBDA * carrier / (n * dx)
    k = 2 * math.pi / LAMBDA
    x = np.tile(coords(n, dx), n)
    y = np.repeat(coords(n, dx), n)
    b1 = np.exp(-((x - 120e-6) ** 2 + (y + 60e-6) ** 2) / (120e-6) ** 2)
    b2 = 0.8 * np.exp(-((x + 180e-6) ** 2 + (y - 120e-6) ** 2) / (70e-6) ** 2)
    obj_re = 0.05 + np.maximum(b1, b2)
    return obj_re, np.zeros_like(obj_re), np.cos(k * sin_t * x), np.sin(k * sin_t * x), x, y


def test_record_hologram_raw_known_answers(oracle):
    ore, oim, rre, rim, _, _ = hologram_inputs()
    h = oracle.record_hologram(ore, oim, rre, rim, "raw")
    rec = h["recorded"]
    assert rec.min() >= 0 and abs(rec.max() - 1) < 1e-12
    assert np.all(h["plate_im"] == 0) and np.array_equal(h["plate_re"], rec)
    assert visibility(rec) > 0.3
    s = (ore + rre) + 1j * (oim + rim)
    assert np.allclose(rec, np.abs(s) ** 2 / (np.abs(s) ** 2).max(), rtol=1e-14)
    b = oracle.record_hologram(ore, oim, rre, rim, "binary")
    assert np.array_equal(b["plate_re"], (rec > 0.5).astype(float)) and np.all(b["plate_im"] == 0)


def test_record_hologram_phase_encodings(oracle):
    ore, oim, rre, rim, _, _ = hologram_inputs(32, 8e-6)
    p = oracle.record_hologram(ore, oim, rre, rim, "phase")
    s = (ore + rre) + 1j * (oim + rim)
    assert np.allclose(p["plate_re"] + 1j * p["plate_im"], np.exp(1j * np.angle(s)), atol=1e-14)
    q = oracle.record_hologram(ore, oim, rre, rim, "phase", levels=4)
    ang = np.angle(q["plate_re"] + 1j * q["plate_im"])
    steps = ang / (math.pi / 2)
    assert np.allclose(steps, np.round(steps), atol=1e-12)
    assert np.max(np.abs(np.angle((q["plate_re"] + 1j * q["plate_im"]) / np.exp(1j * np.angle(s))))) <= math.pi / 4 + 1e-12


def test_reconstruct_hologram_recovers_object(oracle):
    """The reference's off-axis reconstruction check (test/interference.test.js:156-247)."""
    ore, oim, rre, rim, x, y = hologram_inputs()
    h = oracle.record_hologram(ore, oim, rre, rim, "raw")
    r = oracle.reconstruct_hologram(h["plate_re"], h["plate_im"], rre, rim, N, N, DX, DX, LAMBDA, 0.005)
    ill = h["plate_re"] * rre - h["plate_im"] * rim + 1j * (h["plate_re"] * rim + h["plate_im"] * rre)
    assert np.allclose(r["illum_re"] + 1j * r["illum_im"], ill, rtol=0, atol=1e-15)
    irr = r["real_re"] ** 2 + r["real_im"] ** 2
    spec = np.fft.fftshift(np.fft.fft2((irr - irr.mean()).reshape(N, N)))
    fy = np.arange(N) - N // 2
    e = (np.abs(spec[np.abs(fy) <= 3, :]) ** 2).sum(0)
    fxs = np.arange(N) - N // 2
    e[(np.abs(fxs) < 6) | (np.abs(fxs) > 26)] = -1
    fc = int(fxs[np.argmax(e)])
    keep = (np.abs(fxs[None, :] - fc) <= 6) & (np.abs(fy[:, None]) <= 6)
    env = np.abs(np.fft.ifft2(np.fft.ifftshift(np.where(keep, spec, 0)))).ravel()
    fov = (np.abs(x) < 400e-6) & (np.abs(y) < 400e-6)
    dE, dO = env[fov] - env[fov].mean(), ore[fov] - ore[fov].mean()
    corr = (dE * dO).sum() / math.sqrt((dE ** 2).sum() * (dO ** 2).sum())
    assert corr > 0.85
    assert ore[np.argmax(env)] > 0.5
    # the virtual image is the -z propagation of the same illumination
    vr, vi = oracle.asm(r["illum_re"], r["illum_im"], N, N, DX, DX, LAMBDA, -0.005, band_limit=False)
    assert np.array_equal(vr, r["virt_re"]) and np.array_equal(vi, r["virt_im"])
