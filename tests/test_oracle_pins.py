"""Pin the FP64 oracle to the reference's own known-answer tests.

The reference ships no golden vectors; its tests (test/*.test.js) assert analytic
identities and tolerance bounds on seeded inputs. Each test below restates one of
them, with the same inputs (same LCG / xorshift seeds, same grids) and the same
bound, against the oracle. Citations are test files inside the reference project.
"""
import math

import numpy as np
import pytest

LAMBDA = 532e-9


def lcg_array(n, seed, offset=0.5):
    """test/fft.test.js:5-14 LCG, evaluated in IEEE doubles as JavaScript does."""
    s = float(seed)
    out = np.empty(n)
    for i in range(n):
        s = (1103515245.0 * s + 12345.0) % 2147483648.0
        out[i] = s / 2147483648.0 - offset
    return out


def random_field(n, seed=5):
    """test/propagate.test.js:27-39: re, im interleaved from one LCG stream."""
    s = float(seed)
    re = np.empty(n * n)
    im = np.empty(n * n)
    for k in range(n * n):
        s = (1103515245.0 * s + 12345.0) % 2147483648.0
        re[k] = s / 2147483648.0 - 0.5
        s = (1103515245.0 * s + 12345.0) % 2147483648.0
        im[k] = s / 2147483648.0 - 0.5
    return re, im


def gaussian_field(n, dx, w0):
    """test/propagate.test.js:41-51."""
    i = np.arange(n)
    x = (i - n / 2) * dx
    X, Y = np.meshgrid(x, x)
    return np.exp(-(X * X + Y * Y) / (w0 * w0)).ravel(), np.zeros(n * n)


def rel_err(ar, ai, br, bi):
    num = np.sum((ar - br) ** 2 + (ai - bi) ** 2)
    den = np.sum(br ** 2 + bi ** 2)
    return math.sqrt(num / den)


# ------------------------------------------------------------ test/fft.test.js
def test_fft1d_matches_naive_dft(oracle):
    n = 16
    re, im = lcg_array(n, 3), lcg_array(n, 7)
    k = np.arange(n)
    a = (-2 * np.pi * np.outer(k, k)) / n
    er = (re * np.cos(a) - im * np.sin(a)).sum(axis=1)
    ei = (re * np.sin(a) + im * np.cos(a)).sum(axis=1)
    r, i = oracle.fft1d(re, im)
    assert np.max(np.abs(r - er)) < 1e-10 and np.max(np.abs(i - ei)) < 1e-10


def test_fft2d_matches_naive_and_inverts(oracle):
    nx = ny = 8
    re, im = lcg_array(64, 11), lcg_array(64, 13)
    nr, ni = oracle.dft2d_naive(re, im, nx, ny)
    r, i = oracle.fft2d(re, im, nx, ny)
    assert max(np.abs(r - nr).max(), np.abs(i - ni).max()) < 1e-10
    r2, i2 = oracle.fft2d(r, i, nx, ny, inverse=True)
    assert max(np.abs(r2 - re).max(), np.abs(i2 - im).max()) < 1e-12


def test_fftshift_moves_dc_to_centre(oracle):
    re = np.zeros(64)
    re[0] = 1
    r, _ = oracle.fftshift2d(re, np.zeros(64), 8, 8, True)
    assert r[4 + 4 * 8] == 1
    r2, _ = oracle.fftshift2d(r, np.zeros(64), 8, 8, False)
    assert r2[0] == 1


def test_delta_flat_and_parseval(oracle):
    n = 32
    re = np.zeros(n)
    re[0] = 1
    r, i = oracle.fft1d(re, np.zeros(n))
    assert np.all(np.abs(np.hypot(r, i) - 1) < 1e-12)
    x, y = lcg_array(n, 17), lcg_array(n, 19)
    xr, xi = oracle.fft1d(x, y)
    t = np.sum(x * x + y * y)
    f = np.sum(xr * xr + xi * xi)
    assert abs(t - f / n) / t < 1e-12


def test_oracle_fft_agrees_with_pocketfft(oracle):
    """Independent check of the restated radix-2 FFT against numpy's FFT."""
    rng = np.random.default_rng(0)
    for nx, ny in [(1, 8), (16, 4), (64, 64), (256, 32)]:
        re, im = rng.standard_normal(nx * ny), rng.standard_normal(nx * ny)
        r, i = oracle.fft2d(re, im, nx, ny)
        ref = np.fft.fft2((re + 1j * im).reshape(ny, nx)).ravel()
        assert np.abs((r + 1j * i) - ref).max() < 1e-9 * max(1.0, np.abs(ref).max())


# ------------------------------------------------------------ test/propagate.test.js
def test_asm_unitary_and_invertible(oracle):
    n, dx, z = 64, 8e-6, 25e-3
    re, im = random_field(n)
    fr, fi = oracle.asm(re, im, n, n, dx, dx, LAMBDA, z, band_limit=False)
    br, bi = oracle.asm(fr, fi, n, n, dx, dx, LAMBDA, -z, band_limit=False)
    assert rel_err(br, bi, re, im) < 1e-8
    p0 = np.sum(re * re + im * im)
    p1 = np.sum(fr * fr + fi * fi)
    assert abs(p1 / p0 - 1) < 1e-12


def test_asm_gaussian_beam_width(oracle):
    n, dx, w0, z = 256, 6e-6, 120e-6, 0.1
    re, im = gaussian_field(n, dx, w0)
    r, i = oracle.asm(re, im, n, n, dx, dx, LAMBDA, z, band_limit=False)
    irr = (r * r + i * i).reshape(n, n)
    x = (np.arange(n) - n / 2) * dx
    X, Y = np.meshgrid(x, x)
    measured = math.sqrt(np.sum(irr * (X * X + Y * Y)) / np.sum(irr))
    analytic = w0 * math.sqrt(1 + ((LAMBDA * z) / (math.pi * w0 * w0)) ** 2) / math.sqrt(2)
    assert abs(measured / analytic - 1) < 0.01


def test_fresnel_matches_brute_force_integral(oracle):
    n, dx, z = 8, 20e-6, 50e-3
    re, im = gaussian_field(n, dx, 60e-6)
    im[10] = 0.25
    du = (LAMBDA * z) / (n * dx)
    A = (dx * dx) / (LAMBDA * z)
    kz = (2 * math.pi * z) / LAMBDA
    x = (np.arange(n) - n / 2) * dx
    refR = np.zeros(n * n)
    refI = np.zeros(n * n)
    for v in range(n):
        for u in range(n):
            U, V = (u - n / 2) * du, (v - n / 2) * du
            sr = si = 0.0
            for j in range(n):
                for i in range(n):
                    q = (math.pi * ((U - x[i]) ** 2 + (V - x[j]) ** 2)) / (LAMBDA * z) + kz - math.pi / 2
                    vr, vi = re[i + j * n], im[i + j * n]
                    sr += (vr * math.cos(q) - vi * math.sin(q)) * A
                    si += (vr * math.sin(q) + vi * math.cos(q)) * A
            refR[u + v * n], refI[u + v * n] = sr, si
    r, i, _, _ = oracle.fresnel(re, im, n, n, dx, dx, LAMBDA, z)
    assert rel_err(r, i, refR, refI) < 1e-9


def test_fresnel_energy_and_inverse(oracle):
    n, dx, z = 128, 8e-6, 30e-3
    re, im = random_field(n, 21)
    r, i, dux, duy = oracle.fresnel(re, im, n, n, dx, dx, LAMBDA, z)
    pin = np.sum(re * re + im * im) * dx * dx
    pout = np.sum(r * r + i * i) * dux * duy
    assert abs(pout / pin - 1) < 1e-12
    br, bi = oracle.fresnel_inverse(r, i, n, n, dux, duy, LAMBDA, z, dx, dx)
    assert rel_err(br, bi, re, im) < 1e-8


def test_asm_and_fresnel_agree_at_critical_distance(oracle):
    n, dx = 128, 8e-6
    zc = (n * dx * dx) / LAMBDA
    re, im = gaussian_field(n, dx, 150e-6)
    ar, ai = oracle.asm(re, im, n, n, dx, dx, LAMBDA, zc, band_limit=False)
    fr, fi, _, _ = oracle.fresnel(re, im, n, n, dx, dx, LAMBDA, zc)
    a, b = ar * ar + ai * ai, fr * fr + fi * fi
    assert math.sqrt(np.sum((a - b) ** 2) / np.sum(a * a)) < 1e-4


def test_thin_lens_airy_encircled_energy(oracle):
    n, dx, f = 256, 8e-6, 40e-3
    ap = oracle.disc_mask(n, n, dx, dx, ((n * dx) / 2) * 0.6, 0.0)
    x = (np.arange(n) - n / 2) * dx
    X, Y = np.meshgrid(x, x)
    phi = ((-(2 * math.pi / LAMBDA) * (X * X + Y * Y)) / (2 * f)).ravel()
    re, im = ap * np.cos(phi), ap * np.sin(phi)
    r, i = oracle.asm(re, im, n, n, dx, dx, LAMBDA, f, band_limit=False)
    irr = r * r + i * i
    peak = int(np.argmax(irr))
    assert peak % n == n // 2 and peak // n == n // 2
    D = 2 * ((n * dx) / 2) * 0.6
    airy = (1.22 * LAMBDA * f) / D
    rr = np.hypot(X, Y).ravel()
    order = np.argsort(rr, kind="stable")
    acc = np.cumsum(irr[order]) / irr.sum()
    r838 = rr[order][np.searchsorted(acc, 0.838)]
    assert abs(r838 / airy - 1) < 0.15


def test_band_limit_cuts_beyond_local_limit(oracle):
    n, dx, z = 128, 8e-6, 0.05
    lim = oracle.local_frequency_limit(n, dx, LAMBDA, z)
    df = 1 / (n * dx)
    hr, hi, _ = oracle.asm_transfer(n, n, dx, dx, LAMBDA, z, True, True, 0.01)
    over = math.floor(lim / df) + 4
    p = 0.0
    for k in (over, over + 1, over + 2):
        i = n // 2 + k
        if i >= n:
            continue
        idx = i + (n // 2) * n
        p += hr[idx] ** 2 + hi[idx] ** 2
    assert p < 1e-6


# ------------------------------------------------------------ test/doe.test.js
N, DX = 64, 8e-6


def target_disc(n, r):
    i = np.arange(n)
    X, Y = np.meshgrid(i, i)
    return (np.hypot(X - n / 2, Y - n / 2) <= r).astype(np.float64).ravel()


def norm_to_power(amp, power):
    p = np.sum(amp * amp)
    return amp * (math.sqrt(power / p) if p > 0 else 1.0)


def tophat(oracle):
    return oracle.disc_mask(N, N, DX, DX, 0.45 * N * DX, 2 * DX)


def test_gs_reduces_error(oracle):
    ill = tophat(oracle)
    tgt = norm_to_power(np.sqrt(target_disc(N, 0.3 * N)), np.sum(ill * ill))
    r = oracle.design("gs", ill, tgt, nx=N, ny=N, dx=DX, lam=LAMBDA, z=0.03, iterations=40, seed=5)
    assert len(r["error"]) == 40
    assert r["error"][39] < r["error"][0] and r["error"][39] < 0.5
    fr, fi = oracle.asm(ill * np.cos(r["phase"]), ill * np.sin(r["phase"]), N, N, DX, DX, LAMBDA,
                        0.03, band_limit=False)
    irr = fr * fr + fi * fi
    i = np.arange(N)
    X, Y = np.meshgrid(i, i)
    inroi = (np.hypot(X - N / 2, Y - N / 2) <= 0.32 * N).ravel()
    assert irr[inroi].sum() / irr.sum() > 0.5


def test_wgs_fits_signal_region_better_than_gs(oracle):
    ill = tophat(oracle)
    tgt = norm_to_power(np.sqrt(target_disc(N, 0.3 * N)), np.sum(ill * ill))
    kw = dict(nx=N, ny=N, dx=DX, lam=LAMBDA, z=0.03, seed=11, iterations=20)
    plain = oracle.design("gs", ill, tgt, **kw)
    weighted = oracle.design("wgs", ill, tgt, **kw)
    roi = target_disc(N, 0.32 * N)

    def roi_rms(amp):
        measured = np.sum(amp * amp * roi)
        demanded = np.sum(tgt * tgt * roi)
        scale = math.sqrt(measured / demanded)
        m = roi != 0
        return math.sqrt(np.sum((amp[m] / scale - tgt[m]) ** 2) / np.sum(tgt[m] ** 2))

    assert roi_rms(weighted["amplitude"]) < roi_rms(plain["amplitude"])
    assert np.all(np.isfinite(weighted["phase"]))


def test_far_field_cgh_unitary_and_improves(oracle):
    ill = tophat(oracle)
    tgt = norm_to_power(np.sqrt(target_disc(N, 0.25 * N)), np.sum(ill * ill))
    r = oracle.design("fourier", ill, tgt, nx=N, ny=N, dx=DX, lam=LAMBDA, z=0.03, iterations=60, seed=3)
    assert r["error"][59] < r["error"][0]
    er, ei = ill * np.cos(r["phase"]), ill * np.sin(r["phase"])
    fr, fi, dux, duy = oracle.focal_plane(er, ei, N, N, DX, DX, LAMBDA, 0.03)
    pin = np.sum(er * er + ei * ei) * DX * DX
    pout = np.sum(fr * fr + fi * fi) * dux * duy
    assert abs(pout / pin - 1) < 1e-9
    meas = np.hypot(fr, fi)
    scale = math.sqrt(np.sum(meas ** 2) / np.sum(r["amplitude"] ** 2))
    num = np.sum((meas / scale - r["amplitude"]) ** 2)
    assert math.sqrt(num / np.sum(r["amplitude"] ** 2)) < 0.35


def test_focal_plane_scale_invariance(oracle):
    rng = oracle.Rng(17)
    re = np.empty(N * N)
    im = np.empty(N * N)
    for k in range(N * N):
        re[k] = rng() - 0.5
        im[k] = rng() - 0.5
    ar, ai, adx, ady = oracle.focal_plane(re, im, N, N, DX, DX, LAMBDA, 0.02)
    br, bi, bdx, bdy = oracle.focal_plane(re, im, N, N, DX, DX, LAMBDA, 0.05)

    def shape(r, i):
        irr = r * r + i * i
        return irr / (irr.sum() / irr.size)

    sa, sb = shape(ar, ai), shape(br, bi)
    assert math.sqrt(np.sum((sa - sb) ** 2) / np.sum(sa * sa)) < 1e-12
    pa = np.sum(ar * ar + ai * ai) * adx * ady
    pb = np.sum(br * br + bi * bi) * bdx * bdy
    assert abs(pa / pb - 1) < 1e-9


def test_design_is_deterministic(oracle):
    ill = oracle.disc_mask(64, 64, DX, DX, (64 * DX / 2) * 0.95, 2 * DX)
    tgt = oracle.prepare_target(target_disc(64, 20), ill)
    ip = oracle.random_phase(64, 64, 12345)
    a = oracle.design("wgs", ill, tgt, nx=64, ny=64, dx=DX, lam=LAMBDA, z=0.03, iterations=10,
                      init_phase=ip, escape=2)
    b = oracle.design("wgs", ill, tgt, nx=64, ny=64, dx=DX, lam=LAMBDA, z=0.03, iterations=10,
                      init_phase=ip, escape=2)
    assert np.max(np.abs(a["phase"] - b["phase"])) < 1e-12
    assert np.all(np.abs(a["phase"]) <= math.pi + 1e-12)


def test_make_rng_matches_xorshift32(oracle):
    """src/doe.js:65-75: pinned first outputs of makeRng(1) computed by hand."""
    r = oracle.Rng(1)
    s = 1
    for _ in range(5):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        assert r() == s / 4294967296.0
    assert oracle.Rng(0)() == oracle.Rng(1)()  # `seed >>> 0 || 1`


def test_full_screen_metrics_known_answers(oracle):
    """src/metrics.js definitions on planes whose answers are known by construction."""
    n, d = 64, 8e-6
    i = np.arange(n)
    X, Y = np.meshgrid(i, i)
    disc = (np.hypot(X - n / 2, Y - n / 2) <= 12).astype(float).ravel()
    ill = np.ones(n * n)
    flat = np.zeros(n * n)
    # a flat screen over the ROI: uniform; correlation is 0 by definition (no variance)
    amp = np.sqrt(3.0 * disc)
    m = oracle.screen_metrics_full(amp, np.zeros(n * n), n, n, d, d, disc, disc, ill, flat, d, d)
    assert m["rmse"] == 0 and m["correlation"] == 0 and abs(m["ssim"] - 1) < 1e-12
    assert m["uniformity"] == 1 and m["flatness"] == 1 and m["contrast"] == 0 and m["fidelity"] == 0.5
    assert m["snr"] == float("inf") and m["spotUniformity"] is None
    assert abs(m["meanIntensity"] - 3.0) < 1e-12 and abs(m["peakIntensity"] - 3.0) < 1e-12
    # screen = 3 x a structured target: perfect fidelity
    tg = disc * (1.5 + np.cos(X / 3.0).ravel())
    ms = oracle.screen_metrics_full(np.sqrt(3.0 * tg), np.zeros(n * n), n, n, d, d, tg, disc, ill, flat, d, d)
    assert ms["rmse"] < 1e-15 and abs(ms["correlation"] - 1) < 1e-12 and abs(ms["ssim"] - 1) < 1e-12
    # flat element phase: all power in the zero order; a 0/pi checkerboard: none
    assert abs(m["zeroOrder"] - 1) < 1e-12
    cb = np.where((X + Y) % 2 == 0, 0.0, np.pi).ravel()
    m2 = oracle.screen_metrics_full(amp, np.zeros(n * n), n, n, d, d, disc, disc, ill, cb, d, d)
    assert m2["zeroOrder"] < 1e-20
    # rms radius: two equal points at (+-a, 0) from the centre -> r = a
    two = np.zeros((n, n))
    two[n // 2, n // 2 - 5] = two[n // 2, n // 2 + 5] = 1.0
    m3 = oracle.screen_metrics_full(two.ravel(), np.zeros(n * n), n, n, d, d, disc, None, ill, flat, d, d)
    assert abs(m3["rmsRadius"] - 5 * d) < 1e-18
    # spot cells: equal power in every lit cell -> uniformity 1
    spots = np.zeros((n, n))
    for a in range(4):
        for b in range(4):
            spots[8 + 16 * b, 8 + 16 * a] = 2.0
    g = {"cols": 4, "rows": 4}
    m4 = oracle.screen_metrics_full(np.sqrt(spots.ravel()), np.zeros(n * n), n, n, d, d, spots.ravel(), None, ill,
                                    flat, d, d, g)
    assert m4["spotUniformity"] == 1 and m4["uniformity"] == 1
    spots[8, 8] = 1.0  # one cell at half power -> 2 min / (max + min) = 2/3
    m5 = oracle.screen_metrics_full(np.sqrt(spots.ravel()), np.zeros(n * n), n, n, d, d, spots.ravel(), None, ill,
                                    flat, d, d, g)
    assert abs(m5["spotUniformity"] - 2 / 3) < 1e-12


def test_error_diffusion_restatement(oracle):
    """src/doe.js:185-226: levels only, the local mean phase kept better than
    rounding (the reference's stated purpose), the square-grid requirement."""
    n = 64
    i = np.arange(n)
    X, Y = np.meshgrid(i, i)
    phi = (0.37 * X + 0.11 * Y + 0.5 * np.sin(X / 5.0)).ravel()  # smooth, wrapping ramp
    q = oracle.error_diffusion(phi, 4)
    step = 2 * np.pi / 4
    k = np.round(q / step)
    assert np.all(np.abs(q - k * step) < 1e-12) and np.all(q > -np.pi) and np.all(q <= np.pi + 1e-12)
    # the phase of the local mean of exp(i phase) (2x2 and 8x8 cells) stays closer to
    # the continuous one than with nearest-level rounding
    r = oracle.quantize_phase(phi, 4)
    for c in (2, 8):
        cell = lambda p: np.exp(1j * p).reshape(n // c, c, n // c, c).mean(axis=(1, 3))
        ref = cell(phi)
        assert np.mean(np.abs(np.angle(cell(q) / ref))) < 0.8 * np.mean(np.abs(np.angle(cell(r) / ref)))
    # identity at a quantised input (no error to diffuse beyond rounding)
    d = oracle.error_diffusion(r, 4) - r
    assert np.max(np.abs(np.angle(np.exp(1j * d)))) < 1e-12
    with pytest.raises(ValueError, match="square"):
        oracle.error_diffusion(np.zeros(50), 4)  # round(sqrt(50)) = 7 does not divide 50
