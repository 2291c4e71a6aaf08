"""ctypes wrapper over the FP64 C oracle (``oracle/libdoe_oracle.so``).

TEST INFRASTRUCTURE ONLY. Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module, always as the checker or
as the timed CPU baseline, never as part of the product path.

The C library restates the reference's JavaScript loops in FP64 with the same
operation order (see the file:line citations in ``oracle/doe_oracle.c``). The
Python helpers below only marshal arrays, plus the few host-side set-up steps of
``designDOE`` (src/doe.js:796-896), which are done in C as well so that their
sequential sums match the reference's.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdoe_oracle.so")
_lib = None

_dp = C.POINTER(C.c_double)


def build() -> str:
    """Compile the oracle with its Makefile (no -ffast-math)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class DesignOpts(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("lambda_", C.c_double), ("z", C.c_double),
        ("iterations", C.c_int),
        ("feedback", C.c_double),
        ("escape", C.c_int),
        ("beta", C.c_double),
        ("seed", C.c_double),
        ("roi", _dp), ("weights", _dp), ("init_phase", _dp),
    ]


class DesignResult(C.Structure):
    _fields_ = [
        ("phase", _dp), ("amplitude", _dp), ("intensity", _dp),
        ("error", _dp), ("efficiency", _dp), ("weights", _dp),
        ("rmse", C.c_double),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        i, d, l = C.c_int, C.c_double, C.c_long
        L.orc_fft1d.argtypes = [_dp, _dp, i, l, l, i]
        L.orc_fft2d.argtypes = [_dp, _dp, i, i, i]
        L.orc_fftshift2d.argtypes = [_dp, _dp, i, i, i]
        L.orc_dft2d_naive.argtypes = [_dp, _dp, i, i, i, _dp, _dp]
        L.orc_local_frequency_limit.argtypes = [i, d, d, d]
        L.orc_local_frequency_limit.restype = d
        L.orc_asm_transfer.argtypes = [i, i, d, d, d, d, i, i, d, _dp, _dp]
        L.orc_asm_transfer.restype = d
        L.orc_asm_inplace.argtypes = [_dp, _dp, i, i, d, d, d, d, i, i, d]
        L.orc_focal_plane.argtypes = [_dp, _dp, i, i, d, d, d, d, _dp, _dp, _dp]
        L.orc_fresnel_fft.argtypes = [_dp, _dp, i, i, d, d, d, d, _dp, _dp, _dp]
        L.orc_fresnel_fft_inverse.argtypes = [_dp, _dp, i, i, d, d, d, d, d, d, _dp, _dp]
        L.orc_disc_mask.argtypes = [i, i, d, d, d, d, d, d, _dp]
        L.orc_rect_mask.argtypes = [i, i, d, d, d, d, d, _dp]
        L.orc_rng_seed.argtypes = [d]
        L.orc_rng_seed.restype = C.c_uint32
        L.orc_rng_next.argtypes = [C.POINTER(C.c_uint32)]
        L.orc_rng_next.restype = d
        L.orc_random_phase.argtypes = [i, i, d, _dp]
        L.orc_gerchberg_saxton.argtypes = [_dp, _dp, C.POINTER(DesignOpts), C.POINTER(DesignResult)]
        L.orc_fourier_cgh.argtypes = [_dp, _dp, C.POINTER(DesignOpts), C.POINTER(DesignResult)]
        L.orc_weighted_gs.argtypes = [_dp, _dp, C.POINTER(DesignOpts), i, C.POINTER(DesignResult)]
        L.orc_weighted_gs_goal.argtypes = [_dp, _dp, C.POINTER(DesignOpts), _dp, d, C.POINTER(i),
                                           C.POINTER(DesignResult)]
        L.orc_gs_multiplane.argtypes = [_dp, i, _dp, _dp, _dp, _dp, C.POINTER(DesignOpts),
                                        _dp, _dp, _dp, _dp]
        L.orc_auto_roi.argtypes = [_dp, i, i, d, d, d, _dp]
        L.orc_screen_metrics.argtypes = [_dp, _dp, i, i, d, d, _dp, _dp, _dp, d, d, _dp]
        L.orc_quantize_phase.argtypes = [_dp, C.c_long, i, _dp]
        L.orc_error_diffusion.argtypes = [_dp, C.c_long, i, i, i, _dp]
        L.orc_screen_metrics_full.argtypes = [_dp, _dp, i, i, d, d, _dp, _dp, _dp, _dp, d, d, i, i, _dp]
        L.orc_prepare_target.argtypes = [_dp, _dp, C.c_long, _dp]
        L.orc_modal_intensity.argtypes = [i, _dp, _dp, C.c_long, _dp, _dp]
        L.orc_record_hologram.argtypes = [_dp, _dp, _dp, _dp, C.c_long, i, i, _dp, _dp, _dp, _dp, _dp]
        L.orc_reconstruct_hologram.argtypes = [_dp, _dp, _dp, _dp, i, i, d, d, d, d, i, i, d] + [_dp] * 6
        L.orc_partially_coherent_modes.argtypes = [i, i, d, d, i, d, d, d, _dp, _dp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------- fft.js
def fft2d(re, im, nx, ny, inverse=False):
    """In-place semantics of src/fft.js:148-154, returned as new arrays."""
    r, i = _f64(re).copy(), _f64(im).copy()
    if lib().orc_fft2d(_p(r), _p(i), nx, ny, int(inverse)):
        raise ValueError("fft2d: non power-of-two grid")
    return r, i


def fft1d(re, im, inverse=False):
    r, i = _f64(re).copy(), _f64(im).copy()
    if lib().orc_fft1d(_p(r), _p(i), r.size, 1, 0, int(inverse)):
        raise ValueError("fft1d: length must be a power of two")
    return r, i


def fftshift2d(re, im, nx, ny, shift=True):
    r, i = _f64(re).copy(), _f64(im).copy()
    lib().orc_fftshift2d(_p(r), _p(i), nx, ny, int(shift))
    return r, i


def dft2d_naive(re, im, nx, ny, inverse=False):
    r, i = _f64(re), _f64(im)
    orr, oi = np.empty(nx * ny), np.empty(nx * ny)
    lib().orc_dft2d_naive(_p(r), _p(i), nx, ny, int(inverse), _p(orr), _p(oi))
    return orr, oi


# ---------------------------------------------------------------- propagate.js
def local_frequency_limit(n, d, lam, z):
    return lib().orc_local_frequency_limit(n, d, lam, z)


def asm_transfer(nx, ny, dx, dy, lam, z, band_limit=True, evanescent=True, soft_edge=0.02):
    hr, hi = np.empty(nx * ny), np.empty(nx * ny)
    frac = lib().orc_asm_transfer(nx, ny, dx, dy, lam, z, int(band_limit), int(evanescent),
                                  soft_edge, _p(hr), _p(hi))
    return hr, hi, frac


def asm(re, im, nx, ny, dx, dy, lam, z, band_limit=True, evanescent=True, soft_edge=0.02):
    """propagateAngularSpectrum (src/propagate.js:105-133) on copies."""
    r, i = _f64(re).copy(), _f64(im).copy()
    lib().orc_asm_inplace(_p(r), _p(i), nx, ny, dx, dy, lam, z, int(band_limit),
                          int(evanescent), soft_edge)
    return r, i


def focal_plane(re, im, nx, ny, dx, dy, lam, f):
    r, i = _f64(re), _f64(im)
    orr, oi, d = np.empty(nx * ny), np.empty(nx * ny), np.empty(2)
    lib().orc_focal_plane(_p(r), _p(i), nx, ny, dx, dy, lam, f, _p(orr), _p(oi), _p(d))
    return orr, oi, float(d[0]), float(d[1])


def fresnel(re, im, nx, ny, dx, dy, lam, z):
    r, i = _f64(re), _f64(im)
    orr, oi, d = np.empty(nx * ny), np.empty(nx * ny), np.empty(2)
    lib().orc_fresnel_fft(_p(r), _p(i), nx, ny, dx, dy, lam, z, _p(orr), _p(oi), _p(d))
    return orr, oi, float(d[0]), float(d[1])


def fresnel_inverse(re, im, nx, ny, dux, duy, lam, z, dx, dy):
    r, i = _f64(re), _f64(im)
    orr, oi = np.empty(nx * ny), np.empty(nx * ny)
    lib().orc_fresnel_fft_inverse(_p(r), _p(i), nx, ny, dux, duy, lam, z, dx, dy, _p(orr), _p(oi))
    return orr, oi


# ---------------------------------------------------------------- field.js / doe.js helpers
def disc_mask(nx, ny, dx, dy, radius, soft=0.0, cx=0.0, cy=0.0):
    out = np.empty(nx * ny)
    lib().orc_disc_mask(nx, ny, dx, dy, radius, soft, cx, cy, _p(out))
    return out


def rect_mask(nx, ny, dx, dy, width, height, soft=0.0):
    out = np.empty(nx * ny)
    lib().orc_rect_mask(nx, ny, dx, dy, width, height, soft, _p(out))
    return out


def random_phase(nx, ny, seed=1):
    out = np.empty(nx * ny)
    lib().orc_random_phase(nx, ny, float(seed), _p(out))
    return out


class Rng:
    """src/doe.js:65-75 makeRng."""

    def __init__(self, seed=1):
        self._s = C.c_uint32(lib().orc_rng_seed(float(seed)))

    def __call__(self):
        return lib().orc_rng_next(C.byref(self._s))


def auto_roi(irr, nx, ny, dilate=2, soft=2, threshold=0.05):
    out = np.empty(nx * ny)
    lib().orc_auto_roi(_p(_f64(irr)), nx, ny, dilate, soft, threshold, _p(out))
    return out


def prepare_target(irradiance, illumination):
    """designDOE target amplitude + power match (src/doe.js:817-829)."""
    irr, ill = _f64(irradiance), _f64(illumination)
    out = np.empty(irr.size)
    lib().orc_prepare_target(_p(irr), _p(ill), irr.size, _p(out))
    return out


def screen_metrics(fre, fim, nx, ny, sdx, sdy, target_irr, roi, illumination, dx, dy):
    out = np.empty(6)
    lib().orc_screen_metrics(_p(_f64(fre)), _p(_f64(fim)), nx, ny, sdx, sdy,
                             _p(_f64(target_irr)), _p(None if roi is None else _f64(roi)),
                             _p(_f64(illumination)), dx, dy, _p(out))
    keys = ["rmse", "efficiency", "fluxFraction", "powerInSignal", "powerAtScreen",
            "powerIncident"]
    return dict(zip(keys, out.tolist()))


def quantize_phase(phi, levels=4):
    """quantizePhase (src/doe.js:164-173)."""
    p = _f64(phi)
    out = np.empty(p.size)
    lib().orc_quantize_phase(_p(p), p.size, levels, _p(out))
    return out


def error_diffusion(phi, levels=4, snake=True, wrap_first=True):
    """errorDiffusionQuantize (src/doe.js:185-226)."""
    p = _f64(phi)
    out = np.empty(p.size)
    if lib().orc_error_diffusion(_p(p), p.size, levels, int(snake), int(wrap_first), _p(out)):
        raise ValueError("errorDiffusionQuantize: expected a square grid")
    return out


FULL_METRIC_KEYS = ["efficiency", "fluxFraction", "uniformity", "spotUniformity", "flatness", "contrast", "rmse",
                    "fidelity", "correlation", "ssim", "snr", "zeroOrder", "rmsRadius", "meanIntensity",
                    "peakIntensity", "powerInSignal", "powerAtScreen", "powerIncident"]


def screen_metrics_full(fre, fim, nx, ny, sdx, sdy, target_irr, roi, illumination, phase, dx, dy, grid=None):
    """ProjectorSystem.screenMetrics, every field (src/projector.js:554-614)."""
    out = np.empty(18)
    gc, gr = (grid["cols"], grid["rows"]) if grid else (0, 0)
    lib().orc_screen_metrics_full(_p(_f64(fre)), _p(_f64(fim)), nx, ny, sdx, sdy, _p(_f64(target_irr)),
                                  _p(None if roi is None else _f64(roi)), _p(_f64(illumination)),
                                  _p(_f64(phase)), dx, dy, gc, gr, _p(out))
    d = dict(zip(FULL_METRIC_KEYS, out.tolist()))
    if not grid:
        d["spotUniformity"] = None
    return d


# ---------------------------------------------------------------- design loops
def _opts(nx, ny, dx, dy, lam, z, iterations, feedback=0.0, escape=0, beta=0.9, seed=12345,
          roi=None, weights=None, init_phase=None):
    keep = [a for a in (roi, weights, init_phase) if a is not None]
    o = DesignOpts(nx, ny, dx, dy, lam, z, iterations, feedback, escape, beta, float(seed),
                   _p(roi), _p(weights), _p(init_phase))
    return o, keep


def design(algorithm, illumination, target_amp, *, nx, ny, dx, dy=None, lam=532e-9, z=0.03,
           iterations=60, feedback=0.0, escape=0, beta=0.9, seed=12345, roi=None,
           weights=None, init_phase=None, rmse_goal=0.0, screen_irr=None):
    """Run gs / wgs / fourier / wgs-fourier with the reference's semantics.

    algorithm: 'gs' (src/doe.js:327), 'fourier' (:639), 'wgs' (:455 over gs),
    'wgs-fourier' (:455 over fourierCgh). rmse_goal > 0 ('wgs' only) stops at the
    first iteration whose screen RMSE meets it (the engine's stopping rule) and
    reports `iterationsUsed`.
    """
    dy = dx if dy is None else dy
    ill, tgt = _f64(illumination), _f64(target_amp)
    roi = None if roi is None else _f64(roi)
    weights = None if weights is None else _f64(weights)
    init_phase = None if init_phase is None else _f64(init_phase)
    o, keep = _opts(nx, ny, dx, dy, lam, z, iterations, feedback, escape, beta, seed, roi,
                    weights, init_phase)
    n = nx * ny
    nit = max(iterations, 1)
    res = dict(phase=np.empty(n), amplitude=np.empty(n), intensity=np.empty(n),
               error=np.empty(nit), efficiency=np.empty(nit))
    wts = np.empty(n) if algorithm.startswith("wgs") else None
    r = DesignResult(_p(res["phase"]), _p(res["amplitude"]), _p(res["intensity"]),
                     _p(res["error"]), _p(res["efficiency"]), _p(wts), 0.0)
    L = lib()
    if algorithm == "gs":
        rc = L.orc_gerchberg_saxton(_p(ill), _p(tgt), C.byref(o), C.byref(r))
    elif algorithm == "fourier":
        rc = L.orc_fourier_cgh(_p(ill), _p(tgt), C.byref(o), C.byref(r))
    elif algorithm == "wgs" and rmse_goal > 0:
        used = C.c_int(0)
        sirr = None if screen_irr is None else _f64(screen_irr)
        rc = L.orc_weighted_gs_goal(_p(ill), _p(tgt), C.byref(o), _p(sirr), float(rmse_goal), C.byref(used),
                                    C.byref(r))
        res["iterationsUsed"] = used.value
    elif algorithm in ("wgs", "wgs-fourier"):
        rc = L.orc_weighted_gs(_p(ill), _p(tgt), C.byref(o), int(algorithm == "wgs-fourier"),
                               C.byref(r))
    else:
        raise ValueError(algorithm)
    del keep
    if rc:
        raise RuntimeError(f"oracle design failed ({rc})")
    res["error"] = res["error"][:iterations]
    res["efficiency"] = res["efficiency"][:iterations]
    if wts is not None:
        res["weights"] = wts
        res["rmse"] = r.rmse
    return res


def multiplane(illumination, zs, target_amps, rois, weights, *, nx, ny, dx, dy=None,
               lam=532e-9, iterations=60, init_phase=None):
    """src/doe.js:557-626."""
    dy = dx if dy is None else dy
    P = len(zs)
    ill = _f64(illumination)
    z = _f64(zs)
    tg = _f64(np.concatenate([_f64(t) for t in target_amps]))
    ro = None if rois is None else _f64(np.concatenate([_f64(r) for r in rois]))
    w = _f64(weights if weights is not None else np.ones(P))
    ip = None if init_phase is None else _f64(init_phase)
    o, keep = _opts(nx, ny, dx, dy, lam, 0.0, iterations, init_phase=ip)
    phase = np.empty(nx * ny)
    err, eff = np.empty(max(iterations, 1)), np.empty(max(iterations, 1))
    ppe = np.empty(P * max(iterations, 1))
    rc = lib().orc_gs_multiplane(_p(ill), P, _p(z), _p(tg), _p(ro), _p(w), C.byref(o),
                                 _p(phase), _p(err), _p(eff), _p(ppe))
    del keep
    if rc:
        raise RuntimeError(f"oracle multiplane failed ({rc})")
    return dict(phase=phase, error=err[:iterations], efficiency=eff[:iterations],
                perPlaneError=ppe.reshape(P, -1)[:, :iterations])


def modal_intensity(re, im, n, weights=None):
    """modalIntensity (src/interference.js:57-69) of modes [M][n]."""
    r, i = _f64(re), _f64(im)
    M = r.size // n
    w = None if weights is None else _f64(weights)
    out = np.empty(n)
    lib().orc_modal_intensity(M, _p(r), _p(i), n, _p(w), _p(out))
    return out


HOLOGRAM_ENCODINGS = {"raw": 0, "binary": 1, "phase": 2}


def record_hologram(obj_re, obj_im, ref_re, ref_im, encode="raw", levels=0):
    """recordHologram (src/interference.js:347-388) -> dict of plate/recorded/sum planes."""
    a = [_f64(v) for v in (obj_re, obj_im, ref_re, ref_im)]
    n = a[0].size
    out = {k: np.empty(n) for k in ("plate_re", "plate_im", "recorded", "sum_re", "sum_im")}
    lib().orc_record_hologram(*[_p(v) for v in a], n, HOLOGRAM_ENCODINGS[encode], int(levels),
                              *[_p(out[k]) for k in ("plate_re", "plate_im", "recorded", "sum_re", "sum_im")])
    return out


def reconstruct_hologram(plate_re, plate_im, ref_re, ref_im, nx, ny, dx, dy, lam, z, band_limit=False,
                         evanescent=True, soft_edge=0.02):
    """reconstructHologram (src/interference.js:397-411), bandLimit false by default as there."""
    a = [_f64(v) for v in (plate_re, plate_im, ref_re, ref_im)]
    n = nx * ny
    keys = ("real_re", "real_im", "virt_re", "virt_im", "illum_re", "illum_im")
    out = {k: np.empty(n) for k in keys}
    lib().orc_reconstruct_hologram(*[_p(v) for v in a], nx, ny, dx, dy, lam, z, int(band_limit),
                                   int(evanescent), soft_edge, *[_p(out[k]) for k in keys])
    return out


def partially_coherent_modes(nx, ny, dx, dy, modes=8, sigma=40e-6, waist=1e-3, seed=7):
    """partiallyCoherentModes (src/interference.js:79-125) -> (re, im) of shape [modes, nx*ny]."""
    n = nx * ny
    re, im = np.empty(modes * n), np.empty(modes * n)
    lib().orc_partially_coherent_modes(nx, ny, dx, dy, modes, sigma, waist, float(seed), _p(re), _p(im))
    return re.reshape(modes, n), im.reshape(modes, n)
