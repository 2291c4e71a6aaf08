"""Phase retrieval (src/doe.js) on the CUDA engine.

Same names, option objects and result fields as the reference:
``gerchbergSaxton`` (src/doe.js:327-437), ``weightedGerchbergSaxton`` (:455-546),
``fourierCgh`` (:639-730), ``gerchbergSaxtonMultiPlane`` (:557-626), ``designDOE``
(:796-896), ``makeRng`` / ``randomPhase`` / ``flatPhase`` (:65-91),
``illuminationProfile`` (:979-1000).

The iterations run entirely on the GPU; the host only prepares the inputs the
reference prepares (masks, power-matched target amplitude, initial phase). The
``onProgress`` callback is replayed from the per-iteration histories at the
reference's cadence once the device loop has finished.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .field import discMask, rectMask, ringMask

DEFAULT_DESIGN = {
    "lambda": 532e-9,
    "z": 0.03,
    "iterations": 60,
    "seed": 12345,
    "feedback": 0,
    "beta": 0.9,
    "historyEvery": 1,
    "randomRestarts": 1,
    "onProgress": None,
}


# ------------------------------------------------------------------ seeded set-up
def makeRng(seed=1):
    """xorshift32 stream of [0, 1) doubles (src/doe.js:65-75)."""
    s = [(int(math.trunc(seed)) % 4294967296) or 1]

    def nxt():
        x = s[0]
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        s[0] = x
        return x / 4294967296.0

    return nxt


def randomPhase(nx, ny, seed=1) -> np.ndarray:
    """Uniform phase in (-pi, pi] from makeRng(seed) (src/doe.js:81-86)."""
    L = _lib.load_library()
    out = np.empty(nx * ny)
    rc = L.doe_random_phase(int(nx), int(ny), float(seed), _lib.dp(out))
    if rc:
        raise ValueError("randomPhase: bad size")
    return out


def flatPhase(nx, ny) -> np.ndarray:
    return np.zeros(nx * ny)


def wrapPhase(phi):
    """Wrap into (-pi, pi] (src/propagate.js:410-420)."""
    p = np.fmod(np.asarray(phi, dtype=np.float64), 2 * math.pi)
    p = np.where(p > math.pi, p - 2 * math.pi, p)
    return np.where(p <= -math.pi, p + 2 * math.pi, p)


def errorDiffusionQuantize(phi, levels=4, opts=None, *, ctx=None):
    """Floyd-Steinberg error-diffusion quantisation of a wrapped phase (src/doe.js:185-226).

    `phi` is one phase plane or a [B, n] stack (each quantised independently in
    one engine call); options `snake` (default True) and `wrapFirst` (True).
    """
    o = opts or {}
    p = np.ascontiguousarray(phi, dtype=np.float64)
    batch = 1 if p.ndim == 1 else p.shape[0]
    n = p.size // batch
    out = np.empty_like(p)
    c = ctx or _lib.context()
    c.check(c.lib.doe_error_diffusion(c.h, batch, n, int(levels), int(bool(o.get("snake", True))),
                                      int(bool(o.get("wrapFirst", True))), _lib.dp(p), _lib.dp(out)))
    return out


def kinoformLens(nx, ny, dx, dy, lam, f):
    """Wrapped thin-lens phase -k r^2 / (2 f) (src/doe.js:147-151, src/propagate.js:395-407)."""
    k = 2 * math.pi / lam
    x = (np.arange(nx) - nx / 2) * dx
    y = (np.arange(ny) - ny / 2) * dy
    X, Y = np.meshgrid(x, y)
    return wrapPhase(((-k * (X * X + Y * Y)) / (2 * f)).ravel())


def illuminationProfile(type, nx, ny, dx, dy, opts=None):
    """Illumination amplitude on the DOE grid (src/doe.js:979-1000)."""
    opts = opts or {}
    radius = opts.get("radius", (min(nx * dx, ny * dy) / 2) * 0.95)
    ap = discMask(nx, ny, dx, dy, radius, soft=opts.get("soft", 2 * dx))
    if type == "tophat":
        return ap
    if type == "gaussian":
        w = opts.get("waist", radius * 0.6)
        x = (np.arange(nx) - nx / 2) * dx
        y = (np.arange(ny) - ny / 2) * dy
        X, Y = np.meshgrid(x, y)
        return ap * np.exp(-(X * X + Y * Y).ravel() / (w * w))
    if type == "annulus":
        return ringMask(nx, ny, opts.get("inner", 0.6), opts.get("outer", 0.98), soft=0.02)
    if type == "rect":
        return rectMask(nx, ny, dx, dy, opts.get("width", nx * dx * 0.9), opts.get("height", ny * dy * 0.9),
                        soft=2 * dx)
    return ap


def blurRaster(src, nx, ny, sigmaPx=1.0):
    """Separable Gaussian blur with clamped edges (src/doe.js:761-794); target pre-processing."""
    src = np.asarray(src, dtype=np.float64).reshape(ny, nx)
    if sigmaPx <= 0:
        return src.ravel().copy()
    r = max(1, math.ceil(3 * sigmaPx))
    d = np.arange(-r, r + 1)
    k = np.exp(-(d * d) / (2 * sigmaPx * sigmaPx))
    k /= k.sum()
    ix = np.clip(np.arange(nx)[:, None] + d[None, :], 0, nx - 1)
    tmp = (src[:, ix] * k).sum(axis=2)
    iy = np.clip(np.arange(ny)[:, None] + d[None, :], 0, ny - 1)
    out = (tmp[iy, :] * k[None, :, None]).sum(axis=1)
    return out.ravel()


# ------------------------------------------------------------------ device loops
def _nn(d, key, default):
    """The reference's `d.key ?? default`: the default replaces only a missing or
    None entry (an explicit 0 or empty value is kept)."""
    v = d.get(key)
    return default if v is None else v


def _geometry(illumination, o):
    nx = _nn(o, "nx", int(round(math.sqrt(len(illumination)))))
    ny = _nn(o, "ny", nx)
    dx = _nn(o, "dx", 8e-6)
    dy = _nn(o, "dy", dx)
    return int(nx), int(ny), float(dx), float(dy)


def _run(algorithm, illumination, targetAmp, o, ctx=None):
    nx, ny, dx, dy = _geometry(illumination, o)
    n = nx * ny
    it = int(o["iterations"])
    ill = _lib.f64(illumination)
    tgt = _lib.f64(targetAmp)
    if ill.size != n or tgt.size != n:
        raise ValueError(f"designDOE: plane length does not match {nx}x{ny}")
    roi = None if o.get("roi") is None else _lib.f64(o["roi"])
    ip = None if o.get("initPhase") is None else _lib.f64(o["initPhase"])
    d = _lib.DesignDesc(nx, ny, dx, dy, float(o["lambda"]), float(o["z"]), algorithm, it,
                        float(_nn(o, "feedback", 0.0)), int(_nn(o, "escape", 0)), float(_nn(o, "beta", 0.9)),
                        float(_nn(o, "seed", 12345)), _lib.dp(ill), _lib.dp(tgt), _lib.dp(roi), _lib.dp(ip))
    res = {"phase": np.empty(n), "amplitude": np.empty(n), "intensity": np.empty(n),
           "error": np.empty(max(it, 1)), "efficiency": np.empty(max(it, 1))}
    wgs = algorithm in (_lib.DOE_ALG_WGS, _lib.DOE_ALG_WGS_FOURIER)
    if wgs:
        res["weights"] = np.empty(n)
    r = _lib.DesignResult(_lib.dp(res["phase"]), _lib.dp(res["amplitude"]), _lib.dp(res["intensity"]),
                          _lib.dp(res["error"]), _lib.dp(res["efficiency"]), _lib.dp(res.get("weights")), 0.0)
    c = ctx or _lib.context()
    c.check(c.lib.doe_design(c.h, C.byref(d), C.byref(r)))
    out = {"phase": res["phase"], "error": list(res["error"][:it]), "efficiency": list(res["efficiency"][:it]),
           "amplitude": res["amplitude"], "intensity": res["intensity"], "iterations": it, "field": None}
    if wgs:
        out["weights"] = res["weights"]
        out["rmse"] = r.rmse
        out["weightedIterations"] = it
    cb = o.get("onProgress")
    if cb:
        every = _nn(o, "progressEvery", 10)
        for i in range(it):
            if i % every == 0 or i == it - 1:
                cb({"iteration": i, "error": out["error"][i], "efficiency": out["efficiency"][i]})
    return out


def gerchbergSaxton(illumination, targetAmp, opts=None, *, ctx=None):
    """Alternating projections through the angular spectrum (src/doe.js:327-437)."""
    o = {**DEFAULT_DESIGN, **(opts or {})}
    return _run(_lib.DOE_ALG_GS, illumination, targetAmp, o, ctx)


def fourierCgh(illumination, targetAmp, opts=None, *, ctx=None):
    """Far-field (lens focal plane) design with unitary DFTs (src/doe.js:639-730)."""
    o = {**DEFAULT_DESIGN, **(opts or {})}
    return _run(_lib.DOE_ALG_FOURIER, illumination, targetAmp, o, ctx)


def weightedGerchbergSaxton(illumination, targetAmp, opts=None, baseFn=None, *, ctx=None):
    """Weighted GS over gerchbergSaxton (default) or fourierCgh (src/doe.js:455-546)."""
    o = {**DEFAULT_DESIGN, **(opts or {})}
    if baseFn is None or baseFn is gerchbergSaxton:
        alg = _lib.DOE_ALG_WGS
    elif baseFn is fourierCgh:
        alg = _lib.DOE_ALG_WGS_FOURIER
    else:
        raise ValueError("weightedGerchbergSaxton: baseFn must be gerchbergSaxton or fourierCgh")
    if int(o["iterations"]) < 1:
        raise ValueError("weightedGerchbergSaxton: needs at least one iteration")
    return _run(alg, illumination, targetAmp, o, ctx)


def gerchbergSaxtonMultiPlane(illumination, planes, opts=None, *, ctx=None):
    """One element, several target planes along the axis (src/doe.js:557-626)."""
    o = {**DEFAULT_DESIGN, **(opts or {})}
    if len(planes) == 0:
        raise ValueError("gerchbergSaxtonMultiPlane: no planes")
    nx, ny, dx, dy = _geometry(illumination, o)
    n, P, it = nx * ny, len(planes), int(o["iterations"])
    ill = _lib.f64(illumination)
    z = np.array([p["z"] for p in planes], dtype=np.float64)
    tg = _lib.f64(np.concatenate([_lib.f64(p["targetAmp"]) for p in planes]))
    has_roi = [p.get("roi") is not None for p in planes]
    if any(has_roi) and not all(has_roi):
        rois = [(_lib.f64(p["roi"]) if p.get("roi") is not None else np.ones(n)) for p in planes]
    else:
        rois = [_lib.f64(p["roi"]) for p in planes] if all(has_roi) else None
    ro = None if rois is None else _lib.f64(np.concatenate(rois))
    w = np.array([p.get("weight", 1.0) for p in planes], dtype=np.float64)
    ip = None if o.get("initPhase") is None else _lib.f64(o["initPhase"])
    phase = np.empty(n)
    err, eff = np.empty(max(it, 1)), np.empty(max(it, 1))
    ppe = np.empty(P * max(it, 1))
    c = ctx or _lib.context()
    c.check(c.lib.doe_multiplane(c.h, nx, ny, dx, dy, float(o["lambda"]), _lib.dp(ill), P, _lib.dp(z), _lib.dp(tg),
                                 _lib.dp(ro), _lib.dp(w), it, _lib.dp(ip), _lib.dp(phase), _lib.dp(err),
                                 _lib.dp(eff), _lib.dp(ppe)))
    return {"phase": phase, "error": list(err[:it]), "efficiency": list(eff[:it]),
            "perPlaneError": [list(ppe[p * it:(p + 1) * it]) for p in range(P)], "iterations": it}


def _default_disc_target(nx, ny, frac):
    r = frac * min(nx, ny) * 0.5
    i = np.arange(nx) - (nx - 1) / 2
    j = np.arange(ny) - (ny - 1) / 2
    X, Y = np.meshgrid(i, j)
    return (np.hypot(X, Y) <= r).astype(np.float64).ravel()


def prepareTargetAmp(irradiance, illumination):
    """sqrt(max(0, I)) scaled so sum t^2 = sum A^2 (src/doe.js:817-829)."""
    t = np.sqrt(np.maximum(0.0, _lib.f64(irradiance)))
    in_p = float(np.sum(_lib.f64(illumination) ** 2))
    t_p = float(np.sum(t * t))
    return t * math.sqrt(in_p / t_p) if t_p > 0 else t


def designDOE(cfg, *, ctx=None):
    """Design a projection DOE (src/doe.js:796-896)."""
    nx = _nn(cfg, "nx", 256)
    ny = _nn(cfg, "ny", nx)
    dx = _nn(cfg, "dx", 8e-6)
    dy = _nn(cfg, "dy", dx)
    lam = _nn(cfg, "lambda", 532e-9)
    z = _nn(cfg, "z", 0.03)
    mode = _nn(cfg, "mode", "image-plane")
    alg = cfg.get("algorithm")
    algorithm = alg if alg and alg != "auto" else ("gs" if mode == "far-field" else "wgs")  # doe.js:808 (truthy)
    levels = _nn(cfg, "levels", 0)
    iterations = _nn(cfg, "iterations", 60)
    illumination = cfg.get("illumination")
    if illumination is None:
        illumination = discMask(nx, ny, dx, dy, (min(nx * dx, ny * dy) / 2) * 0.95, soft=2 * dx)
    roi = cfg.get("roi")
    target = cfg.get("target")
    if target is None:
        target = _default_disc_target(nx, ny, 0.35)
    if _nn(cfg, "smooth", 0) > 0:
        target = blurRaster(target, nx, ny, cfg["smooth"])
    targetAmp = prepareTargetAmp(target, illumination)
    initPhase = cfg.get("initPhase")
    if initPhase is None:
        init = _nn(cfg, "init", "random")
        if init == "flat":
            initPhase = flatPhase(nx, ny)
        elif init == "lens":
            initPhase = kinoformLens(nx, ny, dx, dy, lam, z)
        else:
            initPhase = randomPhase(nx, ny, _nn(cfg, "seed", 12345))
    common = {
        "nx": nx, "ny": ny, "dx": dx, "dy": dy, "lambda": lam, "z": z, "roi": roi, "iterations": iterations,
        "seed": _nn(cfg, "seed", 12345),
        "feedback": (_nn(cfg, "feedback", 0.8) if algorithm == "hio" else 0),
        "escape": _nn(cfg, "escape", int(math.floor(iterations * 0.2 + 0.5))),
        "beta": _nn(cfg, "beta", 0.9), "initPhase": initPhase, "onProgress": cfg.get("onProgress"),
        "progressEvery": _nn(cfg, "progressEvery", 10),
    }
    if mode == "far-field":
        result = (weightedGerchbergSaxton(illumination, targetAmp, common, fourierCgh, ctx=ctx)
                  if algorithm == "wgs" else fourierCgh(illumination, targetAmp, common, ctx=ctx))
        result["mode"] = "far-field"
    else:
        result = (weightedGerchbergSaxton(illumination, targetAmp, common, ctx=ctx)
                  if algorithm == "wgs" else gerchbergSaxton(illumination, targetAmp, common, ctx=ctx))
        result["mode"] = "image-plane"
    result["algorithm"] = algorithm
    if levels > 1:  # src/doe.js:878-884
        result["phaseContinuous"] = np.array(result["phase"], dtype=np.float64)
        result["phase"] = errorDiffusionQuantize(result["phase"], levels, ctx=ctx)
        result["levels"] = levels
        result["quantized"] = True
    result.update({"illumination": illumination, "targetAmp": targetAmp, "roi": roi, "lambda": lam, "z": z,
                   "nx": nx, "ny": ny, "dx": dx, "dy": dy})
    return result
