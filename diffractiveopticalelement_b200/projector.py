"""The projection pipeline (src/projector.js) on the CUDA engine.

``ProjectorSystem`` keeps the reference's constructor options, ``design()``,
``simulate()``, ``screenMetrics()`` (radiometric subset: rmse, efficiency,
fluxFraction, powers, snr), ``designMultiPlane()``, ``defocusCurve()``,
``focusStack()`` and ``matchDistance()``. Targets and ROIs are host set-up
(``makeTarget``, ``autoRoi``) exactly as the reference prepares them; designing,
propagating and measuring run on the GPU.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from .doe import designDOE, errorDiffusionQuantize, gerchbergSaxtonMultiPlane, illuminationProfile, makeRng
from .field import ComplexField

DEFAULT_PROJECTOR = {
    "n": 256, "pitch": 8e-6, "lambda": 532e-9, "distance": 0.03, "aperture": 0.95, "apodization": 2,
    "source": "tophat", "waist": 0.6, "inner": 0.6, "outer": 0.98,
    "mode": "image-plane", "algorithm": "auto", "iterations": 60, "levels": 0, "seed": 12345, "quantize": False,
    "target": {"kind": "disc"},
}


def _window_any(b, r, axis):
    """1 where any sample within +-r along `axis` is set (clamped at the edges)."""
    n = b.shape[axis]
    c = np.cumsum(np.concatenate([np.zeros_like(np.take(b, [0], axis=axis)), b], axis=axis), axis=axis)
    idx = np.arange(n)
    lo = np.clip(idx - r, 0, n)
    hi = np.clip(idx + r + 1, 0, n)
    s = np.take(c, hi, axis=axis) - np.take(c, lo, axis=axis)
    return (s > 0).astype(np.float64)


def autoRoi(irr, nx, ny, opts=None):
    """Dilated, box-softened support of the target (src/projector.js:262-315)."""
    opts = opts or {}
    dilate, soft, threshold = opts.get("dilate", 2), opts.get("soft", 2), opts.get("threshold", 0.05)
    a = np.asarray(irr, dtype=np.float64).reshape(ny, nx)
    mx = max(0.0, float(a.max()))
    b = (a > threshold * mx).astype(np.float64)
    r = max(1, int(math.floor(dilate + 0.5)))
    dil = _window_any(_window_any(b, r, 1), r, 0)
    if soft <= 0:
        return dil.ravel()
    s = max(1, int(math.floor(soft + 0.5)))
    pad = np.pad(dil, s)
    ones = np.pad(np.ones_like(dil), s)
    c = np.zeros((ny + 2 * s + 1, nx + 2 * s + 1))
    c[1:, 1:] = np.cumsum(np.cumsum(pad, 0), 1)
    k = np.zeros_like(c)
    k[1:, 1:] = np.cumsum(np.cumsum(ones, 0), 1)
    w = 2 * s + 1

    def box(C):
        return C[w:, w:] - C[:-w, w:] - C[w:, :-w] + C[:-w, :-w]

    return (box(c) / box(k)).ravel()


def rectangles_target(nx, ny, seed, window=128, count=(3, 8), width=(4, 40)):
    """Seeded binary mask of axis-aligned rectangles inside the central window.

    Not a reference target kind: the benchmark's image-plane workload passes it as
    a custom irradiance (src/projector.js:369-374). Drawn from makeRng(seed).
    """
    rng = makeRng(seed)
    irr = np.zeros((ny, nx))
    wx, wy = min(window, nx), min(window, ny)
    x0w, y0w = (nx - wx) // 2, (ny - wy) // 2
    k = count[0] + int(rng() * (count[1] - count[0] + 1))
    for _ in range(k):
        w = min(wx, width[0] + int(rng() * (width[1] - width[0] + 1)))
        h = min(wy, width[0] + int(rng() * (width[1] - width[0] + 1)))
        x0 = x0w + int(rng() * (wx - w + 1))
        y0 = y0w + int(rng() * (wy - h + 1))
        irr[y0:y0 + h, x0:x0 + w] = 1.0
    return irr.ravel()


def makeTarget(kind, nx, ny, opts=None):
    """Projection targets (src/projector.js:169-255) with their auto ROI."""
    opts = opts or {}
    cx, cy = (nx - 1) / 2, (ny - 1) / 2
    I, J = np.meshgrid(np.arange(nx), np.arange(ny))
    name = kind
    if kind == "disc":
        r = opts.get("radius", 0.35) * min(nx, ny) * 0.5
        irr = (np.hypot(I - cx, J - cy) <= r).astype(np.float64)
    elif kind == "ring":
        r0 = opts.get("inner", 0.25) * min(nx, ny) * 0.5
        r1 = opts.get("outer", 0.4) * min(nx, ny) * 0.5
        r = np.hypot(I - cx, J - cy)
        irr = ((r >= r0) & (r <= r1)).astype(np.float64)
    elif kind in ("dots", "grid"):
        cols, rows = opts.get("cols", 8), opts.get("rows", 8)
        px, py = nx / cols, ny / rows
        sigma = opts.get("sigma", 0.22) * min(px, py)
        fy = np.fmod((J + 0.5) / py, 1) - 0.5
        fx = np.fmod((I + 0.5) / px, 1) - 0.5
        irr = np.exp(-((fx * px) ** 2 + (fy * py) ** 2) / (2 * sigma * sigma))
        for mi, mj in opts.get("missing", []):
            irr[((I / px).astype(int) == mi) & ((J / py).astype(int) == mj)] = 0.0
    elif kind == "checker":
        cells = opts.get("cells", 8)
        u = np.floor((I / nx) * cells)
        v = np.floor((J / ny) * cells)
        irr = ((u + v) % 2 == 0).astype(np.float64)
    elif kind == "lines":
        period, duty = opts.get("period", 12), opts.get("duty", 0.5)
        irr = (((I % period) / period) < duty).astype(np.float64)
    elif kind == "zone":
        period = opts.get("period", 16)
        r = np.hypot(I - cx, J - cy)
        irr = (np.sin((np.pi * r * r) / period) > 0).astype(np.float64)
    elif kind == "rects":
        irr = rectangles_target(nx, ny, opts.get("seed", 1)).reshape(ny, nx)
        name = f"rects:{opts.get('seed', 1)}"
    elif kind in ("text", "image"):
        raise NotImplementedError(f'makeTarget("{kind}"): raster/text targets are host-side image preparation '
                                  "outside this engine; pass {irradiance} instead")
    else:
        raise ValueError(f'makeTarget: unknown kind "{kind}"')
    irr = irr.ravel().astype(np.float64)
    roi = opts.get("roi")
    if roi is None:
        roi = autoRoi(irr, nx, ny, {"dilate": opts.get("dilate", 2), "soft": opts.get("softEdge", 2)})
    grid = {"cols": opts.get("cols", 8), "rows": opts.get("rows", 8)} if kind in ("dots", "grid") else None
    return {"irradiance": irr, "roi": roi, "name": name, "grid": grid}


# field order of doe_screen_metrics_full (the reference's screenMetrics keys)
SCREEN_METRIC_KEYS = ["efficiency", "fluxFraction", "uniformity", "spotUniformity", "flatness", "contrast", "rmse",
                      "fidelity", "correlation", "ssim", "snr", "zeroOrder", "rmsRadius", "meanIntensity",
                      "peakIntensity", "powerInSignal", "powerAtScreen", "powerIncident"]


class ProjectorSystem:
    """src/projector.js:345-718."""

    def __init__(self, cfg=None, *, ctx=None):
        cfg = dict(cfg or {})
        tgt = {**DEFAULT_PROJECTOR["target"], **(cfg.get("target") or {})}
        self.cfg = {**DEFAULT_PROJECTOR, **cfg, "target": tgt}
        self.ctx = ctx
        self.nx = self.ny = int(self.cfg["n"])
        self.dx = self.dy = float(self.cfg["pitch"])
        self.lam = float(self.cfg["lambda"])
        if cfg.get("distance") is None and self.cfg["mode"] == "far-field":
            self.cfg["distance"] = (self.cfg["n"] * self.cfg["pitch"] ** 2) / self.cfg["lambda"]
        self.z = float(self.cfg["distance"])
        self.target = None
        self.result = None
        self.setTarget(self.cfg["target"])

    @property
    def lambda_(self):
        return self.lam

    def setTarget(self, spec):
        if spec and spec.get("irradiance") is not None:
            irr = np.asarray(spec["irradiance"], dtype=np.float64)
            roi = spec.get("roi")
            self.target = {"irradiance": irr, "roi": autoRoi(irr, self.nx, self.ny) if roi is None else roi,
                           "name": spec.get("name", "custom"), "grid": None}
        else:
            self.target = makeTarget(spec["kind"], self.nx, self.ny, spec)
        return self.target

    def matchDistance(self):
        return (self.nx * self.dx * self.dx) / self.lam

    def illumination(self):
        radius = (min(self.nx * self.dx, self.ny * self.dy) / 2) * self.cfg["aperture"]
        opts = {"radius": radius, "soft": self.cfg["apodization"] * self.dx, "waist": radius * self.cfg["waist"],
                "inner": self.cfg.get("inner", 0.6), "outer": self.cfg.get("outer", 0.98)}
        return illuminationProfile(self.cfg["source"], self.nx, self.ny, self.dx, self.dy, opts)

    def design(self, opts=None):
        opts = opts or {}
        it = opts.get("iterations", self.cfg["iterations"])
        result = designDOE({
            "nx": self.nx, "ny": self.ny, "dx": self.dx, "dy": self.dy, "lambda": self.lam, "z": self.z,
            "mode": self.cfg["mode"], "algorithm": self.cfg["algorithm"], "iterations": it,
            "levels": opts.get("levels", self.cfg["levels"]), "seed": opts.get("seed", self.cfg["seed"]),
            "illumination": self.illumination(), "target": self.target["irradiance"], "roi": self.target["roi"],
            "onProgress": opts.get("onProgress"), "progressEvery": opts.get("progressEvery", 10),
            "beta": opts.get("beta", 0.9), "escape": opts.get("escape"), "initPhase": opts.get("initPhase"),
        }, ctx=self.ctx)
        result["iterations"] = it
        result["target"] = self.target
        self.result = result
        return result

    def simulate(self, opts=None):
        opts = opts or {}
        if self.result is None:
            raise RuntimeError("ProjectorSystem.simulate: call design() first")
        z = opts.get("z")
        dist = self.z if z is None else z
        mode = opts.get("mode") or self.cfg["mode"]
        phase = opts.get("phase")
        phase = self.result["phase"] if phase is None else phase
        far = mode == "far-field"
        if far and not dist > 0:
            raise ValueError("ProjectorSystem.simulate: far-field mode needs a positive throw")
        out = ComplexField(self.nx, self.ny, self.dx, self.dy)
        d = np.zeros(2)
        c = self.ctx or _lib.context()
        c.check(c.lib.doe_simulate(c.h, _lib.dp(_lib.f64(self.result["illumination"])), _lib.dp(_lib.f64(phase)),
                                   self.nx, self.ny, self.dx, self.dy, self.lam, float(dist),
                                   int(bool(opts.get("bandLimit", False))), int(far), int(opts.get("pad", 1)),
                                   _lib.dp(out.re), _lib.dp(out.im), _lib.dp(d)))
        out.dx, out.dy = float(d[0]), float(d[1])
        return out

    def screenMetrics(self, field, opts=None):
        """src/projector.js:554-614: every field, from three FP64 passes on the GPU
        (doe_screen_metrics_full). The zero-order leak is measured on the element
        field illumination * exp(i phase), phase = opts["phase"] or the design's."""
        opts = opts or {}
        tgt = opts.get("target") or self.target
        roi = opts.get("roi")
        mask = tgt["roi"] if roi is None else roi
        phase = opts.get("phase")
        if phase is None:
            if self.result is None:
                raise ValueError("ProjectorSystem.screenMetrics: call design() first (or pass {phase})")
            phase = self.result["phase"]
        ill = self.result["illumination"] if self.result is not None else self.illumination()
        grid = tgt.get("grid")
        out = np.zeros(18)
        c = self.ctx or _lib.context()
        c.check(c.lib.doe_screen_metrics_full(
            c.h, _lib.dp(field.re), _lib.dp(field.im), field.nx, field.ny, field.dx, field.dy,
            _lib.dp(_lib.f64(tgt["irradiance"])), _lib.dp(None if mask is None else _lib.f64(mask)),
            _lib.dp(_lib.f64(ill)), _lib.dp(_lib.f64(phase)), self.dx, self.dy,
            int(grid["cols"]) if grid else 0, int(grid["rows"]) if grid else 0, _lib.dp(out)))
        m = dict(zip(SCREEN_METRIC_KEYS, (float(v) for v in out)))
        if not grid:
            m["spotUniformity"] = None
        return m

    def simulateMany(self, zs, opts=None):
        """simulate (src/projector.js:475-498) at every distance of `zs` in one engine
        call (doe_simulate_sweep): the element's forward transform is shared."""
        opts = opts or {}
        if self.result is None:
            raise RuntimeError("ProjectorSystem.simulate: call design() first")
        zs = np.ascontiguousarray([self.z if z is None else z for z in zs], dtype=np.float64)
        mode = opts.get("mode") or self.cfg["mode"]
        phase = opts.get("phase")
        phase = self.result["phase"] if phase is None else phase
        far = mode == "far-field"
        n = self.nx * self.ny
        re = np.empty(zs.size * n)
        im = np.empty(zs.size * n)
        d = np.zeros(2 * zs.size)
        c = self.ctx or _lib.context()
        c.check(c.lib.doe_simulate_sweep(c.h, _lib.dp(_lib.f64(self.result["illumination"])),
                                         _lib.dp(_lib.f64(phase)), self.nx, self.ny, self.dx, self.dy, self.lam,
                                         _lib.dp(zs), int(zs.size), int(bool(opts.get("bandLimit", False))),
                                         int(far), int(opts.get("pad", 1)), _lib.dp(re), _lib.dp(im), _lib.dp(d)))
        out = []
        for k in range(zs.size):
            f = ComplexField(self.nx, self.ny, float(d[2 * k]), float(d[2 * k + 1]))
            f.re = re[k * n:(k + 1) * n]
            f.im = im[k * n:(k + 1) * n]
            out.append(f)
        return out

    def defocusCurve(self, opts=None):
        """src/projector.js:622-642; the planes come from one simulateMany call."""
        opts = opts or {}
        points, span = opts.get("points", 21), opts.get("span", 0.6)
        z0, z1 = self.z * (1 - span), self.z * (1 + span)
        zs = [z0 + ((z1 - z0) * i) / (points - 1) for i in range(points)]
        fields = self.simulateMany(zs, {"pad": opts.get("pad", 2), "mode": opts.get("mode")})
        out = []
        for z, field in zip(zs, fields):
            m = self.screenMetrics(field)
            out.append({"z": z, "zMm": z * 1e3, "fidelity": m["fidelity"], "correlation": m["correlation"],
                        "ssim": m["ssim"], "rmse": m["rmse"], "efficiency": m["efficiency"],
                        "uniformity": m["uniformity"]})
        return out

    def focusStack(self, opts=None):
        """src/projector.js:645-653; the planes come from one simulateMany call."""
        opts = opts or {}
        points, span = opts.get("points", 9), opts.get("span", 0.5)
        zs = [self.z * (1 - span) + (self.z * 2 * span * i) / (points - 1) for i in range(points)]
        fields = self.simulateMany(zs, {"pad": opts.get("pad", 2), "mode": opts.get("mode")})
        return [{"z": z, "intensity": f.intensity()} for z, f in zip(zs, fields)]

    def designMultiPlane(self, planeSpecs, opts=None):
        """src/projector.js:675-712."""
        opts = opts or {}
        illumination = self.illumination()
        planes = []
        for p in planeSpecs:
            t = p if p.get("irradiance") is not None else makeTarget(p["kind"], self.nx, self.ny, p)
            amp = np.sqrt(np.maximum(0.0, np.asarray(t["irradiance"], dtype=np.float64)))
            roi = t.get("roi")
            planes.append({"z": p["z"], "targetAmp": amp,
                           "roi": autoRoi(t["irradiance"], self.nx, self.ny) if roi is None else roi,
                           "weight": p.get("weight", 1)})
        res = gerchbergSaxtonMultiPlane(illumination, planes, {
            "nx": self.nx, "ny": self.ny, "dx": self.dx, "dy": self.dy, "lambda": self.lam,
            "iterations": opts.get("iterations", self.cfg["iterations"]), "seed": opts.get("seed", self.cfg["seed"]),
            "initPhase": opts.get("initPhase"), "onProgress": opts.get("onProgress")}, ctx=self.ctx)
        out = {**res, "illumination": illumination, "lambda": self.lam, "nx": self.nx, "ny": self.ny,
               "dx": self.dx, "dy": self.dy, "z": self.z, "mode": "multi-plane", "planes": planes,
               "target": self.target, "roi": self.target["roi"]}
        levels = opts.get("levels", self.cfg["levels"]) or 0
        if levels > 1:  # src/projector.js:708
            out["phase"] = errorDiffusionQuantize(out["phase"], levels, ctx=self.ctx)
        self.result = out
        return out


def resample_centred(field: ComplexField, nx2: int, ny2: int) -> ComplexField:
    """Integer zero-pad / centre-crop (src/field.js:443-461), a host container copy."""
    out = ComplexField(nx2, ny2, field.dx, field.dy)
    ox, oy = (nx2 - field.nx) // 2, (ny2 - field.ny) // 2
    src_r = field.re.reshape(field.ny, field.nx)
    src_i = field.im.reshape(field.ny, field.nx)
    dr = out.re.reshape(ny2, nx2)
    di = out.im.reshape(ny2, nx2)
    y0, y1 = max(0, oy), min(ny2, oy + field.ny)
    x0, x1 = max(0, ox), min(nx2, ox + field.nx)
    dr[y0:y1, x0:x1] = src_r[y0 - oy:y1 - oy, x0 - ox:x1 - ox]
    di[y0:y1, x0:x1] = src_i[y0 - oy:y1 - oy, x0 - ox:x1 - ox]
    return out
