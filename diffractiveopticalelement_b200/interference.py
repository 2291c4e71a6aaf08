"""Holography and partial coherence (src/interference.js), executed by the CUDA engine.

Same names, argument meaning and option defaults as the reference:
``modalIntensity`` (src/interference.js:57-69), ``partiallyCoherentModes``
(:79-101, smoothing :104-125), ``recordHologram`` (:347-388) and
``reconstructHologram`` (:397-411, angular-spectrum propagation with
``bandLimit: false`` unless the options say otherwise). ``propagatedModalIntensity``
is the reference tests' pattern -- propagate every mode with
``propagateAngularSpectrumInPlace``, then ``modalIntensity`` -- as one batched call.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .field import ComplexField
from .propagate import _opt

_ENCODINGS = {"raw": 0, "binary": 1, "phase": 2}


def _stack(modes):
    n = modes[0].size
    for m in modes:
        if m.size != n:
            raise ValueError("modalIntensity: modes differ in size")
    re = np.ascontiguousarray(np.concatenate([np.asarray(m.re, dtype=np.float64) for m in modes]))
    im = np.ascontiguousarray(np.concatenate([np.asarray(m.im, dtype=np.float64) for m in modes]))
    return re, im


def _modal(modes, weights, lam, z, opts, ctx, kw):
    if not modes:
        raise ValueError("modalIntensity: no modes")
    f0 = modes[0]
    re, im = _stack(modes)
    w = None if weights is None else np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
    if w is not None and w.size < len(modes):
        raise ValueError("modalIntensity: fewer weights than modes")
    out = np.empty(f0.size)
    c = ctx or _lib.context()
    c.check(c.lib.doe_modal_intensity(
        c.h, len(modes), _lib.dp(re), _lib.dp(im), f0.nx, f0.ny, None if w is None else _lib.dp(w),
        f0.dx, f0.dy, float(lam), float(z), int(bool(_opt(opts, kw, "bandLimit", True))),
        int(bool(_opt(opts, kw, "evanescent", True))), float(_opt(opts, kw, "softEdge", 0.02)), _lib.dp(out)))
    return {"intensity": out, "coherence": 0 if len(modes) > 1 else 1, "modeCount": len(modes)}


def modalIntensity(modes, weights=None, *, ctx=None):
    """Incoherent sum of mode intensities, weighted and normalised by the weight sum."""
    return _modal(modes, weights, 532e-9, 0.0, None, ctx, None)


def propagatedModalIntensity(modes, lam, z, weights=None, opts=None, *, ctx=None, **kw):
    """modalIntensity of every mode angular-spectrum propagated to z (one batch)."""
    return _modal(modes, weights, lam, z, opts, ctx, kw)


def partiallyCoherentModes(nx, ny, dx, dy, opts=None, *, ctx=None, **kw):
    """Gaussian-envelope modes with smoothed random phase screens (seeded, one xorshift32 stream)."""
    modes = int(_opt(opts, kw, "modes", 8))
    sigma = float(_opt(opts, kw, "sigma", 40e-6))
    waist = float(_opt(opts, kw, "waist", 1e-3))
    seed = float(_opt(opts, kw, "seed", 7))
    n = nx * ny
    re = np.empty(modes * n)
    im = np.empty(modes * n)
    c = ctx or _lib.context()
    c.check(c.lib.doe_partially_coherent_modes(c.h, int(nx), int(ny), float(dx), float(dy), modes, sigma, waist,
                                               seed, _lib.dp(re), _lib.dp(im)))
    out = []
    for m in range(modes):
        f = ComplexField(nx, ny, dx, dy)
        f.re = re[m * n:(m + 1) * n]
        f.im = im[m * n:(m + 1) * n]
        out.append(f)
    return out


def recordHologram(object, reference, opts=None, *, ctx=None, **kw):
    """Record |object + reference|^2, peak-normalised, and encode it as a plate."""
    encode = _opt(opts, kw, "encode", "raw")
    levels = int(_opt(opts, kw, "levels", 0))
    n = object.size
    if reference.size != n:
        raise ValueError("recordHologram: shape mismatch")
    if encode not in _ENCODINGS:
        raise ValueError(f'recordHologram: unknown encoding "{encode}"')
    a = [np.ascontiguousarray(np.asarray(v, dtype=np.float64))
         for v in (object.re, object.im, reference.re, reference.im)]
    plate = ComplexField(object.nx, object.ny, object.dx, object.dy)
    total = ComplexField(object.nx, object.ny, object.dx, object.dy)
    recorded = np.empty(n)
    c = ctx or _lib.context()
    c.check(c.lib.doe_hologram_record(c.h, *[_lib.dp(v) for v in a], n, _ENCODINGS[encode], levels,
                                      _lib.dp(plate.re), _lib.dp(plate.im), _lib.dp(recorded),
                                      _lib.dp(total.re), _lib.dp(total.im)))
    return {"plate": plate, "recorded": recorded, "sum": total}


def reconstructHologram(plate, reference, lam, z, opts=None, *, ctx=None, **kw):
    """Illuminate the plate with the reference; real image at +z, virtual image at -z."""
    if reference.size != plate.size:
        raise ValueError("reconstructHologram: shape mismatch")
    a = [np.ascontiguousarray(np.asarray(v, dtype=np.float64))
         for v in (plate.re, plate.im, reference.re, reference.im)]
    mk = lambda: ComplexField(plate.nx, plate.ny, plate.dx, plate.dy)
    real, virtual, illum = mk(), mk(), mk()
    c = ctx or _lib.context()
    c.check(c.lib.doe_hologram_reconstruct(
        c.h, *[_lib.dp(v) for v in a], plate.nx, plate.ny, plate.dx, plate.dy, float(lam), float(z),
        int(bool(_opt(opts, kw, "bandLimit", False))), int(bool(_opt(opts, kw, "evanescent", True))),
        float(_opt(opts, kw, "softEdge", 0.02)), _lib.dp(real.re), _lib.dp(real.im), _lib.dp(virtual.re),
        _lib.dp(virtual.im), _lib.dp(illum.re), _lib.dp(illum.im)))
    return {"real": real, "virtual": virtual, "illumination": illum}
