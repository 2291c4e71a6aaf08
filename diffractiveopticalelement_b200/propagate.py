"""Scalar diffraction propagation (src/propagate.js), executed by the CUDA engine.

Same names, argument meaning and option defaults as the reference:
``angularSpectrumTransferFunction`` (src/propagate.js:57-102),
``propagateAngularSpectrum`` / ``propagateAngularSpectrumInPlace`` (:105-133),
``focalPlaneSpectrum`` (:342-374), ``focusSweep`` (:427-434),
``localFrequencyLimit`` (:48-51), ``fresnelMinDistance`` (:141-143),
``propagateFresnelFFT`` / ``propagateFraunhofer`` (:155-230, :310-312),
``propagateFresnelFFTInverse`` (:237-308), ``propagate`` (:383-389).
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from .field import ComplexField

DEFAULT_WAVELENGTH = 532e-9


def _opt(opts, kw, name, default):
    if kw and name in kw:
        return kw[name]
    if opts and name in opts:
        return opts[name]
    return default


def localFrequencyLimit(n, d, lam, z):
    """src/propagate.js:48-51 (scalar geometry helper)."""
    df = 1 / (n * d)
    return 1 / (lam * math.sqrt(math.pow(2 * df * z, 2) + 1))


def fresnelMinDistance(n, d, lam):
    """src/propagate.js:141-143."""
    return (n * d * d) / lam


def angularSpectrumTransferFunction(nx, ny, dx, dy, lam, z, opts=None, *, ctx=None, **kw):
    """Centred transfer function planes and the propagating fraction."""
    bl = bool(_opt(opts, kw, "bandLimit", True))
    ev = bool(_opt(opts, kw, "evanescent", True))
    se = float(_opt(opts, kw, "softEdge", 0.02))
    c = ctx or _lib.context()
    re = np.empty(nx * ny)
    im = np.empty(nx * ny)
    frac = np.zeros(1)
    c.check(c.lib.doe_asm_transfer(c.h, int(nx), int(ny), float(dx), float(dy), float(lam),
                                   float(z), int(bl), int(ev), se, _lib.dp(re), _lib.dp(im),
                                   _lib.dp(frac)))
    return {"re": re, "im": im, "propagatingFraction": float(frac[0])}


def propagateAngularSpectrumInPlace(field: ComplexField, lam, z, opts=None, *, ctx=None, **kw):
    """In-place angular-spectrum propagation; z < 0 back-propagates, z == 0 is a no-op."""
    bl = bool(_opt(opts, kw, "bandLimit", True))
    ev = bool(_opt(opts, kw, "evanescent", True))
    se = float(_opt(opts, kw, "softEdge", 0.02))
    c = ctx or _lib.context()
    c.check(c.lib.doe_asm(c.h, _lib.dp(field.re), _lib.dp(field.im), field.nx, field.ny,
                          field.dx, field.dy, float(lam), float(z), int(bl), int(ev), se))
    return field


def propagateAngularSpectrum(field: ComplexField, lam, z, opts=None, *, ctx=None, **kw):
    """Angular-spectrum propagation of a copy; the input is left untouched."""
    out = field.clone()
    return propagateAngularSpectrumInPlace(out, lam, z, opts, ctx=ctx, **kw)


def focalPlaneSpectrum(field: ComplexField, lam, f, *, ctx=None) -> ComplexField:
    """Lens focal-plane field; output pitch lam*f/(N*dx)."""
    c = ctx or _lib.context()
    out = ComplexField(field.nx, field.ny, 1.0, 1.0)
    d = np.zeros(2)
    c.check(c.lib.doe_focal_plane(c.h, _lib.dp(field.re), _lib.dp(field.im), field.nx, field.ny,
                                  field.dx, field.dy, float(lam), float(f), _lib.dp(out.re),
                                  _lib.dp(out.im), _lib.dp(d)))
    out.dx, out.dy = float(d[0]), float(d[1])
    return out


def focusSweep(field: ComplexField, lam, zStart, zEnd, steps, opts=None, *, ctx=None, **kw):
    """Planes at zStart + (zEnd - zStart) s / steps for s = 0..steps (one engine call)."""
    bl = bool(_opt(opts, kw, "bandLimit", True))
    ev = bool(_opt(opts, kw, "evanescent", True))
    se = float(_opt(opts, kw, "softEdge", 0.02))
    zs = np.array([zStart + ((zEnd - zStart) * s) / steps for s in range(steps + 1)],
                  dtype=np.float64)
    n = field.size
    ore = np.empty(n * zs.size)
    oim = np.empty(n * zs.size)
    c = ctx or _lib.context()
    c.check(c.lib.doe_asm_sweep(c.h, _lib.dp(field.re), _lib.dp(field.im), field.nx, field.ny,
                                field.dx, field.dy, float(lam), _lib.dp(zs), int(zs.size),
                                int(bl), int(ev), se, _lib.dp(ore), _lib.dp(oim)))
    planes = []
    for k, z in enumerate(zs):
        f = ComplexField(field.nx, field.ny, field.dx, field.dy)
        f.re = ore[k * n:(k + 1) * n]
        f.im = oim[k * n:(k + 1) * n]
        planes.append({"z": float(z), "field": f})
    return planes


def propagateFresnelFFT(field: ComplexField, lam, z, opts=None, *, ctx=None, **kw):
    """Single-FFT Fresnel propagation to the magnified grid (src/propagate.js:155-230).

    Returns {field, dx, dy, z, magnification, undersampled, zCritical} like the
    reference; throwOnUndersampled raises the reference's error below z_c.
    """
    throw = bool(_opt(opts, kw, "throwOnUndersampled", False))
    nx, ny, dx, dy = field.nx, field.ny, field.dx, field.dy
    az = abs(z)
    z_c = fresnelMinDistance(nx, dx, lam)
    under = az < z_c
    if under and throw:
        raise ValueError(
            f"propagateFresnelFFT: z={az * 1e3:.3f} mm is below the critical distance "
            f"z_c={z_c * 1e3:.3f} mm for a {nx}x{ny} grid at {dx * 1e6:.2f} um pitch — the Fresnel chirp is "
            f"under-sampled. Use the angular spectrum instead.")
    c = ctx or _lib.context()
    out = ComplexField(nx, ny, 1.0, 1.0)
    d = np.zeros(2)
    c.check(c.lib.doe_fresnel(c.h, _lib.dp(field.re), _lib.dp(field.im), nx, ny, dx, dy, float(lam), float(z),
                              _lib.dp(out.re), _lib.dp(out.im), _lib.dp(d)))
    out.dx, out.dy = float(d[0]), float(d[1])
    return {"field": out, "dx": out.dx, "dy": out.dy, "z": z, "magnification": out.dx / dx,
            "undersampled": under, "zCritical": z_c}


def propagateFraunhofer(field: ComplexField, lam, z, opts=None, *, ctx=None, **kw):
    """src/propagate.js:310-312 (same transform as propagateFresnelFFT)."""
    return propagateFresnelFFT(field, lam, z, opts, ctx=ctx, **kw)


def propagateFresnelFFTInverse(field: ComplexField, lam, z, opts=None, *, ctx=None, **kw):
    """Exact inverse of propagateFresnelFFT back onto the DOE grid (src/propagate.js:237-308)."""
    dx = _opt(opts, kw, "dx", None)
    dy = _opt(opts, kw, "dy", None)
    if not dx or not dy:
        raise ValueError("propagateFresnelFFTInverse: pass the DOE-plane pitch as {dx, dy}")
    c = ctx or _lib.context()
    out = ComplexField(field.nx, field.ny, dx, dy)
    c.check(c.lib.doe_fresnel_inverse(c.h, _lib.dp(field.re), _lib.dp(field.im), field.nx, field.ny, field.dx,
                                      field.dy, float(lam), float(z), float(dx), float(dy), _lib.dp(out.re),
                                      _lib.dp(out.im)))
    return out


def propagate(field: ComplexField, lam, z, opts=None, *, ctx=None, **kw):
    """Generic entry point (src/propagate.js:383-389): method 'asm' (default) or 'fresnel'."""
    method = _opt(opts, kw, "method", "asm")
    pad = int(_opt(opts, kw, "pad", 1))
    src = field
    if pad > 1:
        from .projector import resample_centred
        src = resample_centred(field, field.nx * pad, field.ny * pad)
    if method == "fresnel":
        return propagateFresnelFFT(src, lam, z, opts, ctx=ctx, **kw)["field"]
    bl = _opt(opts, kw, "bandLimit", True)
    return propagateAngularSpectrum(src, lam, z, {"bandLimit": True if bl is None else bl}, ctx=ctx)
