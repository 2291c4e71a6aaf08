"""ComplexField: the data type that crosses the boundary (src/field.js:22-513).

A sampled scalar field U = A exp(i phi) on an nx-by-ny grid of pitch (dx, dy),
stored as two float64 planes (re, im), row-major, idx = x + y*nx, optical axis at
the array centre: sample (i, j) sits at x = (i - nx/2) dx, y = (j - ny/2) dy.

This class is the host-side container the engine entry points read and write.
Its accessors below are container conveniences for callers; every operation on
the propagate-and-retrieve path (FFTs, propagation, A exp(i phi) set-up inside
the design loops, powers and metrics) runs in the CUDA kernels.
"""
from __future__ import annotations

import numpy as np

from .fft import isPow2


class ComplexField:
    def __init__(self, nx: int, ny: int | None = None, dx: float = 1.0, dy: float | None = None):
        ny = nx if ny is None else ny
        dy = dx if dy is None else dy
        if not isPow2(nx) or not isPow2(ny):
            raise ValueError(f"ComplexField: grid must be power-of-two, got {nx}x{ny}")
        self.nx, self.ny = int(nx), int(ny)
        self.dx, self.dy = float(dx), float(dy)
        self.re = np.zeros(self.nx * self.ny, dtype=np.float64)
        self.im = np.zeros(self.nx * self.ny, dtype=np.float64)

    # -- geometry (src/field.js:41-67)
    @property
    def size(self) -> int:
        return self.nx * self.ny

    @property
    def extentX(self) -> float:
        return self.nx * self.dx

    @property
    def extentY(self) -> float:
        return self.ny * self.dy

    def x(self, i):
        return (i - self.nx / 2) * self.dx

    def y(self, j):
        return (j - self.ny / 2) * self.dy

    def idx(self, i: int, j: int) -> int:
        return i + j * self.nx

    # -- copies (src/field.js:69-86)
    def clone(self) -> "ComplexField":
        f = ComplexField(self.nx, self.ny, self.dx, self.dy)
        f.re[:] = self.re
        f.im[:] = self.im
        return f

    def copyFrom(self, other: "ComplexField") -> "ComplexField":
        if other.nx != self.nx or other.ny != self.ny:
            raise ValueError("ComplexField.copyFrom: shape mismatch")
        self.re[:] = other.re
        self.im[:] = other.im
        self.dx, self.dy = other.dx, other.dy
        return self

    # -- container views
    def intensity(self) -> np.ndarray:
        return self.re * self.re + self.im * self.im

    def amplitude(self) -> np.ndarray:
        return np.hypot(self.re, self.im)

    def phase(self) -> np.ndarray:
        return np.arctan2(self.im, self.re)

    def power(self) -> float:
        """Sum |U|^2 dx dy (src/field.js:190-195), accumulated in float64."""
        return float(np.sum(self.re * self.re + self.im * self.im)) * self.dx * self.dy

    def setAmplitudePhase(self, amp, phi=0.0) -> "ComplexField":
        """re = A cos(phi), im = A sin(phi) (src/field.js:168-179)."""
        a = np.broadcast_to(np.asarray(amp, dtype=np.float64), (self.size,))
        p = np.broadcast_to(np.asarray(phi, dtype=np.float64), (self.size,))
        self.re[:] = a * np.cos(p)
        self.im[:] = a * np.sin(p)
        return self

    def __repr__(self) -> str:
        return f"ComplexField({self.nx}x{self.ny} @ {self.dx * 1e6:.3f}um)"


# ------------------------------------------------------------------ masks (host set-up)
def _grid(nx, ny, dx, dy):
    x = (np.arange(nx) - nx / 2) * dx
    y = (np.arange(ny) - ny / 2) * dy
    return np.meshgrid(x, y)


def discMask(nx, ny, dx, dy, radius, soft=0.0, cx=0.0, cy=0.0):
    """Disc aperture with optional raised-cosine edge (src/field.js:516-536)."""
    X, Y = _grid(nx, ny, dx, dy)
    r = np.hypot(X - cx, Y - cy).ravel()
    if soft > 0:
        v = 0.5 * (1 + np.cos((np.pi * (r - radius + soft)) / soft))
        v = np.where(r <= radius - soft, 1.0, np.where(r >= radius, 0.0, v))
    else:
        v = (r <= radius).astype(np.float64)
    return v


def _edge(x, half, soft):
    v = 0.5 * (1 + np.cos((np.pi * (x - half + soft)) / soft))
    return np.where(x <= half - soft, 1.0, np.where(x >= half, 0.0, v))


def rectMask(nx, ny, dx, dy, width, height, soft=0.0):
    """Rectangular aperture with optional raised-cosine edge (src/field.js:539-558)."""
    X, Y = _grid(nx, ny, dx, dy)
    ax, ay = np.abs(X), np.abs(Y)
    if soft > 0:
        fx, fy = _edge(ax, width / 2, soft), _edge(ay, height / 2, soft)
    else:
        fx, fy = (ax <= width / 2).astype(np.float64), (ay <= height / 2).astype(np.float64)
    return (fx * fy).ravel()


def ringMask(nx, ny, inner=0.5, outer=0.95, soft=0.02):
    """Annulus in half-window units (src/doe.js:288-305)."""
    v = (np.arange(ny) - ny / 2) / (ny / 2)
    u = (np.arange(nx) - nx / 2) / (nx / 2)
    U, V = np.meshgrid(u, v)
    r = np.hypot(U, V).ravel()
    lo, hi = inner + soft, outer - soft
    out = np.zeros_like(r)
    out[(r >= lo) & (r <= hi)] = 1.0
    m = (r > inner) & (r < lo)
    out[m] = 0.5 * (1 - np.cos((np.pi * (r[m] - inner)) / soft))
    m = (r > hi) & (r < outer)
    out[m] = 0.5 * (1 + np.cos((np.pi * (r[m] - hi)) / soft))
    return out
