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
