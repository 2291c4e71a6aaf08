"""2-D FFT with the reference's conventions (src/fft.js).

``fft2d(re, im, nx, ny, inverse)`` transforms in place like src/fft.js:148-154:
forward unscaled, inverse scaled by 1/(nx*ny), planes row-major with
idx = x + y*nx. The transform runs on the GPU (FP32 Stockham passes); the
planes are FP64 on both sides of the call.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def isPow2(n) -> bool:
    """src/fft.js:66-68."""
    return isinstance(n, (int, np.integer)) and n > 0 and (int(n) & (int(n) - 1)) == 0


def nextPow2(n) -> int:
    """src/fft.js:59-63."""
    p = 1
    while p < n:
        p <<= 1
    return p


def _check_planes(re, im, nx, ny):
    if not isinstance(re, np.ndarray) or not isinstance(im, np.ndarray):
        raise TypeError("fft2d: re and im must be numpy float64 arrays")
    if re.size != nx * ny or im.size != nx * ny:
        raise ValueError(f"fft2d: plane length {re.size} does not match {nx}x{ny}")
    if re.dtype != np.float64 or im.dtype != np.float64 or not re.flags.c_contiguous \
            or not im.flags.c_contiguous:
        raise TypeError("fft2d: planes must be C-contiguous float64 (Float64Array)")


def fft2d(re: np.ndarray, im: np.ndarray, nx: int, ny: int, inverse: bool = False, *,
          ctx=None) -> None:
    """In-place 2-D FFT of the (re, im) planes (src/fft.js:148-154)."""
    _check_planes(re, im, nx, ny)
    c = ctx or _lib.context()
    c.check(c.lib.doe_fft2d(c.h, _lib.dp(re), _lib.dp(im), int(nx), int(ny), int(bool(inverse))))


def fft2dOut(re, im, nx: int, ny: int, inverse: bool = False, *, ctx=None):
    """Out-of-place variant (src/fft.js:157-162)."""
    r = np.array(re, dtype=np.float64, copy=True)
    i = np.array(im, dtype=np.float64, copy=True)
    fft2d(r, i, nx, ny, inverse, ctx=ctx)
    return {"re": r, "im": i}
