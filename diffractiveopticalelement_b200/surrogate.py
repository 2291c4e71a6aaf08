"""Warm-start surrogate for image-plane WGS (no reference counterpart).

A U-Net maps a target irradiance (and its ROI) to a DOE phase; WGS then refines
that phase and decides the final screen RMSE (src/projector.js:554-595), so the
network only ever replaces the random starting phase of src/doe.js:81-86. All
network arithmetic runs in the engine's own BF16 kernels (csrc/unet.cu): the
forward pass, the backward pass and Adam. Two training signals are provided:

* ``physics``: the intensity loss of the predicted phase through the same
  image-plane propagation as the design loop, with its exact phase gradient
  (doe_phase_loss_grad), so the network learns phases whose screen matches the
  target, whatever WGS solution they resemble;
* ``supervised``: 1 - cos(phase - phase_wgs) against phases that GPU WGS produced
  for the same targets (doe_phase_supervised_grad).

Tensors are CUDA float32 [B, n*n]; PyTorch only holds device memory.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .batch import _Ordered, _plane


class Surrogate:
    """The U-Net: n x n input, `levels` levels of base << l channels."""

    def __init__(self, n=256, base=32, levels=4, max_batch=16, seed=1, ctx=None):
        self.ctx = ctx or _lib.context()
        self.n, self.base, self.levels, self.max_batch = n, base, levels, max_batch
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.doe_surrogate_create(self.ctx.h, n, base, levels, max_batch, seed, C.byref(h)))
        self.h = h
        self.count = int(self.ctx.lib.doe_surrogate_param_count(h))

    def close(self):
        # the network's memory is released through its context; once that context
        # is gone (interpreter shutdown collects the two in any order) the process
        # is ending and the driver releases everything
        if self.h and getattr(self.ctx, "h", None):
            self.ctx.lib.doe_surrogate_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- parameters
    def params(self, which=0) -> np.ndarray:
        out = np.empty(self.count, dtype=np.float32)
        self.ctx.check(self.ctx.lib.doe_surrogate_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), which))
        return out

    def gradients(self) -> np.ndarray:
        return self.params(1)

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.count:
            raise ValueError(f"expected {self.count} parameters, got {p.size}")
        self.ctx.check(self.ctx.lib.doe_surrogate_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def save(self, path):
        np.save(path, self.params())

    def load(self, path):
        self.set_params(np.load(path))

    # ---------------------------------------------------------------- passes
    def forward(self, irr, roi=None, out=None):
        """Predicted phase [B, n*n] for target irradiances irr [B, n*n] (+ ROI)."""
        torch = _torch()
        nn = self.n * self.n
        B = irr.shape[0]
        if B > self.max_batch:
            return torch.cat([self.forward(irr[i:i + self.max_batch], None if roi is None else roi[i:i + self.max_batch])
                              for i in range(0, B, self.max_batch)])
        irr = _plane(irr.contiguous(), B, nn, "irr")
        roi = _plane(roi.contiguous(), B, nn, "roi") if roi is not None else None
        ph = out if out is not None else torch.empty((B, nn), dtype=torch.float32, device=irr.device)
        with _Ordered(self.ctx):
            self.ctx.check(self.ctx.lib.doe_surrogate_forward(self.h, B, irr.data_ptr(),
                                                              None if roi is None else roi.data_ptr(),
                                                              ph.data_ptr()))
        return ph

    def backward(self, dphase):
        d = dphase.contiguous()
        with _Ordered(self.ctx):
            self.ctx.check(self.ctx.lib.doe_surrogate_backward(self.h, d.data_ptr()))

    def allreduce_gradients(self, world, group=None):
        """Average the accumulated gradients over `world` data-parallel ranks (NCCL)."""
        if world <= 1:
            return
        torch = _torch()
        from .sharding import allreduce_mean_
        buf = torch.empty(self.count, dtype=torch.float32, device="cuda")
        with _Ordered(self.ctx):
            self.ctx.check(self.ctx.lib.doe_surrogate_grads_dev(self.h, buf.data_ptr()))
        allreduce_mean_(buf, world, group)
        with _Ordered(self.ctx):
            self.ctx.check(self.ctx.lib.doe_surrogate_set_grads_dev(self.h, buf.data_ptr()))

    def zero_grad(self):
        with _Ordered(self.ctx):
            self.ctx.check(self.ctx.lib.doe_surrogate_zero_grad(self.h))

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, grad_scale=1.0):
        with _Ordered(self.ctx):
            self.ctx.check(self.ctx.lib.doe_surrogate_adam(self.h, float(lr), float(beta1), float(beta2), float(eps),
                                                           float(weight_decay), float(grad_scale)))


def _torch():
    import torch
    return torch


def phase_loss_grad(ctx, phase, illumination, target_amp, roi, *, nx, ny, dx, dy=None, lam=532e-9, z=0.03):
    """Intensity loss L = sum m (|U|^2 - t^2)^2 / sum m t^4 of each phase and dL/dphase."""
    torch = _torch()
    n = nx * ny
    B = phase.shape[0]
    ph = _plane(phase.contiguous(), B, n, "phase")
    ill = _plane(illumination, B, n, "illumination", shared_ok=True)
    tgt = _plane(target_amp, B, n, "target_amp")
    ro = _plane(roi, B, n, "roi")
    grad = torch.empty_like(ph)
    loss = torch.empty(B, dtype=torch.float64, device=ph.device)
    d = _lib.PhaseLossDesc(B, nx, ny, dx, dx if dy is None else dy, lam, z, ill.data_ptr(), tgt.data_ptr(),
                           None if ro is None else ro.data_ptr(), ph.data_ptr(), grad.data_ptr(), loss.data_ptr())
    with _Ordered(ctx):
        ctx.check(ctx.lib.doe_phase_loss_grad(ctx.h, C.byref(d)))
    return loss, grad


def supervised_grad(ctx, phase, target):
    """L = mean(1 - cos(phase - target)) and dL/dphase."""
    torch = _torch()
    grad = torch.empty_like(phase)
    loss = torch.empty(1, dtype=torch.float64, device=phase.device)
    with _Ordered(ctx):
        ctx.check(ctx.lib.doe_phase_supervised_grad(ctx.h, phase.numel(), phase.data_ptr(), target.data_ptr(),
                                                    grad.data_ptr(), loss.data_ptr()))
    return loss, grad


# ---------------------------------------------------------------- training data
def spot_array_target(n, seed, window=None, sigma=1.5):
    """k x k Gaussian spots (k in 4..32 scaled to the window), weights 1 or U[0.5, 1]."""
    from .doe import makeRng
    rng = makeRng(seed)
    w = window or n // 2
    k = 4 + int(rng() * (min(32, w // 4) - 4 + 1))
    random_w = rng() < 0.5
    pitch = w / k
    x0 = (n - w) / 2 + pitch / 2
    i = np.arange(n)
    amp = np.ones((k, k))
    if random_w:
        for b in range(k):
            for a in range(k):
                amp[b, a] = 0.5 + 0.5 * rng()
    c = x0 + np.arange(k) * pitch
    g = np.exp(-((i[None, :] - c[:, None]) ** 2) / (2 * sigma ** 2))  # [k, n] per axis
    return (g.T @ amp @ g).ravel()  # irr[y, x] = sum_ab amp[b, a] g[b, y] g[a, x]


def smooth_gradient_target(n, seed, window=None, cells=4):
    """Smooth value-noise irradiance in [0, 1] inside the central window (cosine-
    interpolated seeded lattice, two octaves), zero outside."""
    from .doe import makeRng
    rng = makeRng(seed)
    w = window or n // 2
    out = np.zeros((n, n))
    acc = np.zeros((w, w))
    for octave, amp in ((cells, 1.0), (2 * cells, 0.5)):
        lat = np.array([[rng() for _ in range(octave + 1)] for _ in range(octave + 1)])
        t = np.linspace(0, octave, w, endpoint=False)
        i0 = t.astype(int)
        f = t - i0
        s = (1 - np.cos(np.pi * f)) / 2
        a = lat[i0][:, i0] * (1 - s)[None, :] + lat[i0][:, i0 + 1] * s[None, :]
        b = lat[i0 + 1][:, i0] * (1 - s)[None, :] + lat[i0 + 1][:, i0 + 1] * s[None, :]
        acc += amp * (a * (1 - s)[:, None] + b * s[:, None])
    acc = (acc - acc.min()) / max(acc.max() - acc.min(), 1e-12)
    o = (n - w) // 2
    out[o:o + w, o:o + w] = acc
    return out.ravel()


def training_targets(n, count, seed0, kinds=("rectangles", "spots", "smooth")):
    """Seeded mixture of the surrogate's training targets (irradiance planes)."""
    from .projector import rectangles_target
    out = np.empty((count, n * n), dtype=np.float32)
    scale = n / 256
    for k in range(count):
        kind = kinds[k % len(kinds)]
        s = seed0 + k
        if kind == "rectangles":
            out[k] = rectangles_target(n, n, s, window=max(8, int(128 * scale)),
                                       width=(max(2, int(4 * scale)), max(4, int(40 * scale))))
        elif kind == "spots":
            out[k] = spot_array_target(n, s)
        else:
            out[k] = smooth_gradient_target(n, s)
    return out


def train(model, irr_all, roi_all, illumination, target_amp_all, *, dx, lam, z, steps, batch, lr=1e-3,
          loss="physics", target_phase_all=None, seed=0, log_every=0, lr_final=None, world=1, group=None):
    """Adam training on device-resident sets (CUDA float32 [N, n*n]); returns the loss history.

    With world > 1 every rank draws its own batches (seed + rank offsets are the
    caller's) and the gradients are averaged over ranks before each Adam step."""
    torch = _torch()
    gen = torch.Generator(device="cpu").manual_seed(seed)
    N = irr_all.shape[0]
    n = model.n
    hist = []
    for step in range(steps):
        idx = torch.randint(0, N, (batch,), generator=gen).to(irr_all.device)
        irr, roi = irr_all[idx].contiguous(), roi_all[idx].contiguous()
        ph = model.forward(irr, roi)
        if loss == "physics":
            L, g = phase_loss_grad(model.ctx, ph, illumination, target_amp_all[idx].contiguous(), roi, nx=n, ny=n,
                                   dx=dx, lam=lam, z=z)
            g = g / batch
            lval = L.mean()
        else:
            lval, g = supervised_grad(model.ctx, ph, target_phase_all[idx].contiguous())
        model.backward(g)
        model.allreduce_gradients(world, group)
        rate = lr if lr_final is None else lr * (lr_final / lr) ** (step / max(1, steps - 1))
        model.adam(rate)
        if log_every and (step % log_every == 0 or step == steps - 1):
            hist.append((step, float(lval)))
    return hist
