"""Batched, device-resident design calls (no reference counterpart).

The reference designs one element per call on host planes (src/doe.js:327-546).
These wrappers run B designs of one grid size through one engine call on CUDA
tensors that stay on the device: `design_batch` drives doe_design_dev and
`multiplane_batch` drives doe_multiplane_dev and `screen_metrics_batch` drives
doe_screen_metrics_dev. Tensors are float32,
C-contiguous, shaped [B, ny*nx] (or [ny*nx] for a plane shared by every design
where noted). Work is ordered against torch's current stream on entry and exit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

_ALG = {"gs": _lib.DOE_ALG_GS, "wgs": _lib.DOE_ALG_WGS, "fourier": _lib.DOE_ALG_FOURIER,
        "wgs-fourier": _lib.DOE_ALG_WGS_FOURIER}


def _torch():
    import torch
    return torch


def _plane(t, B, n, name, shared_ok=False):
    torch = _torch()
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name}: expected a CUDA tensor")
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise TypeError(f"{name}: expected contiguous float32")
    if t.numel() == n and shared_ok and B > 1:
        return t.reshape(1, n).expand(B, n).contiguous()
    if t.numel() != B * n:
        raise ValueError(f"{name}: expected {B}x{n} values, got {t.numel()}")
    return t


class _Ordered:
    """Run engine work on the context stream, ordered after / before torch's stream."""

    def __init__(self, ctx):
        torch = _torch()
        self.cur = torch.cuda.current_stream()
        self.ext = torch.cuda.ExternalStream(ctx.stream, device=self.cur.device)

    def __enter__(self):
        self.ext.wait_stream(self.cur)
        return self

    def __exit__(self, *exc):
        self.cur.wait_stream(self.ext)
        return False


def design_batch(ctx, illumination, target_amp, phase, *, nx, ny, dx, dy=None, lam=532e-9, z=0.03,
                 iterations=100, algorithm="wgs", beta=0.9, feedback=0.0, escape=0, roi=None,
                 lambdas=None, zs=None, rmse_goal=0.0, screen_irr=None, history=True):
    """B designs of one grid in one call (doe_design_dev).

    `phase` holds the initial phases and receives the results (best iterate for
    WGS). `illumination` may be one shared plane. With rmse_goal > 0 (image-plane
    WGS) a design stops at the first iteration whose screen RMSE is <= rmse_goal
    and `iterations_used` says when. Returns a dict of device tensors.
    """
    desc, out = _design_desc(illumination, target_amp, phase, nx=nx, ny=ny, dx=dx, dy=dy, lam=lam, z=z,
                             iterations=iterations, algorithm=algorithm, beta=beta, feedback=feedback, escape=escape,
                             roi=roi, lambdas=lambdas, zs=zs, rmse_goal=rmse_goal, screen_irr=screen_irr,
                             history=history)
    with _Ordered(ctx):
        ctx.check(ctx.lib.doe_design_dev(ctx.h, C.byref(desc)))
    return out


def autotune_design(ctx, illumination, target_amp, phase, *, trial_iterations=4, **kw):
    """Pick the fastest design-pass shapes (and, for image-plane WGS on 64^2-256^2,
    the cluster-resident loop) for this batch's grid (doe_autotune_design).

    Takes design_batch's arguments; runs `trial_iterations` iterations per
    candidate, leaves `phase` as it was and keeps the choice in the context.
    Returns (row variant, column variant, cluster loop)."""
    desc, _ = _design_desc(illumination, target_amp, phase, **kw)
    chosen = (C.c_int * 3)()
    with _Ordered(ctx):
        ctx.check(ctx.lib.doe_autotune_design(ctx.h, C.byref(desc), int(trial_iterations), chosen))
    return tuple(chosen)


def _design_desc(illumination, target_amp, phase, *, nx, ny, dx, dy=None, lam=532e-9, z=0.03, iterations=100,
                 algorithm="wgs", beta=0.9, feedback=0.0, escape=0, roi=None, lambdas=None, zs=None, rmse_goal=0.0,
                 screen_irr=None, history=True):
    """The doe_design_dev descriptor of a batch and the dict of its output tensors
    (the descriptor's host arrays are kept alive in the dict)."""
    torch = _torch()
    if algorithm not in _ALG:
        raise ValueError(f"unknown algorithm {algorithm!r}")
    n = nx * ny
    if phase.dim() == 1:
        raise ValueError("phase: expected [B, n]")
    B = phase.shape[0]
    ph = _plane(phase, B, n, "phase")
    ill = _plane(illumination, B, n, "illumination", shared_ok=True)
    tgt = _plane(target_amp, B, n, "target_amp")
    ro = _plane(roi, B, n, "roi")
    sirr = _plane(screen_irr, B, n, "screen_irr")
    dev = ph.device
    amp = torch.empty((B, n), dtype=torch.float32, device=dev)
    it_h = max(int(iterations), 1)
    err = torch.empty((B, it_h), dtype=torch.float64, device=dev) if history else None
    eff = torch.empty((B, it_h), dtype=torch.float64, device=dev) if history else None
    wgs = algorithm.startswith("wgs")
    rmse = torch.empty(B, dtype=torch.float64, device=dev) if wgs else None
    used = torch.empty(B, dtype=torch.int32, device=dev)
    lam_a = None if lambdas is None else np.ascontiguousarray(lambdas, dtype=np.float64)
    z_a = None if zs is None else np.ascontiguousarray(zs, dtype=np.float64)
    for a, nm in ((lam_a, "lambdas"), (z_a, "zs")):
        if a is not None and a.size != B:
            raise ValueError(f"{nm}: expected {B} entries")
    ptr = lambda t: None if t is None else t.data_ptr()
    desc = _lib.DesignDevDesc(B, nx, ny, dx, dx if dy is None else dy, lam, z, _lib.dp(lam_a), _lib.dp(z_a),
                              _ALG[algorithm], int(iterations), float(feedback), int(escape), float(beta),
                              ptr(ill), ptr(tgt), ptr(ro), ptr(ph), ptr(amp), None, ptr(err), ptr(eff), ptr(rmse),
                              float(rmse_goal), ptr(sirr), ptr(used) if algorithm == "wgs" else None)
    out = {"phase": ph, "amplitude": amp, "error": err, "efficiency": eff}
    if wgs:
        out["rmse"] = rmse
    if algorithm == "wgs":
        out["iterations_used"] = used
    desc._keep = (ill, tgt, ro, sirr, lam_a, z_a)  # inputs the descriptor points into
    return desc, out


def screen_metrics_batch(ctx, amplitude, target_irr, illumination, *, nx, ny, sdx, sdy=None, dx=None, dy=None,
                         roi=None):
    """Radiometric screen metrics of B screens given by amplitude (doe_screen_metrics_dev).

    Returns a [B, 6] float64 tensor: rmse, efficiency, fluxFraction, powerInSignal,
    powerAtScreen, powerIncident (src/projector.js:554-595). target_irr, roi and
    illumination may be single shared planes.
    """
    torch = _torch()
    n = nx * ny
    B = amplitude.shape[0]
    amp = _plane(amplitude, B, n, "amplitude")
    tgt = _plane(target_irr, 1 if target_irr.numel() == n else B, n, "target_irr")
    ill = _plane(illumination, 1 if illumination.numel() == n else B, n, "illumination")
    ro = None if roi is None else _plane(roi, 1 if roi.numel() == n else B, n, "roi")
    if ro is not None and ro.numel() != tgt.numel():
        raise ValueError("roi and target_irr must both be shared or both per design")
    out = torch.empty((B, 6), dtype=torch.float64, device=amp.device)
    sdy = sdx if sdy is None else sdy
    dx = sdx if dx is None else dx
    dy = dx if dy is None else dy
    with _Ordered(ctx):
        ctx.check(ctx.lib.doe_screen_metrics_dev(ctx.h, B, nx, ny, amp.data_ptr(), tgt.data_ptr(),
                                                 0 if tgt.numel() == n else n, None if ro is None else ro.data_ptr(),
                                                 ill.data_ptr(), 0 if ill.numel() == n else n, sdx, sdy, dx, dy,
                                                 out.data_ptr()))
    return out


def multiplane_batch(ctx, illumination, target_amp, phase, zs, *, nx, ny, dx, dy=None, lam=532e-9, iterations=60,
                     roi=None, weights=None, history=True):
    """B multi-plane designs (src/doe.js:557-626) in one call (doe_multiplane_dev).

    target_amp and roi are [B, P, n] (P = len(zs)); `phase` holds the initial
    phases [B, n] and receives the results. Returns error / efficiency [B, I] and
    per-plane errors [B, P, I] as device tensors.
    """
    torch = _torch()
    n = nx * ny
    B = phase.shape[0]
    P = len(zs)
    ph = _plane(phase, B, n, "phase")
    ill = _plane(illumination, B, n, "illumination", shared_ok=True)
    tgt = _plane(target_amp, B * P, n, "target_amp")
    ro = _plane(roi, B * P, n, "roi")
    z_a = np.ascontiguousarray(zs, dtype=np.float64)
    w_a = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    if w_a is not None and w_a.size != P:
        raise ValueError(f"weights: expected {P} entries")
    it_h = max(int(iterations), 1)
    dev = ph.device
    err = torch.empty((B, it_h), dtype=torch.float64, device=dev) if history else None
    eff = torch.empty((B, it_h), dtype=torch.float64, device=dev) if history else None
    ppe = torch.empty((B, P, it_h), dtype=torch.float64, device=dev) if history else None
    ptr = lambda t: None if t is None else t.data_ptr()
    desc = _lib.MultiplaneDevDesc(B, nx, ny, dx, dx if dy is None else dy, lam, P, _lib.dp(z_a), _lib.dp(w_a),
                                  int(iterations), ptr(ill), ptr(tgt), ptr(ro), ptr(ph), ptr(err), ptr(eff), ptr(ppe))
    with _Ordered(ctx):
        ctx.check(ctx.lib.doe_multiplane_dev(ctx.h, C.byref(desc)))
    return {"phase": ph, "error": err, "efficiency": eff, "perPlaneError": ppe}


class DesignMulti:
    """Size classes of designs submitted together (doe_design_multi_*).

    ``run(classes, mode)``: classes is a list of dicts with the keyword arguments of
    `design_batch` (tensors stay alive in this object until the next run); mode 0
    runs directly, 1 captures a CUDA graph and launches it, 2 relaunches it and
    returns the outputs of the capturing call (the graph's tensors are kept for
    as long as the graph). A mode-0 call that grows the engine's scratch makes the
    graph stale: mode 2 then raises DOEError (capture again with mode 1).
    Returns one result dict per class, as `design_batch`.
    """

    def __init__(self, ctx):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(ctx.lib.doe_design_multi_create(ctx.h, C.byref(h)))
        self.h = h
        self._keep = None        # tensors of the last call
        self._graph_keep = None  # tensors baked into the captured graph (mode 1)

    def close(self):
        if self.h:
            self.ctx.lib.doe_design_multi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, classes=None, mode=0):
        torch = _torch()
        if mode == 2:
            if self._graph_keep is None:
                raise ValueError("DesignMulti.run(mode=2): no captured graph (run mode=1 first)")
            with _Ordered(self.ctx):
                self.ctx.check(self.ctx.lib.doe_design_multi_run(self.h, 0, None, 2))
            return self._graph_keep[1]
        descs = (_lib.DesignDevDesc * len(classes))()
        outs, keep = [], []
        for k, cl in enumerate(classes):
            nx, ny = cl["nx"], cl.get("ny", cl["nx"])
            n = nx * ny
            ph = cl["phase"]
            B = ph.shape[0]
            alg = cl.get("algorithm", "wgs")
            it = int(cl.get("iterations", 100))
            ill = _plane(cl["illumination"], B, n, "illumination", shared_ok=True)
            tgt = _plane(cl["target_amp"], B, n, "target_amp")
            ro = _plane(cl.get("roi"), B, n, "roi")
            amp = torch.empty((B, n), dtype=torch.float32, device=ph.device)
            err = torch.empty((B, max(it, 1)), dtype=torch.float64, device=ph.device)
            eff = torch.empty_like(err)
            wgs = alg.startswith("wgs")
            rmse = torch.empty(B, dtype=torch.float64, device=ph.device) if wgs else None
            ptr = lambda t: None if t is None else t.data_ptr()
            descs[k] = _lib.DesignDevDesc(B, nx, ny, cl["dx"], cl.get("dy", cl["dx"]), cl.get("lam", 532e-9),
                                          cl.get("z", 0.03), None, None, _ALG[alg], it, float(cl.get("feedback", 0.0)),
                                          int(cl.get("escape", 0)), float(cl.get("beta", 0.9)), ptr(ill), ptr(tgt),
                                          ptr(ro), ptr(ph), ptr(amp), None, ptr(err), ptr(eff), ptr(rmse), 0.0, None,
                                          None)
            o = {"phase": ph, "amplitude": amp, "error": err, "efficiency": eff}
            if wgs:
                o["rmse"] = rmse
            outs.append(o)
            keep += [ill, tgt, ro, ph, amp, err, eff, rmse]
        with _Ordered(self.ctx):
            self.ctx.check(self.ctx.lib.doe_design_multi_run(self.h, len(classes), descs, int(mode)))
        self._keep = (keep, outs, descs)
        if mode == 1:  # the graph reads and writes these tensors on every relaunch
            self._graph_keep = self._keep
        return outs
