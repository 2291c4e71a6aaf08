#!/usr/bin/env python
"""Benchmark of the propagate-and-retrieve engine on B200.

Default workload (one "step" = one pass over the whole batch): the batched
angular-spectrum focus sweep of 64 fields of 1024x1024 complex64 (pitch 4 um,
wavelength per field from {450, 532, 633} nm, Gaussian beam of waist 200-800 um
times a seeded phase screen of 20 random Zernike terms up to radial order 6 with
rms 0-3 rad), each propagated to 64 distances drawn uniformly in 15-48 mm with
the band-limited, raised-cosine-apodised transfer function: 4096 propagations
per step. Inputs (512 MiB) and outputs (32 GiB) are larger than L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0). `--impl reference` times the FP64 CPU port of the
reference's propagateAngularSpectrum (the reference is JavaScript and no JS
runtime exists on the GPU box) on all host cores over a bounded sample.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

NX = NY = 1024
NFIELDS, NZ = 64, 64
DX = 4e-6
LAMBDAS = (450e-9, 532e-9, 633e-9)
BYTES_PER_PX = 16  # read complex64 spectrum + write complex64 output, per output plane
# profiler labels of the two focus-sweep passes (CUDA-core and tensor-core forms)
SWEEP_PASSES = {"asm_sweep_col": "column", "tc_sweep_col": "column", "fft_row_inv": "row", "tc_sweep_row": "row"}


TRAFFIC_RECORD = "traffic_sweep_1024.md"


def recorded_traffic(kernel, planes_per_launch):
    """DRAM bytes of one launch of `kernel` (this many planes) from the committed
    ncu capture record of the sweep passes (its table rows read `| kernel | dram
    bytes per plane | ... |`); None when the kernel has no record."""
    path = os.path.join(ROOT, "profiles", TRAFFIC_RECORD)
    if not os.path.exists(path):
        return None
    for line in open(path):
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) >= 2 and cells[0] == f"`{kernel}`":
            try:
                return float(cells[1]) * planes_per_launch
            except ValueError:
                return None
    return None
METRIC = "1024^2 ASM props/s (batched band-limited focus sweep)"
CONFIG = {"workload": "asm_focus_sweep", "fields": NFIELDS, "distances_per_field": NZ, "grid": [NX, NY],
          "pitch_um": DX * 1e6, "lambda_nm": [450, 532, 633], "z_mm": [15, 48], "band_limit": True,
          "soft_edge": 0.02, "l2_flush": "inputs 512 MiB and outputs 32 GiB exceed L2"}


def xorshift_stream(seed):
    """makeRng (reference src/doe.js:65-75) as a Python generator of [0, 1) doubles."""
    s = (int(seed) & 0xFFFFFFFF) or 1
    while True:
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        yield s / 4294967296.0


def zernike_terms(nmax=6):
    return [(n, m) for n in range(1, nmax + 1) for m in range(-n, n + 1, 2)]


def workload_params(seed=2024):
    """Per-field wavelength, waist, rms, Zernike terms/coefficients and distances."""
    rng = xorshift_stream(seed)
    terms = zernike_terms()
    fields = []
    for f in range(NFIELDS):
        lam = LAMBDAS[int(next(rng) * 3) % 3]
        waist = 200e-6 + 600e-6 * next(rng)
        rms = 3.0 * next(rng)
        order = sorted(range(len(terms)), key=lambda k: next(rng))[:20]
        coef = [(terms[k], 2 * next(rng) - 1) for k in order]
        z = [15e-3 + 33e-3 * next(rng) for _ in range(NZ)]
        fields.append({"lam": lam, "waist": waist, "rms": rms, "coef": coef, "z": z})
    return fields


def synth_fields(params, device):
    """Complex64 fields on the device: Gaussian amplitude x exp(i * Zernike screen)."""
    import torch
    n = NX
    i = torch.arange(n, device=device, dtype=torch.float64)
    u = (i - n / 2) / (n / 2)
    V, U = torch.meshgrid(u, u, indexing="ij")
    r = torch.hypot(U, V)
    th = torch.atan2(V, U)
    disc = r <= 1
    x = (i - n / 2) * DX
    Y, X = torch.meshgrid(x, x, indexing="ij")
    r2 = X * X + Y * Y
    basis = {}
    for (nn, m) in zernike_terms():
        am = abs(m)
        rad = torch.zeros_like(r)
        for s in range((nn - am) // 2 + 1):
            c = ((-1) ** s) * math.factorial(nn - s) / (
                math.factorial(s) * math.factorial((nn + am) // 2 - s) * math.factorial((nn - am) // 2 - s))
            rad = rad + c * r ** (nn - 2 * s)
        ang = torch.cos(m * th) if m >= 0 else torch.sin(-m * th)
        basis[(nn, m)] = torch.where(disc, rad * ang, torch.zeros_like(r))
    out = torch.empty((len(params), n, n), dtype=torch.complex64, device=device)
    for f, p in enumerate(params):
        ph = torch.zeros_like(r)
        for (t, a) in p["coef"]:
            ph = ph + a * basis[t]
        cur = torch.sqrt(torch.mean(ph[disc] ** 2))
        ph = ph * (p["rms"] / cur if cur > 0 else 0.0)
        amp = torch.exp(-r2 / (p["waist"] ** 2))
        out[f] = torch.polar(amp, ph).to(torch.complex64)
    return out


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Algorithmic bytes per pixel of each design pass: the complex64 work plane read
# and written (16 B) plus the FP32 side planes the pass must read or write.
PASS_BYTES_PX = {
    "design_col_fwd": 24, "design_col_back": 24,              # + the tabulated transfer function (8 B)
    "design_row_wgs_first": 32, "design_row_wgs_target": 32,  # W in, U out, t, m in, w in/out
    "design_row_wgs_constrain": 28,                           # U in, t, m, w in, W out
    "design_row_doe_update": 24, "design_row_doe_last": 16,   # W in/out, A in, phase out
    "design_row_doe_fwd": 16,                                 # A, phase in, W out
    "design_col_fourier": 28, "design_col_fourier_wgs": 36,   # W in/out, t, m in, amplitude out (+ w in/out)
    "design_row_gs_target": 24, "design_row_gs_final": 20,    # W in/out, t, m in (final: amplitude out)
    # the cluster-resident WGS loop, one launch for the fixed 100 iterations: only the
    # side planes move (t, m, w in + w out twice, A in, phase out, the table twice)
    "design_wgs_cluster": 52 * 100,
}


def kernel_roofline(prof, px_per_launch, table=None):
    """Roofline of the dominant kernel of a profiled step (each launch timed alone
    between CUDA events on its stream): its algorithmic bytes per launch (bytes
    per pixel x pixels per launch) over its average launch time."""
    table = PASS_BYTES_PX if table is None else table
    known = {k: v for k, v in prof.items() if k in table and v[1] > 0}
    if not known:
        return None
    peak, peak_kind = peaks()
    name, (tot_ms, cnt) = max(known.items(), key=lambda kv: kv[1][0])
    avg_s = tot_ms / cnt / 1e3
    bpl = table[name] * px_per_launch
    ach = bpl / avg_s / 1e9
    return {"bound": "hbm", "kernel": name, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_kind": peak_kind, "bytes_per_px": table[name], "bytes_per_launch": bpl,
            "avg_launch_us": avg_s * 1e6, "launches": cnt, "traffic": None,
            "per_kernel_ms": {k: round(v[0], 4) for k, v in prof.items()}}


WGS_CONFIG = {"workload": "wgs256", "grid": [256, 256], "max_iterations": 100,
              "goal": "screen RMSE <= 1% (src/projector.js:554-595)", "pitch_um": 8, "lambda_nm": 532, "z_mm": 30,
              "illumination": "rect, 0.9 N dx, raised-cosine edge 2 dx (src/doe.js:979-1000)",
              "targets": "3-8 seeded rectangles 4-40 px in the central 128^2, autoRoi", "band_limit": False}


DESIGN_TUNE = [True]  # --no-design-tune clears it


def tune_wgs(ctx, n_designs, rank=0, trial_iterations=4):
    """Design-pass autotuning (doe_autotune_design) on this rank's own C1 batch,
    before any timing: shape variants of the passes and the cluster-resident loop."""
    import torch
    from diffractiveopticalelement_b200 import batch
    ill, irr, roi, tgt, ph = wgs_inputs(n_designs, seed0=1 + rank * n_designs)
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()
    ch = batch.autotune_design(ctx, f32(ill), f32(tgt), f32(ph), nx=WGS_N, ny=WGS_N, dx=WGS_DX, lam=WGS_LAM,
                               z=WGS_Z, iterations=WGS_ITERS, roi=f32(roi), trial_iterations=trial_iterations)
    return {"row_variant": ch[0], "col_variant": ch[1], "cluster_loop": ch[2], "trial_iterations": trial_iterations,
            "tuner": "doe_autotune_design (fastest of every pass shape variant and the cluster loop, timed)"}


def measure_wgs(ctx, device, designs, warmup, steps, surrogate_steps, cpu, rank=0, world=1):
    """C1 (plain GPU WGS to the goal) and C4 (surrogate warm start + WGS to the goal)
    on the same seeded designs, the fixed 100-iteration loop (all designs active,
    profiled for the per-kernel roofline), and the CPU port on all host threads and
    on one."""
    import torch
    import torch.distributed as dist
    tuning = tune_wgs(ctx, designs, rank) if DESIGN_TUNE[0] else None
    r = run_wgs(ctx, device, designs, max(warmup, 3), steps, goal=0.01, rank=rank)
    fixed = run_wgs(ctx, device, designs, 1, 1, rank=rank)
    ms, reached = r["ms_per_step"], r["reached"]
    if world > 1:
        t = torch.tensor([ms, reached], dtype=torch.float64, device=device)
        dist.all_reduce(t[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        ms, reached = float(t[0].item()), int(t[1].item())
    r.pop("_used")
    roof = kernel_roofline(fixed.pop("_prof"), designs * WGS_N * WGS_N)
    r.pop("_prof", None)
    if roof:
        roof["basis"] = ("dominant pass of the fixed 100-iteration loop (every design active): bytes per pixel x "
                         "designs x 256^2 over its average launch time")
        # FFT arithmetic of the fixed loop: 4 2-D FFTs per iteration at 5 N^2 log2(N^2) FLOP each
        flop = 20.0 * WGS_N * WGS_N * np.log2(WGS_N * WGS_N) * WGS_ITERS * designs
        roof["fft_tflops"] = flop / (fixed["ms_per_step"] / 1e3) / 1e12
        roof["fft_basis"] = "20 N^2 log2(N^2) FLOP per WGS iteration (4 2-D FFTs), fixed 100-iteration loop"
    out = {"metric": WGS_METRIC, "value": reached / (ms / 1e3), "unit": "designs/s", "ms_per_step": ms,
           "config": dict(WGS_CONFIG, designs=designs, design_tuning=tuning), "roofline": roof, "wgs256": r,
           "fixed_100_iterations": fixed, "gpu_launches": int(r["gpu_launches_per_step"] * steps)}
    if surrogate_steps > 0:
        warm = run_warm(ctx, device, designs, surrogate_steps)
        warm["vs_plain"] = warm["designs_per_s"] / out["value"] if out["value"] else None
        out["surrogate_warm_start"] = warm
    out["cpu_baseline"] = wgs_cpu_baseline() if cpu else None
    if cpu:
        one = wgs_cpu_baseline(n_designs=2, threads=1)
        out["cpu_baseline"]["single_core"] = {"value": one["value"], "cores": 1, "sample": one["sample"]}
    return out


def main_wgs(args, ctx, device, rank, world, local):
    """--workload wgs256: batched image-plane WGS designs/s to screen RMSE <= 1%."""
    sampler = ClockSampler(local)
    steps = max(1, args.steps if args.steps != 20 else 3)
    sampler.start()
    body = measure_wgs(ctx, device, args.designs, args.warmup, steps, args.surrogate_steps,
                       rank == 0 and world == 1 and not args.no_cpu_baseline, rank, world)
    clocks = sampler.stop()
    if rank == 0:
        line = dict(body, n_gpus=world, steps=steps, warmup=max(args.warmup, 3), higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="fp32 fields, fp64 reductions", data="synthetic",
                    clocks=clocks, e2e=None)
        line["config"]["l2_flush"] = f"{args.designs} designs x 4 MiB of state exceed L2"
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


# ----------------------------------------------------------------- multi-plane 2048^2 workload
MP_N, MP_B, MP_ITERS, MP_DX, MP_LAM, MP_Z = 2048, 4, 100, 8e-6, 532e-9, (0.025, 0.030, 0.035)
MP_METRIC = "4 x 2048^2 three-plane GS design-iterations/s (batched, flat start)"
MP_CONFIG = {"workload": "multiplane2048", "designs": MP_B, "grid": [MP_N, MP_N], "planes_mm": [25, 30, 35],
             "iterations": MP_ITERS, "pitch_um": 8, "lambda_nm": 532, "init": "flat (src/doe.js:568)",
             "targets": "per plane 3-8 seeded rectangles 32-320 px in the central 1024^2, amplitude sqrt(I) and "
                        "autoRoi as designMultiPlane (src/projector.js:675-690)",
             "band_limit": False, "l2_flush": "4 designs x 3 planes x 2048^2 state (~600 MB) exceed L2"}


def mp_inputs(n=MP_N, B=MP_B):
    import diffractiveopticalelement_b200 as E
    from diffractiveopticalelement_b200.projector import autoRoi, rectangles_target
    ill = E.illuminationProfile("rect", n, n, MP_DX, MP_DX, {})
    w, wr = min(1024, n // 2), (max(4, n // 64), max(8, n * 5 // 32))
    irr = np.array([[rectangles_target(n, n, 1000 * d + p + 1, window=w, width=wr) for p in range(len(MP_Z))]
                    for d in range(B)])
    tgt = np.sqrt(np.maximum(0.0, irr))
    roi = np.array([[autoRoi(irr[d, p], n, n) for p in range(len(MP_Z))] for d in range(B)])
    return ill, irr, tgt, roi


def mp_cpu_baseline(iters=1, threads=None):
    """Oracle multi-plane GS at 2048^2: one design per host thread for `iters`
    iterations (the full 100 would take minutes per design); design-iterations/s."""
    from oracle import oracle as O
    O.build()
    threads = threads or os.cpu_count() or 1
    nd = threads
    ill, irr, tgt, roi = mp_inputs(B=1)

    def one(_):
        O.multiplane(ill, list(MP_Z), list(tgt[0]), list(roi[0]), None, nx=MP_N, ny=MP_N, dx=MP_DX, lam=MP_LAM,
                     iterations=iters)

    from concurrent.futures import ThreadPoolExecutor
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(one, range(nd)))
    dt = time.perf_counter() - t0
    return {"value": nd * iters / dt, "unit": "design-iterations/s", "cores": threads, "kind": "port",
            "sample": f"{nd} copies of design 0 x {iters} iteration(s) of the 3-plane 2048^2 loop, one per thread, "
                      f"FP64 C restatement of gerchbergSaxtonMultiPlane (no JS runtime on this box)"}


def measure_multiplane(ctx, device, warmup, steps, cpu, e2e_on, rank=0, world=1):
    """C5: batched 4 x 2048^2 three-plane GS, 100 iterations from a flat start."""
    import torch
    import torch.distributed as dist
    import diffractiveopticalelement_b200 as E
    from diffractiveopticalelement_b200 import batch
    n = MP_N * MP_N
    P = len(MP_Z)
    ill, irr, tgt, roi = mp_inputs()
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device)
    d_ill, d_tgt, d_roi = f32(ill), f32(tgt).reshape(MP_B * P, n), f32(roi).reshape(MP_B * P, n)
    d_ph = torch.zeros((MP_B, n), dtype=torch.float32, device=device)
    res = {}
    tuning = None
    if DESIGN_TUNE[0]:  # the 2048-point design-pass shapes, timed on GS over plane 0 of each design
        ch = batch.autotune_design(ctx, d_ill, f32(tgt[:, 0]), d_ph, nx=MP_N, ny=MP_N, dx=MP_DX, lam=MP_LAM,
                                   z=MP_Z[0], iterations=MP_ITERS, algorithm="gs", trial_iterations=2)
        tuning = {"row_variant": ch[0], "col_variant": ch[1],
                  "tuner": "doe_autotune_design on gerchbergSaxton at 2048^2 (the multi-plane loop's passes)"}

    def step():
        d_ph.zero_()
        res["r"] = batch.multiplane_batch(ctx, d_ill, d_tgt, d_ph, list(MP_Z), nx=MP_N, ny=MP_N, dx=MP_DX,
                                          lam=MP_LAM, iterations=MP_ITERS, roi=d_roi)

    for _ in range(max(warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    n0 = ctx.lib.doe_ctx_launch_count(ctx.h)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    e1.synchronize()
    launches = int(ctx.lib.doe_ctx_launch_count(ctx.h) - n0)
    ms = e0.elapsed_time(e1) / steps
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = MP_B * MP_ITERS * world / (ms / 1e3)
    ctx.lib.doe_ctx_set_profiling(ctx.h, 1)
    step()
    torch.cuda.synchronize()
    prof = profile_read(None, ctx)
    ctx.lib.doe_ctx_set_profiling(ctx.h, 0)
    peak, peak_kind = peaks()
    roof = kernel_roofline(prof, MP_B * n)
    if roof:
        roof["basis"] = "dominant pass: bytes per pixel x 4 designs x 2048^2 over its average launch time"
        alg = 96.0 * n * MP_B * MP_ITERS  # 6 propagations per iteration x 16 B/px
        roof["whole_loop"] = {"achieved": alg / (ms / 1e3) / 1e9, "frac": alg / (ms / 1e3) / 1e9 / peak,
                              "basis": "96 B/px per iteration (6 propagations x 16 B/px)"}
    err = res["r"]["error"][:, -1].cpu().numpy()
    e2e = None
    if e2e_on:  # one design through the host-buffer call (FP64 planes, copies inside the region)
        planes = [{"z": MP_Z[p], "targetAmp": tgt[0, p], "roi": roi[0, p]} for p in range(P)]
        o = {"nx": MP_N, "dx": MP_DX, "lambda": MP_LAM, "iterations": MP_ITERS}
        E.gerchbergSaxtonMultiPlane(ill, planes, dict(o, iterations=2))
        t0 = time.perf_counter()
        E.gerchbergSaxtonMultiPlane(ill, planes, o)
        dt = time.perf_counter() - t0
        e2e = {"value": MP_ITERS / dt, "unit": "design-iterations/s", "h2d_bytes_per_step": (2 + 2 * P) * n * 8,
               "d2h_bytes_per_step": n * 8,
               "sample": "design 0 through gerchbergSaxtonMultiPlane (doe_multiplane, FP64 host planes)"}
    cb = None
    if cpu:
        cb = mp_cpu_baseline()
        one = mp_cpu_baseline(threads=1)
        cb["single_core"] = {"value": one["value"], "cores": 1, "sample": one["sample"]}
    return {"metric": MP_METRIC, "value": value, "unit": "design-iterations/s", "ms_per_step": ms,
            "config": dict(MP_CONFIG, design_tuning=tuning), "roofline": roof,
            "final_error": {"median": float(np.median(err)), "max": float(err.max())},
            "cpu_baseline": cb, "e2e": e2e, "gpu_launches": launches}


def main_multiplane(args, ctx, device, rank, world, local):
    """--workload multiplane2048: batched 4 x 2048^2 three-plane GS."""
    steps = max(1, args.steps if args.steps != 20 else 2)
    sampler = ClockSampler(local)
    sampler.start()
    body = measure_multiplane(ctx, device, args.warmup, steps, rank == 0 and world == 1 and not args.no_cpu_baseline,
                              rank == 0 and not args.no_e2e, rank, world)
    clocks = sampler.stop()
    if rank == 0:
        line = dict(body, n_gpus=world, steps=steps, warmup=max(args.warmup, 3), higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="fp32 fields, fp64 reductions", data="synthetic",
                    clocks=clocks)
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


# ----------------------------------------------------------------- uneven far-field batch
UN_COUNT, UN_ITERS, UN_DX, UN_LAM = 512, 200, 8e-6, 532e-9
UN_SIZES, UN_PROBS = (128, 256, 512, 1024), (0.4, 0.3, 0.2, 0.1)
UN_METRIC = "far-field GS designs/s, 512 designs of uneven size (128^2-1024^2), one graph launch"
UN_CONFIG = {"workload": "farfield_uneven", "designs": UN_COUNT, "sizes": list(UN_SIZES), "probabilities": list(UN_PROBS),
             "iterations": UN_ITERS, "algorithm": "fourierCgh (designDOE far-field default)", "pitch_um": 8,
             "lambda_nm": 532, "z": "N dx^2 / lambda (src/projector.js:359-361)",
             "targets": "seeded k x k Gaussian spot arrays (sigma 1.5 px, k 4..32, weights 1 or U[0.5, 1]) in the "
                        "central half window, ROI autoRoi", "illumination": "designDOE default disc",
             "l2_flush": "512 designs of state (~3 GB) exceed L2"}


def uneven_specs(seed=7):
    from diffractiveopticalelement_b200.doe import makeRng
    rng = makeRng(seed)
    cum = np.cumsum(UN_PROBS)
    sizes = []
    for _ in range(UN_COUNT):
        u = rng()
        sizes.append(UN_SIZES[int(np.searchsorted(cum, u, side="right"))] if u < cum[-1] else UN_SIZES[-1])
    return sizes


def uneven_inputs(sizes):
    """Per size class: illumination, target amplitudes, ROIs, initial phases, irradiance."""
    import diffractiveopticalelement_b200 as E
    from diffractiveopticalelement_b200 import surrogate as S
    from diffractiveopticalelement_b200.projector import autoRoi
    out = {}
    for n in UN_SIZES:
        idx = [k for k, s in enumerate(sizes) if s == n]
        if not idx:
            continue
        ill = E.discMask(n, n, UN_DX, UN_DX, (n * UN_DX / 2) * 0.95, soft=2 * UN_DX)
        irr = np.array([S.spot_array_target(n, 5000 + k) for k in idx])
        roi = np.array([autoRoi(t, n, n) for t in irr])
        tgt = np.array([E.prepareTargetAmp(t, ill) for t in irr])
        ph = np.array([E.randomPhase(n, n, 5000 + k) for k in idx])
        out[n] = (ill, irr, roi, tgt, ph)
    return out


def uneven_cpu_baseline(iters=2):
    """Oracle fourierCgh: one design per size for `iters` iterations on one thread,
    extrapolated to the workload (counts x 200 iterations) over all host threads
    (and over one)."""
    from oracle import oracle as O
    O.build()
    sizes = uneven_specs()
    inp = uneven_inputs([n for n in UN_SIZES])  # one design per size
    per_iter = {}
    for n in UN_SIZES:
        ill, irr, roi, tgt, ph = inp[n]
        t0 = time.perf_counter()
        O.design("fourier", ill, tgt[0], nx=n, ny=n, dx=UN_DX, lam=UN_LAM, z=n * UN_DX ** 2 / UN_LAM,
                 iterations=iters, roi=roi[0], init_phase=ph[0])
        per_iter[n] = (time.perf_counter() - t0) / iters
    threads = os.cpu_count() or 1
    t1 = sum(per_iter[n] * UN_ITERS for n in sizes)
    timing = ", ".join(f"{n}^2: {1e3 * per_iter[n]:.1f} ms/it" for n in UN_SIZES)
    return {"value": UN_COUNT / (t1 / threads), "unit": "designs/s", "cores": threads, "kind": "port",
            "sample": f"one design per size x {iters} iterations of the FP64 C restatement of fourierCgh on one "
                      f"thread ({timing}), extrapolated to the 512-design, 200-iteration workload over {threads} "
                      f"threads",
            "single_core": {"value": UN_COUNT / t1, "cores": 1,
                            "sample": "the same per-iteration timings extrapolated to one thread"}}


def measure_uneven(ctx, device, warmup, steps, cpu, rank=0, world=1):
    """C3: 512 far-field GS designs of four sizes in one CUDA-graph launch."""
    import torch
    import torch.distributed as dist
    from diffractiveopticalelement_b200 import batch
    sizes = uneven_specs(seed=7 + rank)
    inp = uneven_inputs(sizes)
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device)
    classes, ph0 = [], []
    for n, (ill, irr, roi, tgt, ph) in inp.items():
        p0 = f32(ph)
        ph0.append(p0)
        classes.append({"nx": n, "dx": UN_DX, "lam": UN_LAM, "z": n * UN_DX ** 2 / UN_LAM, "algorithm": "fourier",
                        "iterations": UN_ITERS, "illumination": f32(ill), "target_amp": f32(tgt), "roi": f32(roi),
                        "phase": p0.clone()})
    m = batch.DesignMulti(ctx)
    tuning = {}
    if DESIGN_TUNE[0]:  # design-pass shapes per size class, on that class's own designs, before any timing
        for cl in classes:
            kw = {k: cl[k] for k in ("nx", "dx", "lam", "z", "algorithm", "iterations", "roi")}
            ch = batch.autotune_design(ctx, cl["illumination"], cl["target_amp"], cl["phase"], ny=cl["nx"],
                                       trial_iterations=3, **kw)
            tuning[str(cl["nx"])] = {"row_variant": ch[0], "col_variant": ch[1]}

    def reset():
        for cl, p in zip(classes, ph0):
            cl["phase"].copy_(p)

    reset()
    m.run(classes, 0)  # sizes the scratch of every class
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reset()
    e0.record()
    m.run(classes, 0)  # direct submission (no graph), for comparison
    e1.record()
    e1.synchronize()
    ms_direct = e0.elapsed_time(e1)
    reset()
    m.run(classes, 1)  # capture + launch
    torch.cuda.synchronize()
    for _ in range(max(warmup, 3) - 1):
        reset()
        m.run(None, 2)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    n0 = ctx.lib.doe_ctx_launch_count(ctx.h)
    e0.record()
    for _ in range(steps):
        reset()
        outs = m.run(None, 2)
    e1.record()
    e1.synchronize()
    launches = int(ctx.lib.doe_ctx_launch_count(ctx.h) - n0)
    ms = e0.elapsed_time(e1) / steps
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = UN_COUNT * world / (ms / 1e3)
    counts = {n: sum(1 for s_ in sizes if s_ == n) for n in UN_SIZES}
    flops = sum(c * 10.0 * n * n * np.log2(n * n) * UN_ITERS for n, c in counts.items())
    per_iter_px = PASS_BYTES_PX["design_col_fourier"] + PASS_BYTES_PX["design_row_doe_update"]
    bytes_ = sum(c * float(per_iter_px) * n * n * UN_ITERS for n, c in counts.items())
    peak, peak_kind = peaks()
    err = np.concatenate([o["error"][:, -1].cpu().numpy() for o in outs])
    cb = uneven_cpu_baseline() if cpu else None
    m.close()
    return {"metric": UN_METRIC, "value": value, "unit": "designs/s", "ms_per_step": ms,
            "config": dict(UN_CONFIG, counts={str(k): v for k, v in counts.items()}, design_tuning=tuning),
            "roofline": {"bound": "hbm", "kernel": "whole graph (column + row pass per iteration, all classes)",
                         "achieved": bytes_ / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": bytes_ / (ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None,
                         "basis": f"{per_iter_px} B/px per iteration (far-field column pass "
                                  f"{PASS_BYTES_PX['design_col_fourier']} + row pass "
                                  f"{PASS_BYTES_PX['design_row_doe_update']}), all designs, over the graph's time",
                         "fft_tflops": flops / (ms / 1e3) / 1e12,
                         "fft_basis": "10 N^2 log2(N^2) FLOP per iteration"},
            "graph": {"ms_per_step_graph": ms, "ms_per_step_direct": ms_direct, "kernels_per_step": launches / steps},
            "final_error": {"median": float(np.median(err)), "max": float(err.max())},
            "cpu_baseline": cb, "e2e": None, "gpu_launches": launches}


def main_uneven(args, ctx, device, rank, world, local):
    """--workload farfield_uneven: 512 far-field GS designs of four sizes in one CUDA-graph launch."""
    steps = max(1, args.steps if args.steps != 20 else 3)
    sampler = ClockSampler(local)
    sampler.start()
    body = measure_uneven(ctx, device, args.warmup, steps, rank == 0 and world == 1 and not args.no_cpu_baseline,
                          rank, world)
    clocks = sampler.stop()
    if rank == 0:
        line = dict(body, n_gpus=world, steps=steps, warmup=max(args.warmup, 3), higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="fp32 fields, fp64 reductions", data="synthetic",
                    clocks=clocks)
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def profile_read(E, ctx):
    names = C.create_string_buffer(64 * 64)
    ms = (C.c_double * 64)()
    cnt = (C.c_ulonglong * 64)()
    L = ctx.lib
    L.doe_ctx_profile_read.restype = C.c_int
    L.doe_ctx_profile_read.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_double),
                                       C.POINTER(C.c_ulonglong)]
    n = L.doe_ctx_profile_read(ctx.h, 64, names, 64, ms, cnt)
    out = {}
    for k in range(max(n, 0)):
        nm = names.raw[k * 64:(k + 1) * 64].split(b"\0")[0].decode()
        out[nm] = (ms[k], int(cnt[k]))
    return out


# ----------------------------------------------------------------- widened rows
# The reference's other callers of the transforms (Fresnel propagation, focus stack
# and full screen metrics, error-diffusion quantiser, hologram reconstruction):
# each timed through its reference-facing C-ABI call with FP64 host planes (the
# only form the reference has), with its device kernels timed alone by the
# context's per-launch events and the FP64 C restatement timed on one host core.
WR_LAM, WR_Z = 532e-9, 0.03


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _row_block(ctx, metric, unit, units, call, alg_bytes, basis, h2d, d2h, reps, cpu_fn, cpu_units, cpu_desc,
               config):
    """Time `call` (one reference-facing call, `units` units of work) end to end,
    then once more with per-launch device timing; `alg_bytes` is the call's
    algorithmic device traffic (the roofline basis)."""
    L = ctx.lib
    for _ in range(3):
        call()
    t0 = time.perf_counter()
    for _ in range(reps):
        call()
    dt = (time.perf_counter() - t0) / reps
    L.doe_ctx_set_profiling(ctx.h, 1)
    call()
    prof = profile_read(None, ctx)
    L.doe_ctx_set_profiling(ctx.h, 0)
    dev_ms = sum(v[0] for v in prof.values())
    name, (kms, kcnt) = max(prof.items(), key=lambda kv: kv[1][0])
    peak, peak_kind = peaks()
    achieved = alg_bytes / (dev_ms / 1e3) / 1e9 if dev_ms > 0 else None
    out = {"metric": metric, "value": units / dt, "unit": unit, "ms_per_call": dt * 1e3, "config": config,
           "e2e": {"value": units / dt, "unit": unit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
           "device": {"value": units / (dev_ms / 1e3) if dev_ms > 0 else None, "unit": unit,
                      "kernel_ms_per_call": dev_ms,
                      "note": "sum of the call's kernel durations (each launch timed alone), copies excluded"},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak if achieved else None, "peak_kind": peak_kind, "basis": basis,
                        "algorithmic_bytes_per_call": alg_bytes, "dominant_kernel": name,
                        "dominant_share": kms / dev_ms if dev_ms > 0 else None, "traffic": None,
                        "per_kernel_ms": {k: round(v[0], 4) for k, v in prof.items()}}}
    if cpu_fn is not None:
        t0 = time.perf_counter()
        cpu_fn()
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": cpu_units / tc, "unit": unit, "cores": 1, "kind": "port",
                               "sample": cpu_desc}
    return out


def measure_widened(ctx, cpu):
    """One block per widened row, each a few seconds of GPU and host time."""
    O = None
    if cpu:
        from oracle import oracle as O
        O.build()
    L = ctx.lib
    rng = np.random.default_rng(11)
    out = {}

    # f1: propagateFresnelFFT, 1024^2 beam with a seeded phase screen
    n1 = 1024
    y, x = np.mgrid[0:n1, 0:n1]
    r2 = ((x - n1 / 2) ** 2 + (y - n1 / 2) ** 2) * DX * DX
    amp = np.exp(-r2 / (600e-6) ** 2).ravel()
    phs = rng.uniform(-np.pi, np.pi, n1 * n1)
    re, im = amp * np.cos(phs), amp * np.sin(phs)
    ore, oim, od = np.empty(n1 * n1), np.empty(n1 * n1), np.empty(2)
    out["fresnel"] = _row_block(
        ctx, "1024^2 single-FFT Fresnel propagations/s (propagateFresnelFFT, FP64 host planes)", "props/s", 1,
        lambda: ctx.check(L.doe_fresnel(ctx.h, _dp(re), _dp(im), n1, n1, DX, DX, WR_LAM, WR_Z, _dp(ore), _dp(oim),
                                        _dp(od))),
        n1 * n1 * 32, "32 B/px: FP64 complex plane read once and written once", n1 * n1 * 16, n1 * n1 * 16, 20,
        (lambda: O.fresnel(re, im, n1, n1, DX, DX, WR_LAM, WR_Z)) if O else None, 1,
        "one 1024^2 Fresnel propagation, FP64 C restatement of propagateFresnelFFT on one thread",
        {"grid": [n1, n1], "pitch_um": DX * 1e6, "lambda_nm": 532, "z_mm": WR_Z * 1e3})

    # a5 / a2: the reference's basic calls on one 1024^2 plane, in place
    w_re, w_im = re.copy(), im.copy()
    out["asm"] = _row_block(
        ctx, "1024^2 band-limited angular-spectrum propagations/s (propagateAngularSpectrumInPlace, FP64 host "
             "planes)", "props/s", 1,
        lambda: ctx.check(L.doe_asm(ctx.h, _dp(w_re), _dp(w_im), n1, n1, DX, DX, WR_LAM, WR_Z, 1, 1, 0.02)),
        n1 * n1 * 32, "32 B/px: FP64 complex plane read once and written once", n1 * n1 * 16, n1 * n1 * 16, 20,
        (lambda: O.asm(re, im, n1, n1, DX, DX, WR_LAM, WR_Z)) if O else None, 1,
        "one 1024^2 band-limited propagation, FP64 C restatement of propagateAngularSpectrum on one thread",
        {"grid": [n1, n1], "pitch_um": DX * 1e6, "lambda_nm": 532, "z_mm": WR_Z * 1e3, "band_limit": True})
    def fft_pair():  # forward then inverse, so that the plane stays bounded over the repeats
        ctx.check(L.doe_fft2d(ctx.h, _dp(w_re), _dp(w_im), n1, n1, 0))
        ctx.check(L.doe_fft2d(ctx.h, _dp(w_re), _dp(w_im), n1, n1, 1))

    out["fft2d"] = _row_block(
        ctx, "1024^2 2-D FFTs/s (fft2d, FP64 host planes, in place; forward and inverse alternate)", "ffts/s", 2,
        fft_pair, 2 * n1 * n1 * 32, "32 B/px per transform: FP64 complex plane read once and written once",
        2 * n1 * n1 * 16, 2 * n1 * n1 * 16, 10,
        (lambda: (O.fft2d(re, im, n1, n1), O.fft2d(re, im, n1, n1, inverse=True))) if O else None, 2,
        "one forward and one inverse 1024^2 FFT, FP64 C restatement of fft2d on one thread", {"grid": [n1, n1]})

    # f2: focus stack (ProjectorSystem.simulate at 16 distances, one forward FFT shared)
    n2, nz, dx2 = 512, 16, 8e-6
    y, x = np.mgrid[0:n2, 0:n2]
    half = 0.45 * n2
    illum = (((np.abs(x - n2 / 2) <= half) & (np.abs(y - n2 / 2) <= half)).astype(np.float64)).ravel()
    phase2 = rng.uniform(-np.pi, np.pi, n2 * n2)
    zs2 = np.linspace(0.025, 0.035, nz)
    s_re, s_im, s_d = np.empty(nz * n2 * n2), np.empty(nz * n2 * n2), np.empty(2 * nz)
    el_re, el_im = illum * np.cos(phase2), illum * np.sin(phase2)
    out["focus_stack"] = _row_block(
        ctx, "512^2 focus-stack planes/s (ProjectorSystem.simulate at 16 distances, FP64 host planes)",
        "planes/s", nz,
        lambda: ctx.check(L.doe_simulate_sweep(ctx.h, _dp(illum), _dp(phase2), n2, n2, dx2, dx2, WR_LAM, _dp(zs2),
                                               nz, 1, 0, 1, _dp(s_re), _dp(s_im), _dp(s_d))),
        n2 * n2 * (16 + nz * 24),
        "16 B/px element in, then per plane 8 B/px shared spectrum read + 16 B/px FP64 plane written",
        n2 * n2 * 16, nz * n2 * n2 * 16, 10,
        (lambda: [O.asm(el_re, el_im, n2, n2, dx2, dx2, WR_LAM, z) for z in zs2[:2]]) if O else None, 2,
        "2 band-limited 512^2 angular-spectrum planes of the element, FP64 C restatement on one thread",
        {"grid": [n2, n2], "distances": nz, "z_mm": [25, 35], "band_limit": True})

    # f2: screenMetrics, every field, on a 1024^2 screen
    tgt = np.zeros((n1, n1))
    tgt[384:640, 320:704] = 1.0
    tgt = tgt.ravel()
    roi = (tgt > 0).astype(np.float64)
    ill1 = np.ones(n1 * n1)
    ph1 = rng.uniform(-np.pi, np.pi, n1 * n1)
    mout = np.empty(18)
    out["screen_metrics"] = _row_block(
        ctx, "1024^2 screenMetrics evaluations/s (every field, FP64 host planes)", "screens/s", 1,
        lambda: ctx.check(L.doe_screen_metrics_full(ctx.h, _dp(re), _dp(im), n1, n1, DX, DX, _dp(tgt), _dp(roi),
                                                    _dp(ill1), _dp(ph1), DX, DX, 0, 0, _dp(mout))),
        n1 * n1 * 48, "48 B/px: six FP64 planes read once (field re/im, target, ROI, illumination, phase)",
        n1 * n1 * 48, 18 * 8, 20,
        (lambda: [O.screen_metrics_full(re, im, n1, n1, DX, DX, tgt, roi, ill1, ph1, DX, DX) for _ in range(10)])
        if O else None, 10, "ten 1024^2 screenMetrics, FP64 C restatement on one thread",
        {"grid": [n1, n1], "target": "binary rectangle with its ROI", "spot_grid": None})

    # f3: errorDiffusionQuantize of 512 designs of 256^2 (the image-plane batch)
    nb, n3 = 512, 256
    ph3 = rng.uniform(-4.0, 4.0, nb * n3 * n3)
    q3 = np.empty_like(ph3)
    out["error_diffusion"] = _row_block(
        ctx, "256^2 errorDiffusionQuantize phase maps/s (512 maps per call, 4 levels, serpentine)", "maps/s", nb,
        lambda: ctx.check(L.doe_error_diffusion(ctx.h, nb, n3 * n3, 4, 1, 1, _dp(ph3), _dp(q3))),
        nb * n3 * n3 * 16, "16 B/px: FP64 phase read once, FP64 levels written once (the scan is serial per map)",
        nb * n3 * n3 * 8, nb * n3 * n3 * 8, 5,
        (lambda: [O.error_diffusion(ph3[k * n3 * n3:(k + 1) * n3 * n3], 4) for k in range(64)]) if O else None, 64,
        "64 maps of 256^2, FP64 C restatement of errorDiffusionQuantize on one thread",
        {"maps": nb, "grid": [n3, n3], "levels": 4, "snake": True, "wrap_first": True})

    # f4: reconstructHologram, 1024^2 plate lit by a tilted plane wave, +-z in one batch
    kx = 2 * np.pi * 0.02 / DX
    xs = (np.arange(n1 * n1) % n1) * DX
    ref_re, ref_im = np.cos(kx * xs), np.sin(kx * xs)
    pl_re = (np.abs(re + ref_re) ** 2 + im ** 2)
    pl_re /= pl_re.max()
    pl_im = np.zeros_like(pl_re)
    h = [np.empty(n1 * n1) for _ in range(4)]
    out["hologram"] = _row_block(
        ctx, "1024^2 hologram reconstructions/s (reconstructHologram: real and virtual image, FP64 host planes)",
        "reconstructions/s", 1,
        lambda: ctx.check(L.doe_hologram_reconstruct(ctx.h, _dp(pl_re), _dp(pl_im), _dp(ref_re), _dp(ref_im), n1,
                                                     n1, DX, DX, WR_LAM, WR_Z, 0, 1, 0.02, *[_dp(a) for a in h],
                                                     None, None)),
        n1 * n1 * 64, "64 B/px: plate and reference FP64 complex planes read, two FP64 complex images written",
        n1 * n1 * 32, n1 * n1 * 32, 20,
        (lambda: O.reconstruct_hologram(pl_re, pl_im, ref_re, ref_im, n1, n1, DX, DX, WR_LAM, WR_Z)) if O else None,
        1, "one 1024^2 reconstruction (two angular-spectrum planes), FP64 C restatement on one thread",
        {"grid": [n1, n1], "band_limit": False, "z_mm": WR_Z * 1e3})
    return out


# ----------------------------------------------------------------- CPU (oracle port)
def cpu_sample(params, fields_np, nplanes, threads):
    """Time `nplanes` FP64 propagations of the workload on `threads` host threads."""
    from oracle import oracle as O
    O.build()
    jobs = []
    nf = len(fields_np)
    for k in range(nplanes):
        f = k % nf
        jobs.append((f, params[f]["lam"], params[f]["z"][(k // nf) % NZ]))
    planes = {}
    for f, _, _ in jobs:
        if f not in planes:
            a = fields_np[f].astype(np.complex128).ravel()
            planes[f] = (np.ascontiguousarray(a.real), np.ascontiguousarray(a.imag))
    idx = [0]
    lock = threading.Lock()

    def worker():
        while True:
            with lock:
                if idx[0] >= len(jobs):
                    return
                f, lam, z = jobs[idx[0]]
                idx[0] += 1
            re, im = planes[f]
            O.asm(re, im, NX, NY, DX, DX, lam, z, True, True, 0.02)  # ctypes releases the GIL

    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker) for _ in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return time.perf_counter() - t0


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    if args.workload == "farfield_uneven":
        cb = uneven_cpu_baseline()
        line = {"metric": UN_METRIC, "value": cb["value"], "unit": "designs/s", "n_gpus": args.gpus, "steps": 1,
                "warmup": 0, "ms_per_step": 1000.0 * UN_COUNT / cb["value"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": UN_CONFIG, "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "designs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    if args.workload == "multiplane2048":
        cb = mp_cpu_baseline()
        line = {"metric": MP_METRIC, "value": cb["value"], "unit": "design-iterations/s", "n_gpus": args.gpus,
                "steps": 1, "warmup": 0, "ms_per_step": 1000.0 / cb["value"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": MP_CONFIG, "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "design-iterations/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    if args.workload == "wgs256":
        for _ in range(args.warmup):
            wgs_cpu_baseline(n_designs=2)
        rs = [wgs_cpu_baseline() for _ in range(max(1, args.steps if args.steps != 20 else 1))]
        value = float(np.mean([r["value"] for r in rs]))
        cb = dict(rs[0], value=value)
        line = {"metric": WGS_METRIC, "value": value, "unit": "designs/s", "n_gpus": args.gpus, "steps": len(rs),
                "warmup": args.warmup, "ms_per_step": 1000.0 * (os.cpu_count() or 1) / max(value, 1e-12), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": "wgs256", "grid": [WGS_N, WGS_N], "max_iterations": WGS_ITERS},
                "cpu_baseline": cb,
                "e2e": {"value": value, "unit": "designs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    params = workload_params()
    # same field construction as the GPU arm (fields 0-3), evaluated on the host
    fields_np = synth_fields(params[:4], "cpu").numpy()
    threads = os.cpu_count() or 1
    per_step = threads
    for _ in range(args.warmup):
        cpu_sample(params, fields_np, min(per_step, 2), threads)
    times = [cpu_sample(params, fields_np, per_step, threads) for _ in range(args.steps)]
    t = sum(times)
    value = per_step * args.steps / t
    line = {"metric": METRIC, "value": value, "unit": "props/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": CONFIG,
            "cpu_baseline": {"value": value, "unit": "props/s", "cores": threads, "kind": "port",
                             "sample": f"{per_step} planes of the workload per step (fields 0-3), one plane per "
                                       f"thread, FP64 restatement of propagateAngularSpectrum; the reference "
                                       f"is JavaScript and no JS runtime exists on this machine"},
            "e2e": {"value": value, "unit": "props/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- image-plane WGS workload
WGS_N, WGS_ITERS, WGS_DX, WGS_LAM, WGS_Z = 256, 100, 8e-6, 532e-9, 0.03


def wgs_inputs(n_designs, seed0=1):
    """Seeded 256^2 image-plane WGS designs: rect-apodised square illumination,
    3-8 random rectangles (4-40 px) inside the central 128^2 window, auto ROI,
    random initial phase, target power-matched to the illumination."""
    import diffractiveopticalelement_b200 as E
    from diffractiveopticalelement_b200.projector import autoRoi, rectangles_target
    n = WGS_N
    ill = E.illuminationProfile("rect", n, n, WGS_DX, WGS_DX, {})
    irr, roi, tgt, ph = [], [], [], []
    for k in range(n_designs):
        t = rectangles_target(n, n, seed0 + k)
        irr.append(t)
        roi.append(autoRoi(t, n, n))
        tgt.append(E.prepareTargetAmp(t, ill))
        ph.append(E.randomPhase(n, n, seed0 + k))
    return ill, np.array(irr), np.array(roi), np.array(tgt), np.array(ph)


def wgs_cpu_baseline(n_designs=None, iters=WGS_ITERS, goal=0.01, threads=None):
    """Oracle WGS designs on `threads` host threads (default all; one design per
    thread), each stopped at the first iteration whose screen RMSE is <= goal (at
    most `iters`), the same rule as the GPU arm. Returns the rate of designs that
    met the goal."""
    from oracle import oracle as O
    O.build()
    threads = threads or os.cpu_count() or 1
    nd = n_designs or threads
    ill, irr, roi, tgt, ph = wgs_inputs(nd, seed0=1)
    used, ok = [0] * nd, [False] * nd
    idx = [0]
    lock = threading.Lock()

    def worker():
        while True:
            with lock:
                if idx[0] >= nd:
                    return
                k = idx[0]
                idx[0] += 1
            r = O.design("wgs", ill, tgt[k], nx=WGS_N, ny=WGS_N, dx=WGS_DX, lam=WGS_LAM, z=WGS_Z, iterations=iters,
                         roi=roi[k], init_phase=ph[k], rmse_goal=goal, screen_irr=irr[k])
            used[k] = r.get("iterationsUsed", iters)
            m = O.screen_metrics(r["amplitude"], np.zeros(WGS_N * WGS_N), WGS_N, WGS_N, WGS_DX, WGS_DX, irr[k], roi[k],
                                 ill, WGS_DX, WGS_DX)
            ok[k] = m["rmse"] <= goal

    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker) for _ in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    dt = time.perf_counter() - t0
    return {"value": sum(ok) / dt, "unit": "designs/s", "cores": threads, "kind": "port",
            "sample": f"{nd} designs of 256^2 WGS (seeds 1-{nd}) to screen RMSE <= {goal:g} (median "
                      f"{int(np.median(used))} iterations, {sum(ok)} met it) on {threads} thread(s), FP64 C "
                      f"restatement of weightedGerchbergSaxton (no JS runtime on this box)"}


def run_wgs(ctx, device, n_designs, warmup, steps, goal=0.0, iters=WGS_ITERS, rank=0):
    """Batched image-plane WGS: designs/s, screen RMSE of every design, kernel split.

    goal > 0: every design stops at the first iteration whose screen RMSE is <= goal
    (at most `iters`); the rate counts only designs whose returned screen meets it."""
    import torch
    from diffractiveopticalelement_b200 import batch
    L = ctx.lib
    ill, irr, roi, tgt, ph = wgs_inputs(n_designs, seed0=1 + rank * n_designs)  # rank r: its own designs
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device)
    d_ill = f32(ill)
    d_tgt, d_roi, d_irr, d_ph0 = f32(tgt), f32(roi), f32(irr), f32(ph)
    d_ph = torch.empty_like(d_ph0)
    res = {}

    def step():
        d_ph.copy_(d_ph0)  # the initial phase is an input of every design
        res["d"] = batch.design_batch(ctx, d_ill, d_tgt, d_ph, nx=WGS_N, ny=WGS_N, dx=WGS_DX, lam=WGS_LAM, z=WGS_Z,
                                      iterations=iters, roi=d_roi, rmse_goal=goal)
        res["m"] = batch.screen_metrics_batch(ctx, res["d"]["amplitude"], d_irr, d_ill, nx=WGS_N, ny=WGS_N,
                                              sdx=WGS_DX, roi=d_roi)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    n0 = L.doe_ctx_launch_count(ctx.h)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    launches = int(L.doe_ctx_launch_count(ctx.h) - n0)
    L.doe_ctx_set_profiling(ctx.h, 1)
    step()
    torch.cuda.synchronize()
    prof = profile_read(None, ctx)
    L.doe_ctx_set_profiling(ctx.h, 0)
    met = res["m"].cpu().numpy()
    rm = met[:, 0]
    used = res["d"]["iterations_used"].cpu().numpy()
    reached = int(np.sum(rm <= (goal if goal else 0.01)))
    out = {"designs": n_designs, "max_iterations": iters, "ms_per_step": ms,
           "designs_per_s": (reached if goal else n_designs) / (ms / 1e3),
           "screen_rmse": {"median": float(np.median(rm)), "min": float(rm.min()), "max": float(rm.max()),
                           "le_1pct": int(np.sum(rm <= 0.01))},
           "efficiency_median": float(np.median(met[:, 1])), "gpu_launches_per_step": launches / steps,
           "per_kernel_ms": {k: round(v[0], 3) for k, v in prof.items()}, "_prof": prof}
    if goal:
        out.update({"goal": goal, "reached": reached,
                    "iterations_used": {"median": float(np.median(used)), "min": int(used.min()),
                                        "max": int(used.max())},
                    "_used": used})
    return out


WGS_METRIC = "256^2 image-plane WGS designs/s to screen RMSE<=1% (plain GPU start, batched)"


def run_warm(ctx, device, n_designs, steps, goal=0.01):
    """The surrogate arm: train the U-Net on the GPU (physics loss on a seeded
    mixture of rectangles / spot arrays / smooth gradients, held apart from the
    evaluation seeds), then time surrogate inference + WGS to the goal on the same
    designs as the plain arm. Training time is reported, not timed in the rate."""
    import torch
    import diffractiveopticalelement_b200 as E
    from diffractiveopticalelement_b200 import batch, surrogate as S
    from diffractiveopticalelement_b200.projector import autoRoi
    n = WGS_N
    t0 = time.perf_counter()
    ill = E.illuminationProfile("rect", n, n, WGS_DX, WGS_DX, {})
    irr_t = S.training_targets(n, 4096, 1_000_000)
    roi_t = np.array([autoRoi(t, n, n) for t in irr_t])
    tgt_t = np.array([E.prepareTargetAmp(t, ill) for t in irr_t])
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device)
    d_ill = f32(ill)
    model = S.Surrogate(n=n, base=32, levels=4, max_batch=16, seed=1, ctx=ctx)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    hist = S.train(model, f32(irr_t), f32(roi_t), d_ill, f32(tgt_t), dx=WGS_DX, lam=WGS_LAM, z=WGS_Z, steps=steps,
                   batch=16, lr=1e-3, lr_final=1e-4, log_every=max(1, steps // 4))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    _, irr, roi, tgt, ph = wgs_inputs(n_designs)
    d_irr, d_roi, d_tgt = f32(irr), f32(roi), f32(tgt)

    def step():
        ph0 = model.forward(d_irr, d_roi)
        d = batch.design_batch(ctx, d_ill, d_tgt, ph0, nx=n, ny=n, dx=WGS_DX, lam=WGS_LAM, z=WGS_Z,
                               iterations=WGS_ITERS, roi=d_roi, rmse_goal=goal)
        m = batch.screen_metrics_batch(ctx, d["amplitude"], d_irr, d_ill, nx=n, ny=n, sdx=WGS_DX, roi=d_roi)
        return d, m

    step()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    ph0 = model.forward(d_irr, d_roi)
    e1.record()
    d = batch.design_batch(ctx, d_ill, d_tgt, ph0, nx=n, ny=n, dx=WGS_DX, lam=WGS_LAM, z=WGS_Z,
                           iterations=WGS_ITERS, roi=d_roi, rmse_goal=goal)
    m = batch.screen_metrics_batch(ctx, d["amplitude"], d_irr, d_ill, nx=n, ny=n, sdx=WGS_DX, roi=d_roi)
    e2.record()
    e2.synchronize()
    t_inf, t_all = e0.elapsed_time(e1), e0.elapsed_time(e2)
    rm = m[:, 0].cpu().numpy()
    used = d["iterations_used"].cpu().numpy()
    reached = int(np.sum(rm <= goal))
    model.close()
    return {"designs_per_s": reached / (t_all / 1e3), "reached": reached, "ms_per_step": t_all,
            "inference_ms": t_inf, "iterations_used": {"median": float(np.median(used)), "max": int(used.max())},
            "network": "U-Net 4 levels 32-256 ch, 2.15M params, BF16 (own kernels), 18.2 GFLOP per 256^2 design",
            "training": {"steps": steps, "batch": 16, "seconds": t_train, "setup_seconds": t1 - t0,
                         "loss": "intensity loss through the design propagation (doe_phase_loss_grad)",
                         "loss_history": hist}}


# ----------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-fields", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="sweep",
                    choices=["sweep", "wgs256", "multiplane2048", "farfield_uneven", "widened_rows"])
    ap.add_argument("--designs", type=int, default=1024, help="designs per step of the WGS workload")
    ap.add_argument("--no-wgs", action="store_true", help="skip the WGS block of the default line")
    ap.add_argument("--no-extras", action="store_true",
                    help="default line without the WGS, uneven far-field and multi-plane keys")
    ap.add_argument("--surrogate-steps", type=int, default=1500,
                    help="training steps of the warm-start surrogate in the wgs256 workload (0: skip the warm arm)")
    ap.add_argument("--pin-tuning", default=None,
                    help="profiling runs: skip the autotuner (its timings are distorted under a profiler) and set "
                         "these variants instead, e.g. fft_row=3,fft_col=0,sweep_row=3,sweep_col=4,sweep_fused=1,"
                         "sweep_group=64 (the choices the tuner makes on B200)")
    ap.add_argument("--no-design-tune", action="store_true",
                    help="skip doe_autotune_design before the design workloads (default shapes)")
    ap.add_argument("--fields", type=int, default=NFIELDS,
                    help="fields per step (profiling runs use fewer; the benchmark uses 64)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "b200" else args.warmup
    DESIGN_TUNE[0] = not args.no_design_tune

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)

    import diffractiveopticalelement_b200 as E
    ctx = E.Context(local)
    L = ctx.lib
    if args.workload == "wgs256":
        return main_wgs(args, ctx, device, rank, world, local)
    if args.workload == "multiplane2048":
        return main_multiplane(args, ctx, device, rank, world, local)
    if args.workload == "farfield_uneven":
        return main_uneven(args, ctx, device, rank, world, local)
    if args.workload == "widened_rows":
        for item in (args.pin_tuning.split(",") if args.pin_tuning else []):
            key, val = item.split("=")
            ctx.check(L.doe_ctx_set_tuning(ctx.h, key.encode(), int(val)))
        if rank == 0:
            print(json.dumps({"workload": "widened_rows", **measure_widened(ctx, not args.no_cpu_baseline)}),
                  flush=True)
        ctx.close()
        return 0

    params = workload_params(seed=2024 + rank)[:max(1, min(args.fields, NFIELDS))]
    nfields = len(params)
    fields = synth_fields(params, device)
    out = torch.empty((nfields * NZ, NY, NX), dtype=torch.complex64, device=device)
    lam = np.array([p["lam"] for p in params], dtype=np.float64)
    zs = np.array([z for p in params for z in p["z"]], dtype=np.float64)
    dp = C.POINTER(C.c_double)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)

    def step():
        ctx.check(L.doe_asm_sweep_dev(ctx.h, fields.data_ptr(), nfields, NX, NY, DX, DX, lam.ctypes.data_as(dp),
                                      zs.ctypes.data_as(dp), NZ, 1, 1, 0.02, out.data_ptr()))

    # shape autotuning for this grid and geometry (untimed set-up)
    L.doe_autotune.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                               C.POINTER(C.c_int)]
    chosen = (C.c_int * 5)()
    if args.pin_tuning:
        lg = int(math.log2(NX))
        slots = {"fft_row": 0, "fft_col": 1, "sweep_row": 2, "sweep_col": 3}
        for item in args.pin_tuning.split(","):
            key, val = item.split("=")
            val = int(val)
            if key in slots:
                ctx.check(L.doe_ctx_set_tuning(ctx.h, key.encode(), (lg << 8) | val))
                chosen[slots[key]] = val
            else:
                ctx.check(L.doe_ctx_set_tuning(ctx.h, key.encode(), val))
                if key == "sweep_group":
                    chosen[4] = val
    else:
        ctx.check(L.doe_autotune(ctx.h, NX, NY, DX, DX, 532e-9, 0.03, chosen))
    fused = C.c_longlong(0)
    ctx.check(L.doe_ctx_get_tuning(ctx.h, b"sweep_fused", C.byref(fused)))
    graph, hsym, tc = C.c_longlong(0), C.c_longlong(0), C.c_longlong(0)
    ctx.check(L.doe_ctx_get_tuning(ctx.h, b"sweep_graph", C.byref(graph)))
    ctx.check(L.doe_ctx_get_tuning(ctx.h, b"sweep_hsym", C.byref(hsym)))
    ctx.check(L.doe_ctx_get_tuning(ctx.h, b"sweep_tc", C.byref(tc)))
    res = C.c_longlong(1)
    ctx.check(L.doe_ctx_get_tuning(ctx.h, b"sweep_res", C.byref(res)))
    tuned = {"fft_row": chosen[0], "fft_col": chosen[1], "sweep_row": chosen[2], "sweep_col": chosen[3],
             "sweep_group": chosen[4], "sweep_fused_load": int(fused.value), "sweep_mirror_h": int(hsym.value),
             "sweep_tensor_core": int(tc.value), "sweep_graph": int(graph.value),
             "sweep_resident_planes": int(res.value)}
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        step()
    ctx.synchronize()

    # ---- timed region
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = L.doe_ctx_launch_count(ctx.h)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = int(L.doe_ctx_launch_count(ctx.h) - n0)
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    props = nfields * NZ * args.steps * world
    value = props / (ms / 1000.0)

    # ---- per-kernel durations: one instrumented step right after the timed region,
    # with the two passes serialised on one stream so that each launch is timed alone
    L.doe_ctx_set_profiling(ctx.h, 1)
    step()
    prof = profile_read(E, ctx)
    L.doe_ctx_set_profiling(ctx.h, 0)
    peak, peak_kind = peaks()
    roofline = None
    sweep_kernels = {k: v for k, v in prof.items() if k in SWEEP_PASSES}
    if sweep_kernels:
        name, (tot_ms, cnt) = max(sweep_kernels.items(), key=lambda kv: kv[1][0])
        planes_per_launch = nfields * NZ / cnt
        # column pass: the spectrum once per launch + every intermediate plane written
        # (8 B/px each); row pass: read intermediate + write output (16 B/px per plane)
        if SWEEP_PASSES[name] == "column":
            bytes_per_launch = (planes_per_launch + 1) * NX * NY * 8
        else:
            bytes_per_launch = planes_per_launch * NX * NY * 16
        avg_s = tot_ms / cnt / 1000.0
        achieved = bytes_per_launch / avg_s / 1e9
        traffic = recorded_traffic(name, planes_per_launch)
        roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                    "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the same kernel at "
                                       "full size, per plane, scaled to this launch's planes "
                                       f"(profiles/{TRAFFIC_RECORD})") if traffic else None,
                    "bytes_per_launch": bytes_per_launch, "avg_launch_us": avg_s * 1e6, "launches": cnt,
                    "per_kernel_ms": {k: round(v[0], 4) for k, v in prof.items()},
                    "per_kernel_note": "instrumented step with both passes on one stream (each launch timed alone)"}
        sweep_bytes = nfields * NZ * NX * NY * BYTES_PER_PX
        roofline["sweep_frac"] = (sweep_bytes / (ms / 1000.0 / args.steps) / 1e9) / peak

    # ---- e2e through the reference-facing host-buffer call (focusSweep, FP64 planes)
    e2e = None
    if rank == 0 and not args.no_e2e:
        nf = max(1, min(args.e2e_fields, nfields))
        n = NX * NY
        hin = C.c_void_p()
        hout = C.c_void_p()
        ctx.check(L.doe_host_alloc(ctx.h, C.byref(hin), 2 * n * 8 * nf))
        ctx.check(L.doe_host_alloc(ctx.h, C.byref(hout), 2 * n * NZ * 8))
        hin_a = np.ctypeslib.as_array((C.c_double * (2 * n * nf)).from_address(hin.value))
        hout_a = np.ctypeslib.as_array((C.c_double * (2 * n * NZ)).from_address(hout.value))
        src = fields[:nf].cpu().numpy().astype(np.complex128).reshape(nf, -1)
        for f in range(nf):
            hin_a[2 * n * f:2 * n * f + n] = src[f].real
            hin_a[2 * n * f + n:2 * n * (f + 1)] = src[f].imag
        reps = max(1, min(args.steps, 3))

        def e2e_step():
            for f in range(nf):
                base = hin.value + 2 * n * 8 * f
                ctx.check(L.doe_asm_sweep(ctx.h, C.cast(base, dp), C.cast(base + n * 8, dp), NX, NY, DX, DX,
                                          float(lam[f]), zs[f * NZ:(f + 1) * NZ].ctypes.data_as(dp), NZ, 1, 1,
                                          0.02, C.cast(hout.value, dp), C.cast(hout.value + n * NZ * 8, dp)))
        e2e_step()
        t0 = time.perf_counter()
        for _ in range(reps):
            e2e_step()
        dt = (time.perf_counter() - t0) / reps
        e2e = {"value": nf * NZ / dt, "unit": "props/s", "h2d_bytes_per_step": nf * 2 * n * 8,
               "d2h_bytes_per_step": nf * NZ * 2 * n * 8,
               "sample": f"{nf} fields x {NZ} distances per step through doe_asm_sweep "
                         f"(FP64 split planes in pinned host memory, copies inside the timed region)"}
        _ = hout_a
        L.doe_host_free(ctx.h, hin)
        L.doe_host_free(ctx.h, hout)

    # ---- CPU baseline (oracle port on this box's host cores)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        host_fields = fields[:4].cpu().numpy()
        nplanes = threads * 2
        t = cpu_sample(params, host_fields, nplanes, threads)
        t1 = cpu_sample(params, host_fields, 2, 1)
        cpu = {"value": nplanes / t, "unit": "props/s", "cores": threads, "kind": "port",
               "sample": f"{nplanes} band-limited 1024^2 propagations of the workload (fields 0-3) on {threads} "
                         f"threads, FP64 C restatement of propagateAngularSpectrum (no JS runtime on this box)",
               "single_core": {"value": 2 / t1, "cores": 1,
                               "sample": "2 propagations of the workload on one thread (the reference is "
                                         "single-threaded JavaScript)"}}

    # ---- the other configurations, as keys of the same line (one GPU only)
    extras = {}
    if world == 1 and not args.no_extras:
        del out
        out = None
        torch.cuda.empty_cache()
        cpu_on = not args.no_cpu_baseline
        if not args.no_wgs:
            extras["wgs256"] = measure_wgs(ctx, device, 512, 1, 2, args.surrogate_steps, cpu_on)
        torch.cuda.empty_cache()
        extras["farfield_uneven"] = measure_uneven(ctx, device, 1, 2, cpu_on)
        torch.cuda.empty_cache()
        extras["multiplane2048"] = measure_multiplane(ctx, device, 1, 2, cpu_on, False)
        torch.cuda.empty_cache()
        extras["widened_rows"] = measure_widened(ctx, cpu_on)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "props/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c64 (fp32), fp64 phase reduction",
                "data": "synthetic", "config": dict(CONFIG, fields=nfields, tuned_variants=tuned), "clocks": clocks, "roofline": roofline,
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, **extras}
        print(json.dumps(line), flush=True)
    del out, fields
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
