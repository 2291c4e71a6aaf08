"""Small, fixed cases of single kernels for profiler captures (no reference
counterpart). Each case builds the benchmark's seeded inputs at a reduced batch and
runs the kernel of interest a few times, so that a profiler can capture one launch of
it on a few GB of device memory at most:

    python -m diffractiveopticalelement_b200.profile_cases cluster [designs] [iterations] [cluster]
        image-plane WGS on 256^2 designs, twice, through batch.design_batch on a context
        with tuning "design_cluster" set as given (1: the cluster-resident kernel)
    python -m diffractiveopticalelement_b200.profile_cases surrogate [designs] [surrogate_tc]
        two forward passes of the 4-level, 32-channel 256^2 surrogate, with tuning
        "surrogate_tc" as given (default: the context's)

Run from the repository root (the inputs come from bench.wgs_inputs).
"""
from __future__ import annotations

import os
import sys


def _f32(a):
    import numpy as np
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def cluster(designs: int = 74, iterations: int = 5, cl: int = 1) -> float:
    import bench
    from . import _lib, batch
    ill, irr, roi, tgt, ph = bench.wgs_inputs(designs)
    ctx = _lib.Context(0)
    ctx.check(ctx.lib.doe_ctx_set_tuning(ctx.h, b"design_cluster", cl))
    d_ill, d_tgt, d_roi, d_ph0 = _f32(ill), _f32(tgt), _f32(roi), _f32(ph)
    r = None
    for _ in range(2):
        d_ph = d_ph0.clone()
        r = batch.design_batch(ctx, d_ill, d_tgt, d_ph, nx=256, ny=256, dx=bench.WGS_DX, lam=bench.WGS_LAM,
                               z=bench.WGS_Z, iterations=iterations, roi=d_roi)
        ctx.synchronize()
    err = float(r["error"][:, -1].mean())
    ctx.close()
    return err


def surrogate(designs: int = 16, tc: int = -1) -> float:
    import bench
    from . import _lib
    from . import surrogate as S
    ill, irr, roi, tgt, ph = bench.wgs_inputs(designs)
    ctx = _lib.Context(0)
    if tc >= 0:
        ctx.check(ctx.lib.doe_ctx_set_tuning(ctx.h, b"surrogate_tc", tc))
    m = S.Surrogate(n=256, base=32, levels=4, max_batch=designs, seed=1, ctx=ctx)
    out = None
    for _ in range(2):
        out = m.forward(_f32(irr), _f32(roi))
    ctx.synchronize()
    val = float(out.abs().mean())
    m.close()
    ctx.close()
    return val


def main(argv) -> int:
    root = os.getcwd()
    if root not in sys.path:
        sys.path.insert(0, root)
    if not argv or argv[0] not in ("cluster", "surrogate"):
        print(__doc__)
        return 2
    args = [int(a) for a in argv[1:]]
    print("ok", (cluster if argv[0] == "cluster" else surrogate)(*args))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
