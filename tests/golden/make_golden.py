"""Regenerate the golden fixtures of tests/golden/ from the FP64 oracle.

Test infrastructure: the fixtures pin the oracle (the CPU restatement of the
reference's algorithms in oracle/) against silent regressions and give the GPU
parity tests committed vectors to compare with. Inputs are seeded (numpy
default_rng, the reference's xorshift32 for phases) and small (n <= 64) so the
whole set stays a few hundred KB. Each case is one .npz with its inputs and
outputs; golden.json records the SHA-256 of every file.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402

LAM = 532e-9


def cplx(rng, n):
    return rng.standard_normal(n) - 0.1, rng.standard_normal(n) + 0.2


def disc(n, r):
    i = np.arange(n)
    X, Y = np.meshgrid(i, i)
    return (np.hypot(X - n / 2, Y - n / 2) <= r).astype(np.float64).ravel()


def cases():
    rng = np.random.default_rng(20240601)
    out = {}
    # fft2d forward / inverse on a ragged (non-square) grid
    re, im = cplx(rng, 16 * 8)
    fr, fi = O.fft2d(re, im, 16, 8, False)
    ir, ii = O.fft2d(re, im, 16, 8, True)
    out["fft2d_16x8"] = dict(re=re, im=im, fwd_re=fr, fwd_im=fi, inv_re=ir, inv_im=ii)
    # angular spectrum, band limited and not, forward and back
    re, im = cplx(rng, 32 * 32)
    a1 = O.asm(re, im, 32, 32, 8e-6, 8e-6, LAM, 0.03, True, True, 0.02)
    a2 = O.asm(re, im, 32, 32, 8e-6, 8e-6, LAM, -0.021, False, True, 0.02)
    out["asm_32"] = dict(re=re, im=im, bl_re=a1[0], bl_im=a1[1], back_re=a2[0], back_im=a2[1],
                         params=np.array([8e-6, LAM, 0.03, -0.021]))
    # lens focal plane and single-FFT Fresnel
    re, im = cplx(rng, 32 * 32)
    fo = O.focal_plane(re, im, 32, 32, 8e-6, 8e-6, LAM, 0.05)
    fz = O.fresnel(re, im, 32, 32, 8e-6, 8e-6, LAM, 0.2)
    out["lens_fresnel_32"] = dict(re=re, im=im, lens_re=fo[0], lens_im=fo[1], lens_d=np.array(fo[2:4]),
                                  fres_re=fz[0], fres_im=fz[1], fres_d=np.array(fz[2:4]))
    # design loops at 32^2
    n = 32
    ill = O.disc_mask(n, n, 8e-6, 8e-6, 0.45 * n * 8e-6, 2 * 8e-6)
    tgt = O.prepare_target(disc(n, 0.3 * n), ill)
    roi = O.auto_roi(disc(n, 0.3 * n), n, n)
    ip = O.random_phase(n, n, 7)
    for alg in ("gs", "wgs", "fourier"):
        r = O.design(alg, ill, tgt, nx=n, ny=n, dx=8e-6, lam=LAM, z=0.03, iterations=5, init_phase=ip, roi=roi)
        case = dict(ill=ill, tgt=tgt, roi=roi, init_phase=ip, phase=r["phase"], amplitude=r["amplitude"],
                    error=r["error"], efficiency=r["efficiency"])
        if "weights" in r:
            case["weights"] = r["weights"]
            case["rmse"] = np.array([r["rmse"]])
        out[f"design_{alg}_32"] = case
    # multi-plane, two planes
    t1 = O.prepare_target(disc(n, 0.2 * n), ill)
    t2 = O.prepare_target(disc(n, 0.35 * n), ill)
    mp = O.multiplane(ill, [0.025, 0.035], [t1, t2], None, [1.0, 0.5], nx=n, ny=n, dx=8e-6, iterations=3,
                      init_phase=ip)
    out["multiplane_32"] = dict(ill=ill, t1=t1, t2=t2, init_phase=ip, phase=mp["phase"], error=mp["error"],
                                per_plane=mp["perPlaneError"])
    # full screen metrics of a propagated design field
    fre, fim = O.asm(ill * np.cos(ip), ill * np.sin(ip), n, n, 8e-6, 8e-6, LAM, 0.03, False, True, 0.02)
    irr = disc(n, 0.3 * n)
    m = O.screen_metrics_full(fre, fim, n, n, 8e-6, 8e-6, irr, roi, ill, ip, 8e-6, 8e-6, grid={"cols": 4, "rows": 4})
    out["screen_metrics_32"] = dict(fre=fre, fim=fim, irr=irr, roi=roi, ill=ill, phase=ip,
                                    metrics=np.array([m[k] for k in O.FULL_METRIC_KEYS]))
    # error diffusion quantiser (serpentine and raster)
    phi = rng.uniform(-4, 4, 32 * 32)
    out["error_diffusion_32"] = dict(phi=phi, snake=O.error_diffusion(phi, 4, True, True),
                                     raster=O.error_diffusion(phi, 3, False, True))
    # hologram record / reconstruct and partial coherence
    ore, oim = np.abs(rng.standard_normal(32 * 32)), 0.1 * rng.standard_normal(32 * 32)
    x = np.tile((np.arange(32) - 16) * 8e-6, 32)
    k = 2 * np.pi / LAM * (LAM * 4 / (32 * 8e-6))
    rre, rim = np.cos(k * x), np.sin(k * x)
    h = O.record_hologram(ore, oim, rre, rim, "phase", 4)
    rc = O.reconstruct_hologram(h["plate_re"], h["plate_im"], rre, rim, 32, 32, 8e-6, 8e-6, LAM, 0.004)
    pre, pim = O.partially_coherent_modes(16, 16, 8e-6, 8e-6, modes=3, sigma=24e-6, waist=50e-6, seed=5)
    mi = O.modal_intensity(pre, pim, 256, np.array([1.0, 0.5, 2.0]))
    out["interference_32"] = dict(obj_re=ore, obj_im=oim, ref_re=rre, ref_im=rim, plate_re=h["plate_re"],
                                  plate_im=h["plate_im"], recorded=h["recorded"], real_re=rc["real_re"],
                                  real_im=rc["real_im"], virt_re=rc["virt_re"], virt_im=rc["virt_im"],
                                  modes_re=pre, modes_im=pim, modal=mi)
    return out


def main():
    O.build()
    manifest = {}
    for name, arrays in cases().items():
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in arrays.items()})
        with open(path, "rb") as f:
            manifest[name + ".npz"] = hashlib.sha256(f.read()).hexdigest()
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(f"{len(manifest)} fixtures written")


if __name__ == "__main__":
    main()
