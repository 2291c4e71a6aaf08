"""The surrogate's CPU oracle pinned against central finite differences (FP64)."""
import numpy as np

from oracle import unet_oracle as U


def test_layout_matches_engine_parameter_count():
    # 4 levels, 32-256 channels: the configuration of the warm-start workload
    assert U.param_count(32, 4) == 2_149_026
    assert [s for s in U.layer_shapes(32, 3)] == [(32, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128),
                                                  (128, 64), (128, 64), (64, 64), (64, 32), (64, 32), (32, 32)]


def test_backward_matches_finite_differences():
    n, base, L, B = 16, 32, 3, 2
    p = U.he_init(base, L, seed=3).astype(np.float64)
    rng = np.random.default_rng(5)
    irr = rng.random((B, n * n))
    roi = (rng.random((B, n * n)) > 0.3).astype(np.float64)
    dphase = rng.standard_normal((B, n * n))
    net = U.UNet(p, n, base, L, emu=False)
    net.forward(irr, roi)
    g = net.backward(dphase)
    idx = rng.choice(p.size, 40, replace=False)
    # include head and first / last conv layers explicitly
    idx = np.concatenate([idx, [0, 5, p.size - 1, p.size - 3, p.size - 2 * base - 10]])
    eps = 1e-6
    worst = 0.0
    for i in idx:
        q = p.copy()
        q[i] += eps
        fp = np.sum(dphase * U.UNet(q, n, base, L, emu=False).forward(irr, roi))
        q[i] -= 2 * eps
        fm = np.sum(dphase * U.UNet(q, n, base, L, emu=False).forward(irr, roi))
        fd = (fp - fm) / (2 * eps)
        worst = max(worst, abs(fd - g[i]) / max(1e-3, abs(fd), abs(g[i])))
    assert worst < 1e-4, worst


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 3.14159265])
    r = U.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 + 2 ** -7 or r[1] == 1.0  # tie -> even
    assert r[2] == 1.0 + 2 ** -7
    assert r[3] == -2.5 and r[4] == 0.0
    assert abs(r[5] - 3.140625) < 1e-12


def test_phase_loss_restatement_matches_finite_differences(oracle):
    """The FP64 physics-loss gradient used to check the GPU, against central differences."""
    import importlib.util, os
    spec = importlib.util.spec_from_file_location("tgs", os.path.join(os.path.dirname(__file__),
                                                                      "test_gpu_surrogate.py"))
    tgs = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(tgs)
    n = 16
    rng = np.random.default_rng(2)
    ill = oracle.disc_mask(n, n, tgs.DX, tgs.DX, 0.45 * n * tgs.DX, 2 * tgs.DX)
    tg = oracle.prepare_target((rng.random(n * n) > 0.6).astype(float), ill)
    ro = (rng.random(n * n) > 0.3).astype(float)
    ph = rng.uniform(-np.pi, np.pi, n * n)
    L, g = tgs.phase_loss_fp64(oracle, ph, ill, tg, ro, n)
    for i in rng.choice(n * n, 12, replace=False):
        q = ph.copy()
        q[i] += 1e-6
        Lp, _ = tgs.phase_loss_fp64(oracle, q, ill, tg, ro, n)
        q[i] -= 2e-6
        Lm, _ = tgs.phase_loss_fp64(oracle, q, ill, tg, ro, n)
        fd = (Lp - Lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-8, (i, fd, g[i])
