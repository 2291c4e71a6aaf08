"""CPU oracle of the warm-start surrogate network (test infrastructure only).

The surrogate has no counterpart in the reference, so this restatement is the
oracle for its kernels: a NumPy FP64 forward and backward pass of the same U-Net
(parameter layout, graph and head as the engine's csrc/unet.cu). With emu=True it
rounds weights and stored activations / activation gradients to BF16 at the same
points as the GPU kernels, so the comparison isolates accumulation order; with
emu=False it is plain FP64 and is pinned against central finite differences.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + ((u >> 16) & 1) + 0x7FFF) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layer_shapes(base, levels):
    """(cin, cout) of every 3x3 convolution in parameter order, then the head."""
    ch = lambda l: base << l
    L = levels
    convs = []
    for l in range(L - 1):
        convs.append((base if l == 0 else ch(l - 1), ch(l)))
        convs.append((ch(l), ch(l)))
    convs.append((ch(L - 2), ch(L - 1)))
    convs.append((ch(L - 1), ch(L - 1)))
    for l in range(L - 2, -1, -1):
        convs += [(ch(l + 1), ch(l)), (2 * ch(l), ch(l)), (ch(l), ch(l))]
    return convs


def unpack(params, base, levels):
    """Flat FP32 parameter vector -> list of (W [co, 9, ci], b [co]) and the head (W [2, base], b [2])."""
    p = np.asarray(params, dtype=np.float64)
    out, o = [], 0
    for ci, co in layer_shapes(base, levels):
        W = p[o:o + co * 9 * ci].reshape(co, 9, ci)
        o += co * 9 * ci
        b = p[o:o + co]
        o += co
        out.append((W, b))
    hw = p[o:o + 2 * base].reshape(2, base)
    o += 2 * base
    hb = p[o:o + 2]
    o += 2
    assert o == p.size, (o, p.size)
    return out, (hw, hb)


def param_count(base, levels):
    return sum(co * 9 * ci + co for ci, co in layer_shapes(base, levels)) + 2 * base + 2


def _shift(xp, t, H, W):
    ky, kx = divmod(t, 3)
    return xp[:, ky:ky + H, kx:kx + W, :]


def conv3x3(x, W, b=None):
    """x [B, H, W, ci], W [co, 9, ci] -> [B, H, W, co] (pad 1)."""
    B, H, Wd, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((B, H, Wd, W.shape[0]))
    for t in range(9):
        out += _shift(xp, t, H, Wd) @ W[:, t, :].T
    if b is not None:
        out += b
    return out


def conv3x3_wgrad(x, g):
    """dW [co, 9, ci] = sum_p g[p, co] x[p + tap, ci]."""
    B, H, Wd, ci = x.shape
    co = g.shape[-1]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dW = np.zeros((co, 9, ci))
    g2 = g.reshape(-1, co)
    for t in range(9):
        dW[:, t, :] = g2.T @ _shift(xp, t, H, Wd).reshape(-1, ci)
    return dW, g2.sum(axis=0)


def flip_t(W):
    """Kernel of the input gradient: Wt[ci, t', co] = W[co, 8 - t', ci]."""
    return np.transpose(W[:, ::-1, :], (2, 1, 0))


def pool(x):
    B, H, W, C = x.shape
    return 0.25 * x.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def up_bwd(g):
    B, H, W, C = g.shape
    return g.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


class UNet:
    def __init__(self, params, n, base=32, levels=4, emu=True):
        self.n, self.base, self.L, self.emu = n, base, levels, emu
        self.convs, self.head = unpack(params, base, levels)
        self.r = bf16 if emu else (lambda a: np.asarray(a, dtype=np.float64))
        self.Wq = [self.r(W) for W, _ in self.convs]

    def _conv(self, k, x):
        return self.r(np.maximum(conv3x3(x, self.Wq[k], self.convs[k][1]), 0.0))

    def forward(self, irr, roi=None):
        """irr, roi: [B, n*n] -> phase [B, n*n]."""
        r, n, base, L = self.r, self.n, self.base, self.L
        irr = np.asarray(irr, dtype=np.float64).reshape(-1, n, n)
        B = irr.shape[0]
        mx = irr.reshape(B, -1).max(axis=1)
        sc = np.where(mx > 0, 1.0 / np.where(mx > 0, mx, 1.0), 0.0)
        if self.emu:
            sc = np.float32(1.0) / np.where(mx > 0, mx, 1.0).astype(np.float32)
            sc = np.where(mx > 0, sc, 0.0).astype(np.float64)
            x0v = np.float32(irr) * sc[:, None, None].astype(np.float32)
        else:
            x0v = irr * sc[:, None, None]
        x0 = np.zeros((B, n, n, base))
        x0[..., 0] = r(x0v)
        x0[..., 1] = r(np.ones((B, n, n)) if roi is None else np.asarray(roi, dtype=np.float64).reshape(B, n, n))
        x0[..., 2] = 1.0
        S = {"x0": x0}
        k = 0
        x = x0
        for l in range(L - 1):
            a = self._conv(k, x)
            k += 1
            e = self._conv(k, a)
            k += 1
            S[f"in{l}"], S[f"a{l}"], S[f"e{l}"] = x, a, e
            x = r(pool(e))
        S[f"in{L - 1}"] = x
        b1 = self._conv(k, x)
        k += 1
        b2 = self._conv(k, b1)
        k += 1
        S["b1"], S["b2"] = b1, b2
        prev = b2
        for l in range(L - 2, -1, -1):
            u = up(prev)
            dup = self._conv(k, u)
            k += 1
            cat = np.concatenate([S[f"e{l}"], dup], axis=-1)
            da = self._conv(k, cat)
            k += 1
            d = self._conv(k, da)
            k += 1
            S[f"u{l}"], S[f"cat{l}"], S[f"da{l}"], S[f"d{l}"] = u, cat, da, d
            prev = d
        hw, hb = self.head
        d0 = S["d0"]
        c = d0 @ hw[0] + hb[0]
        s = d0 @ hw[1] + hb[1]
        S["c"], S["s"] = c, s
        self.S = S
        return np.arctan2(s, c).reshape(B, -1)

    def backward(self, dphase):
        """dL/dphase [B, n*n] of the last forward -> flat parameter gradient."""
        r, n, L, base = self.r, self.n, self.L, self.base
        S = self.S
        B = S["c"].shape[0]
        g = np.asarray(dphase, dtype=np.float64).reshape(B, n, n)
        c, s = S["c"], S["s"]
        r2 = c * c + s * s
        inv = np.where(r2 > 1e-20, 1.0 / np.where(r2 > 1e-20, r2, 1.0), 0.0)
        gc, gs = -s * inv * g, c * inv * g
        hw, _ = self.head
        d0 = S["d0"]
        dhw = np.stack([np.einsum("bhw,bhwk->k", gc, d0), np.einsum("bhw,bhwk->k", gs, d0)])
        dhb = np.array([gc.sum(), gs.sum()])
        gd = r((gc[..., None] * hw[0] + gs[..., None] * hw[1]) * (d0 > 0))
        nconv = len(self.convs)
        dW = [None] * nconv
        db = [None] * nconv
        # layer indices (creation order)
        enc = [(2 * l, 2 * l + 1) for l in range(L - 1)]
        kb = 2 * (L - 1)
        dec = {}
        k = kb + 2
        for l in range(L - 2, -1, -1):
            dec[l] = (k, k + 1, k + 2)
            k += 3

        def dgrad(kk, gout, mask):
            out = conv3x3(gout, r(flip_t(self.convs[kk][0])))
            if mask is not None:
                out = out * (mask > 0)
            return r(out)

        def wgrad(kk, x, gout):
            dW[kk], db[kk] = conv3x3_wgrad(x, gout)

        gprev = gd
        gcat = {}
        for l in range(L - 1):
            kup, ka, kbb = dec[l]
            C = base << l
            wgrad(kbb, S[f"da{l}"], gprev)
            gda = dgrad(kbb, gprev, S[f"da{l}"])
            wgrad(ka, S[f"cat{l}"], gda)
            gc_ = dgrad(ka, gda, S[f"cat{l}"])
            gcat[l] = gc_
            wgrad(kup, S[f"u{l}"], gc_[..., C:])
            gu = dgrad(kup, gc_[..., C:], None)
            pv = S[f"d{l + 1}"] if l + 1 <= L - 2 else S["b2"]
            gprev = r(up_bwd(gu) * (pv > 0))
        wgrad(kb + 1, S["b1"], gprev)
        gb1 = dgrad(kb + 1, gprev, S["b1"])
        wgrad(kb, S[f"in{L - 1}"], gb1)
        gin = dgrad(kb, gb1, None)
        for l in range(L - 2, -1, -1):
            ka, kbb = enc[l]
            C = base << l
            ge = r((gcat[l][..., :C] + 0.25 * up(gin)) * (S[f"e{l}"] > 0))
            wgrad(kbb, S[f"a{l}"], ge)
            ga = dgrad(kbb, ge, S[f"a{l}"])
            wgrad(ka, S[f"in{l}"], ga)
            if l > 0:
                gin = dgrad(ka, ga, None)
        flat = []
        for kk in range(nconv):
            flat += [dW[kk].ravel(), db[kk]]
        flat += [dhw.ravel(), dhb]
        return np.concatenate(flat)


def he_init(base, levels, seed=0):
    """Seeded FP32 parameter vector with He-normal weights (for CPU checks)."""
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co in layer_shapes(base, levels):
        parts += [rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci)), 0.01 * rng.standard_normal(co)]
    parts += [rng.standard_normal(2 * base) * np.sqrt(1.0 / base), np.zeros(2)]
    return np.concatenate(parts).astype(np.float32)
