"""CPU restatement of the warm-start U-Net (numpy, FP64) with forward and backward.

TEST INFRASTRUCTURE ONLY: the checker of libunet3d.so (tests/).  The reference
(LBM3D_BB) has no learned component, so there is nothing of it to pin; this file is
pinned instead by finite differences of its own loss (tests/test_unet_oracle.py)
and follows the layer order of lbm3d_bb_b200/unet.py.

With ``bf16=True`` every stored activation, gradient and working weight is rounded
to BF16 (round to nearest even) where the GPU stores it, so the GPU result can be
compared to rounding level; accumulation stays FP64.
"""
from __future__ import annotations

import numpy as np

IN_CH, OUT_CH, N_TARGET = 16, 16, 4
OFFS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]  # tap order


def to_bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even); returns FP64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return (u.astype(np.uint32).view(np.float32)).astype(np.float64)


def shift(x: np.ndarray, off) -> np.ndarray:
    """s[v] = x[v + off] (zero outside), x of shape (n, d, h, w, c)."""
    dz, dy, dx = off
    s = np.zeros_like(x)
    n, d, h, w, _ = x.shape

    def rng(k, size):
        return (slice(max(0, -k), size - max(0, k)), slice(max(0, k), size - max(0, -k)))

    (zo, zi), (yo, yi), (xo, xi) = rng(dz, d), rng(dy, h), rng(dx, w)
    s[:, zo, yo, xo] = x[:, zi, yi, xi]
    return s


def conv(x, w, b):
    y = np.zeros(x.shape[:4] + (w.shape[1],))
    for t, off in enumerate(OFFS):
        y += shift(x, off) @ w[t].T
    return y + (0.0 if b is None else b)


def conv_bwd(x, w, dy):
    """(dx, dw, db) of y = conv(x, w, b)."""
    dx = np.zeros_like(x)
    dw = np.zeros_like(w)
    flat = dy.reshape(-1, dy.shape[-1])
    for t, off in enumerate(OFFS):
        dx += shift(dy @ w[t], tuple(-o for o in off))
        dw[t] = flat.T @ shift(x, off).reshape(-1, x.shape[-1])
    return dx, dw, flat.sum(axis=0)


def pool(x):
    n, d, h, w, c = x.shape
    return x.reshape(n, d // 2, 2, h // 2, 2, w // 2, 2, c).mean(axis=(2, 4, 6))


def pool_bwd(dy):
    return np.repeat(np.repeat(np.repeat(dy, 2, 1), 2, 2), 2, 3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 1), 2, 2), 2, 3)


def up_bwd(dy):
    n, d, h, w, c = dy.shape
    return dy.reshape(n, d // 2, 2, h // 2, 2, w // 2, 2, c).sum(axis=(2, 4, 6))


LAYERS = ["e1a", "e1b", "e2a", "e2b", "e3a", "e3b", "d2a", "d2b", "d1a", "d1b", "head"]


class UNetRef:
    def __init__(self, params: dict, width: int = 16, bf16: bool = True):
        self.p = {k: np.asarray(v, np.float64) for k, v in params.items()}
        self.w = width
        self.bf = bf16
        self.r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
        self.wb = {n: self.r(self.p[f"{n}.w"]) for n in LAYERS}

    def _c(self, name, x, relu=True):
        y = conv(x, self.wb[name], self.p[f"{name}.b"])
        return self.r(np.maximum(y, 0.0) if relu else y)

    def forward(self, x):
        r, A = self.r, {}
        A["x"] = r(x)
        A["a1"] = self._c("e1a", A["x"])
        A["s1"] = self._c("e1b", A["a1"])
        A["p1"] = r(pool(A["s1"]))
        A["a2"] = self._c("e2a", A["p1"])
        A["s2"] = self._c("e2b", A["a2"])
        A["p2"] = r(pool(A["s2"]))
        A["a3"] = self._c("e3a", A["p2"])
        A["b3"] = self._c("e3b", A["a3"])
        A["c2"] = np.concatenate([up(A["b3"]), A["s2"]], axis=-1)
        A["a4"] = self._c("d2a", A["c2"])
        A["a5"] = self._c("d2b", A["a4"])
        A["c1"] = np.concatenate([up(A["a5"]), A["s1"]], axis=-1)
        A["a6"] = self._c("d1a", A["c1"])
        A["a7"] = self._c("d1b", A["a6"])
        A["out"] = self._c("head", A["a7"], relu=False)
        self.A = A
        return A["out"]

    def loss(self, target, mask, cw, count):
        """Masked weighted MSE and its output gradient (rounded like the GPU's)."""
        o = self.A["out"][..., :N_TARGET]
        m = (mask != 0)[..., None]
        d = (o - target) * m
        loss = float(np.sum(cw * d * d) / count)
        g = np.zeros_like(self.A["out"])
        g[..., :N_TARGET] = 2.0 * cw * d / count
        return loss, self.r(g)

    def backward(self, dout):
        A, r, G = self.A, self.r, {}

        def back(name, x, g, y=None):
            if y is not None:
                g = g * (y > 0)
            dx, dw, db = conv_bwd(x, self.wb[name], g)
            G[f"{name}.w"], G[f"{name}.b"] = dw, db
            return r(dx)

        w = self.w
        d = back("head", A["a7"], dout)
        d = back("d1b", A["a6"], d, A["a7"])
        dc1 = back("d1a", A["c1"], d, A["a6"])
        d_a5 = r(up_bwd(dc1[..., : 2 * w]))
        d_s1 = dc1[..., 2 * w:]
        d = back("d2b", A["a4"], d_a5, A["a5"])
        dc2 = back("d2a", A["c2"], d, A["a4"])
        d_b3 = r(up_bwd(dc2[..., : 4 * w]))
        d_s2 = dc2[..., 4 * w:]
        d = back("e3b", A["a3"], d_b3, A["b3"])
        d_p2 = back("e3a", A["p2"], d, A["a3"])
        d_s2 = r(pool_bwd(d_p2) + d_s2)
        d = back("e2b", A["a2"], d_s2, A["s2"])
        d_p1 = back("e2a", A["p1"], d, A["a2"])
        d_s1 = r(pool_bwd(d_p1) + d_s1)
        d = back("e1b", A["a1"], d_s1, A["s1"])
        back("e1a", A["x"], d, A["a1"])
        return G
