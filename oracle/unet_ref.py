"""CPU restatement of the learned warm start's network (test infrastructure:
the checker of the CUDA forward and backward passes, never part of the
product path).

The same U-Net as bevy_eulerian_fluid_b200/csrc/efl_unet.cuh (an extension
with no reference counterpart): NHWC activations rounded to bf16 wherever the
CUDA kernels store bf16 (round to nearest even), weights rounded to bf16,
products and sums in float64 here (fp32 accumulation on the GPU), ReLU, 2x2
average pooling, nearest upsampling, concatenation [upsampled, skip].  The
parameter vector is the C layout: for every convolution, weights
[tap][cout][cin] (tap = (dy + 1) * 3 + (dx + 1)) then biases [cout].
"""
from __future__ import annotations

import numpy as np

# (cin, cout, relu) of the 15 convolutions, in parameter order.
SPEC = [(16, 16, 1), (16, 16, 1), (16, 32, 1), (32, 32, 1), (32, 64, 1), (64, 64, 1), (64, 64, 1), (64, 64, 1),
        (128, 64, 1), (64, 64, 1), (96, 32, 1), (32, 32, 1), (48, 16, 1), (16, 16, 1), (16, 16, 0)]


def num_params() -> int:
    return sum(9 * ci * co + co for ci, co, _ in SPEC)


def bf16(a) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(a, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray, rounding=True):
    out, off = [], 0
    for ci, co, relu in SPEC:
        w = params[off:off + 9 * ci * co].reshape(9, co, ci)
        off += 9 * ci * co
        b = params[off:off + co]
        off += co
        out.append((bf16(w) if rounding else w.astype(np.float64), b.astype(np.float64), relu))
    return out


def _shift(x, dy, dx):
    """s[y, x] = x[y + dy, x + dx] with zeros outside."""
    H, W = x.shape[:2]
    s = np.zeros_like(x)
    ys, yd = slice(max(0, -dy), H - max(0, dy)), slice(max(0, dy), H - max(0, -dy))
    xs, xd = slice(max(0, -dx), W - max(0, dx)), slice(max(0, dx), W - max(0, -dx))
    s[ys, xs] = x[yd, xd]
    return s


def conv(x, w, b):
    H, W, _ = x.shape
    y = np.zeros((H, W, w.shape[1]), np.float64)
    for t in range(9):
        y += _shift(x, t // 3 - 1, t % 3 - 1).astype(np.float64) @ w[t].T.astype(np.float64)
    return y + b


def conv_dx(g, w):
    H, W, _ = g.shape
    d = np.zeros((H, W, w.shape[2]), np.float64)
    for t in range(9):
        d += _shift(g, -(t // 3 - 1), -(t % 3 - 1)).astype(np.float64) @ w[t].astype(np.float64)
    return d


def conv_dw(x, g):
    H, W, ci = x.shape
    co = g.shape[2]
    gw = np.zeros((9, co, ci))
    g2 = g.reshape(-1, co).astype(np.float64)
    for t in range(9):
        gw[t] = g2.T @ _shift(x, t // 3 - 1, t % 3 - 1).reshape(-1, ci).astype(np.float64)
    return gw, g2.sum(0)


def pool(x):
    return 0.25 * (((x[0::2, 0::2] + x[0::2, 1::2]) + x[1::2, 0::2]) + x[1::2, 1::2])


def up(x):
    return np.repeat(np.repeat(x, 2, axis=0), 2, axis=1)


def pool_bwd(g):
    return 0.25 * up(g)


def up_bwd(g):
    return ((g[0::2, 0::2] + g[0::2, 1::2]) + g[1::2, 0::2]) + g[1::2, 1::2]


class Net:
    """Forward with the activations kept, backward of the masked MSE."""

    def __init__(self, params: np.ndarray, rounding: bool = True):
        self.L = unpack(np.asarray(params, np.float32 if rounding else np.float64), rounding)
        self.r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))

    def _c(self, i, x):
        w, b, relu = self.L[i]
        y = conv(x, w, b)
        if relu:
            y = np.maximum(y, 0.0)
            return self.r(y)
        return y

    def forward(self, feats):
        r, c = self.r, self._c
        a = {}
        a["X0"] = r(feats)
        a["t0"] = c(0, a["X0"])
        a["s0"] = c(1, a["t0"])
        a["p1"] = r(pool(a["s0"]))
        a["t1"] = c(2, a["p1"])
        a["s1"] = c(3, a["t1"])
        a["p2"] = r(pool(a["s1"]))
        a["t2"] = c(4, a["p2"])
        a["s2"] = c(5, a["t2"])
        a["p3"] = r(pool(a["s2"]))
        a["t3"] = c(6, a["p3"])
        a["u3"] = c(7, a["t3"])
        a["cat2"] = np.concatenate([up(a["u3"]), a["s2"]], axis=2)
        a["t4"] = c(8, a["cat2"])
        a["u4"] = c(9, a["t4"])
        a["cat1"] = np.concatenate([up(a["u4"]), a["s1"]], axis=2)
        a["t5"] = c(10, a["cat1"])
        a["u5"] = c(11, a["t5"])
        a["cat0"] = np.concatenate([up(a["u5"]), a["s0"]], axis=2)
        a["t6"] = c(12, a["cat0"])
        a["u6"] = c(13, a["t6"])
        a["out"] = c(14, a["u6"])
        self.a = a
        return a["out"][:, :, 0]

    def backward(self, target, mask):
        """Relative squared error of output channel 0 over the mask,
        sum (pred - t)^2 / sum t^2; returns (loss, gradient vector)."""
        a, r = self.a, self.r
        m = mask.astype(bool)
        t2 = float((np.asarray(target, np.float64)[m] ** 2).sum())
        inv = 1.0 / t2 if t2 > 0 else 0.0
        d = a["out"][:, :, 0] - target
        loss = float((d[m] ** 2).sum() * inv)
        g = np.zeros_like(a["out"])
        g[:, :, 0] = np.where(m, 2.0 * d * inv, 0.0)
        grads = [None] * len(SPEC)

        def cb(i, x, y, g, need_dx=True):
            w, _, relu = self.L[i]
            dy = r(np.where(y > 0, g, 0.0) if relu else g)
            gw, gb = conv_dw(x, dy)
            grads[i] = (gw, gb)
            return conv_dx(dy, w) if need_dx else None

        g_u6 = cb(14, a["u6"], a["out"], g)
        g_t6 = cb(13, a["t6"], a["u6"], g_u6)
        g_cat0 = cb(12, a["cat0"], a["t6"], g_t6)
        g_u5 = up_bwd(g_cat0[:, :, :32])
        g_t5 = cb(11, a["t5"], a["u5"], g_u5)
        g_cat1 = cb(10, a["cat1"], a["t5"], g_t5)
        g_u4 = up_bwd(g_cat1[:, :, :64])
        g_t4 = cb(9, a["t4"], a["u4"], g_u4)
        g_cat2 = cb(8, a["cat2"], a["t4"], g_t4)
        g_u3 = up_bwd(g_cat2[:, :, :64])
        g_t3 = cb(7, a["t3"], a["u3"], g_u3)
        g_p3 = cb(6, a["p3"], a["t3"], g_t3)
        g_s2 = g_cat2[:, :, 64:] + pool_bwd(g_p3)
        g_t2 = cb(5, a["t2"], a["s2"], g_s2)
        g_p2 = cb(4, a["p2"], a["t2"], g_t2)
        g_s1 = g_cat1[:, :, 64:] + pool_bwd(g_p2)
        g_t1 = cb(3, a["t1"], a["s1"], g_s1)
        g_p1 = cb(2, a["p1"], a["t1"], g_t1)
        g_s0 = g_cat0[:, :, 32:] + pool_bwd(g_p1)
        g_t0 = cb(1, a["t0"], a["s0"], g_s0)
        cb(0, a["X0"], a["t0"], g_t0, need_dx=False)
        vec = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
        return loss, vec
