"""CPU oracle of the learned preconditioner's network (test infrastructure only: tests import it to
check the GPU kernels; the product never calls it).

The network has no reference counterpart (the reference is a direct solver only,
docs/linear-solvers.md:375-376); this is a plain numpy restatement of the same architecture the GPU
builds (include/fieldcraft_unet.h): 3x3x3 'same' convolutions with zero padding, leaky ReLU
(slope SLOPE), 2x2x2
average pooling (sum / 8 over the children present), nearest upsampling, additive skips. With
`bf16=True` values are rounded to bfloat16 (round to nearest even) at the points where the GPU
stores BF16 (inputs, weights, every stored activation and activation gradient), and sums are
exact-ish (float64), so the GPU differs from it only by its FP32 summation order. With
`bf16=False` everything is float64, for finite-difference checks of the gradients themselves.

Grids are arrays [Z, Y, X, C]; weights [27, cout, cin] with tap = dx+1 + 3 (dy+1) + 9 (dz+1).
"""
from __future__ import annotations

import numpy as np

C, CIO = 32, 16
SLOPE = 0.05  # leaky ReLU: x for x > 0, SLOPE x otherwise


def layers(levels: int = 3):
    """(cin, cout, level) of each convolution in forward order for a network of `levels` levels:
    two per level on the way down (the first from the CIO input channels), two at the bottom, two
    per level on the way up, and the output convolution to CIO channels (4 levels - 1 in all)."""
    out = []
    for lv in range(levels):
        out += [(CIO if lv == 0 else C, C, lv), (C, C, lv)]
    for lv in range(levels - 2, -1, -1):
        out += [(C, C, lv), (C, C, lv)]
    return out + [(C, CIO, 0)]


LAYERS = layers(3)


def bf16(a) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split_params(flat: np.ndarray, levels: int = 3):
    """The flat FP32 parameter vector (per layer: weights [27][cout][cin], then biases) as lists."""
    ws, bs, off = [], [], 0
    for cin, cout, _ in layers(levels):
        nw = 27 * cin * cout
        ws.append(np.asarray(flat[off:off + nw], np.float64).reshape(27, cout, cin))
        off += nw
        bs.append(np.asarray(flat[off:off + cout], np.float64))
        off += cout
    return ws, bs


def join_params(ws, bs) -> np.ndarray:
    return np.concatenate([np.concatenate([w.reshape(-1), b]) for w, b in zip(ws, bs)])


def coarser(shape):
    return tuple((s + 1) // 2 for s in shape)


def _shift(a: np.ndarray, dz: int, dy: int, dx: int) -> np.ndarray:
    """out[z, y, x] = a[z + dz, y + dy, x + dx], zero outside."""
    out = np.zeros_like(a)
    Z, Y, X = a.shape[:3]
    zs, ys, xs = slice(max(0, -dz), min(Z, Z - dz)), slice(max(0, -dy), min(Y, Y - dy)), slice(max(0, -dx), min(X, X - dx))
    zt, yt, xt = slice(max(0, dz), min(Z, Z + dz)), slice(max(0, dy), min(Y, Y + dy)), slice(max(0, dx), min(X, X + dx))
    out[zs, ys, xs] = a[zt, yt, xt]
    return out


def taps():
    for t in range(27):
        yield t, t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1


def conv(x, w, b=None):
    out = np.zeros(x.shape[:3] + (w.shape[1],))
    for t, dx, dy, dz in taps():
        out += _shift(x, dz, dy, dx) @ w[t].T
    if b is not None:
        out += b
    return out


def conv_t(dy, w):
    """The input gradient of conv: sum over taps of dy[v - tap] w[tap]."""
    out = np.zeros(dy.shape[:3] + (w.shape[2],))
    for t, dx, ddy, dz in taps():
        out += _shift(dy, -dz, -ddy, -dx) @ w[t]
    return out


def conv_dw(x, dy):
    gw = np.zeros((27, dy.shape[3], x.shape[3]))
    for t, dx, ddy, dz in taps():
        xs = _shift(x, dz, ddy, dx)
        gw[t] = dy.reshape(-1, dy.shape[3]).T @ xs.reshape(-1, xs.shape[3])
    return gw, dy.reshape(-1, dy.shape[3]).sum(axis=0)


def pool(f):
    Zc, Yc, Xc = coarser(f.shape[:3])
    out = np.zeros((Zc, Yc, Xc, f.shape[3]))
    for k in range(8):
        oz, oy, ox = k >> 2, (k >> 1) & 1, k & 1
        part = f[oz::2, oy::2, ox::2]
        out[:part.shape[0], :part.shape[1], :part.shape[2]] += part
    return out * 0.125


def up(c, shape):
    Z, Y, X = shape
    return c[np.arange(Z)[:, None, None] // 2, np.arange(Y)[None, :, None] // 2, np.arange(X)[None, None, :] // 2]


def up_adjoint(df, shape_c):
    out = np.zeros(tuple(shape_c) + (df.shape[3],))
    for k in range(8):
        oz, oy, ox = k >> 2, (k >> 1) & 1, k & 1
        part = df[oz::2, oy::2, ox::2]
        out[:part.shape[0], :part.shape[1], :part.shape[2]] += part
    return out


def pool_adjoint(dc, shape_f):
    return up(dc, shape_f) * 0.125


class Net:
    """forward(x) -> y, keeping what backward(dy) needs; backward returns (grads_w, grads_b).
    `levels` levels: per level on the way down two convolutions (the second's output is the skip)
    and a 2x2x2 average pooling, two convolutions at the bottom, per level on the way up nearest
    upsampling plus the skip and two convolutions, then the output convolution."""

    def __init__(self, flat_params: np.ndarray, use_bf16: bool = True, levels: int = 3):
        self.levels = levels
        self.ws, self.bs = split_params(flat_params, levels)
        self.q = bf16 if use_bf16 else (lambda a: np.asarray(a, np.float64))
        self.ws = [self.q(w) for w in self.ws]

    def forward(self, x):
        q, W, Bv, D = self.q, self.ws, self.bs, self.levels
        relu = lambda a: np.where(a > 0, a, SLOPE * a)
        s = self.s = {"x": q(x)}
        inp, k = s["x"], 0
        for lv in range(D):  # down, then the bottom
            s[f"in{lv}"] = inp
            s[f"a{lv}"] = q(relu(conv(inp, W[k], Bv[k])))
            s[f"s{lv}"] = q(relu(conv(s[f"a{lv}"], W[k + 1], Bv[k + 1])))
            k += 2
            if lv < D - 1:
                inp = q(pool(s[f"s{lv}"]))
        low = s[f"s{D - 1}"]
        for lv in range(D - 2, -1, -1):  # up
            s[f"u{lv}"] = q(up(low, s[f"s{lv}"].shape[:3]) + s[f"s{lv}"])
            s[f"b{lv}"] = q(relu(conv(s[f"u{lv}"], W[k], Bv[k])))
            s[f"d{lv}"] = q(relu(conv(s[f"b{lv}"], W[k + 1], Bv[k + 1])))
            k += 2
            low = s[f"d{lv}"]
        s["top"] = low
        s["y"] = q(conv(low, W[k], Bv[k]))
        return s["y"]

    def backward(self, dy):
        q, W, s, D = self.q, self.ws, self.s, self.levels
        mask = lambda a: np.where(a > 0, 1.0, SLOPE)
        nl = len(W)
        gw, gb = [None] * nl, [None] * nl
        dy = q(dy)
        k = nl - 1
        gw[k], gb[k] = conv_dw(s["top"], dy)
        g = q(conv_t(dy, W[k]) * mask(s["top"]))  # dL/d(top), through its activation
        gskip = {}
        for lv in range(0, D - 1):  # up path, from the top level down to the coarsest
            k -= 2
            gw[k + 1], gb[k + 1] = conv_dw(s[f"b{lv}"], g)
            g = q(conv_t(g, W[k + 1]) * mask(s[f"b{lv}"]))
            gw[k], gb[k] = conv_dw(s[f"u{lv}"], g)
            gu = q(conv_t(g, W[k]))  # dL/du: to the skip and, upsampled, to the level below
            gskip[lv] = gu
            below = s[f"d{lv + 1}"] if lv + 1 < D - 1 else s[f"s{D - 1}"]
            g = q(up_adjoint(gu, below.shape[:3]) * mask(below))
        for lv in range(D - 1, -1, -1):  # down path, from the bottom up
            k -= 2
            gw[k + 1], gb[k + 1] = conv_dw(s[f"a{lv}"], g)
            g = q(conv_t(g, W[k + 1]) * mask(s[f"a{lv}"]))
            gw[k], gb[k] = conv_dw(s[f"in{lv}"], g)
            if lv == 0:
                break
            g = q(conv_t(g, W[k]))  # dL/d(pooled input of level lv)
            g = q((pool_adjoint(g, s[f"s{lv - 1}"].shape[:3]) + gskip[lv - 1]) * mask(s[f"s{lv - 1}"]))
        return gw, gb


def init_params(seed: int, levels: int = 3) -> np.ndarray:
    """Random parameters of the network's layout (for checks; not the GPU's initialisation)."""
    rng = np.random.default_rng(seed)
    ws, bs = [], []
    for cin, cout, _ in layers(levels):
        ws.append(rng.standard_normal((27, cout, cin)) * np.sqrt(2.0 / (27 * cin)))
        bs.append(rng.standard_normal(cout) * 0.05)
    return join_params(ws, bs).astype(np.float32)
