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
LAYERS = [(CIO, C, 0), (C, C, 0), (C, C, 1), (C, C, 1), (C, C, 2), (C, C, 2), (C, C, 1), (C, C, 1), (C, C, 0),
          (C, C, 0), (C, CIO, 0)]  # (cin, cout, level)


def bf16(a) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split_params(flat: np.ndarray):
    """The flat FP32 parameter vector (per layer: weights [27][cout][cin], then biases) as lists."""
    ws, bs, off = [], [], 0
    for cin, cout, _ in LAYERS:
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
    """forward(x) -> y, keeping what backward(dy) needs; backward returns (grads_w, grads_b)."""

    def __init__(self, flat_params: np.ndarray, use_bf16: bool = True):
        self.ws, self.bs = split_params(flat_params)
        self.q = bf16 if use_bf16 else (lambda a: np.asarray(a, np.float64))
        self.ws = [self.q(w) for w in self.ws]

    def forward(self, x):
        q, W, Bv = self.q, self.ws, self.bs
        relu = lambda a: np.where(a > 0, a, SLOPE * a)
        s = self.s = {}
        g0 = x.shape[:3]
        g1 = coarser(g0)
        s["x"] = q(x)
        s["a0"] = q(relu(conv(s["x"], W[0], Bv[0])))
        s["s0"] = q(relu(conv(s["a0"], W[1], Bv[1])))
        s["p1"] = q(pool(s["s0"]))
        s["a1"] = q(relu(conv(s["p1"], W[2], Bv[2])))
        s["s1"] = q(relu(conv(s["a1"], W[3], Bv[3])))
        s["p2"] = q(pool(s["s1"]))
        s["a2"] = q(relu(conv(s["p2"], W[4], Bv[4])))
        s["m2"] = q(relu(conv(s["a2"], W[5], Bv[5])))
        s["u1"] = q(up(s["m2"], g1) + s["s1"])
        s["a3"] = q(relu(conv(s["u1"], W[6], Bv[6])))
        s["d1"] = q(relu(conv(s["a3"], W[7], Bv[7])))
        s["u0"] = q(up(s["d1"], g0) + s["s0"])
        s["a4"] = q(relu(conv(s["u0"], W[8], Bv[8])))
        s["d0"] = q(relu(conv(s["a4"], W[9], Bv[9])))
        s["y"] = q(conv(s["d0"], W[10], Bv[10]))
        return s["y"]

    def backward(self, dy):
        q, W, s = self.q, self.ws, self.s
        mask = lambda a: np.where(a > 0, 1.0, SLOPE)
        g0, g1, g2 = s["x"].shape[:3], s["p1"].shape[:3], s["p2"].shape[:3]
        gw, gb = [None] * 11, [None] * 11
        dy = q(dy)
        gw[10], gb[10] = conv_dw(s["d0"], dy)
        g = q(conv_t(dy, W[10]) * mask(s["d0"]))
        gw[9], gb[9] = conv_dw(s["a4"], g)
        g = q(conv_t(g, W[9]) * mask(s["a4"]))
        gw[8], gb[8] = conv_dw(s["u0"], g)
        gs0 = q(conv_t(g, W[8]))
        g = q(up_adjoint(gs0, g1) * mask(s["d1"]))
        gw[7], gb[7] = conv_dw(s["a3"], g)
        g = q(conv_t(g, W[7]) * mask(s["a3"]))
        gw[6], gb[6] = conv_dw(s["u1"], g)
        gs1 = q(conv_t(g, W[6]))
        g = q(up_adjoint(gs1, g2) * mask(s["m2"]))
        gw[5], gb[5] = conv_dw(s["a2"], g)
        g = q(conv_t(g, W[5]) * mask(s["a2"]))
        gw[4], gb[4] = conv_dw(s["p2"], g)
        g = q(conv_t(g, W[4]))
        g = q((pool_adjoint(g, g1) + gs1) * mask(s["s1"]))
        gw[3], gb[3] = conv_dw(s["a1"], g)
        g = q(conv_t(g, W[3]) * mask(s["a1"]))
        gw[2], gb[2] = conv_dw(s["p1"], g)
        g = q(conv_t(g, W[2]))
        g = q((pool_adjoint(g, g0) + gs0) * mask(s["s0"]))
        gw[1], gb[1] = conv_dw(s["a0"], g)
        g = q(conv_t(g, W[1]) * mask(s["a0"]))
        gw[0], gb[0] = conv_dw(s["x"], g)
        return gw, gb


def init_params(seed: int) -> np.ndarray:
    """Random parameters of the network's layout (for checks; not the GPU's initialisation)."""
    rng = np.random.default_rng(seed)
    ws, bs = [], []
    for cin, cout, _ in LAYERS:
        ws.append(rng.standard_normal((27, cout, cin)) * np.sqrt(2.0 / (27 * cin)))
        bs.append(rng.standard_normal(cout) * 0.05)
    return join_params(ws, bs).astype(np.float32)
