"""CPU reference of the neural radiance cache (TEST INFRASTRUCTURE ONLY).

Restates, in numpy, the encoding, forward pass, relative-L2 loss and the
backward pass of strelka_b200/csrc/nrc.cu with the same rounding points
(FP16 inputs, activations and backward intermediates; FP32 encoding
arithmetic in the kernel's order; products accumulated in FP64 here where
the kernel accumulates in FP32 on tensor cores), so the GPU's gradients can
be checked against it.  The cache has no counterpart in the reference.
"""
from __future__ import annotations

import numpy as np

LEVELS = 16
IN = 64
WIDTH = 64
OUT_PAD = 16
PARAMS = 4 * WIDTH * IN + OUT_PAD * IN
GRAD_SCALE = 1.0 / 128.0
GRAD_CLAMP = 1024.0

SH_C = dict(c00=0.28209479177387814, c1=0.4886025119029199, c2m2=1.0925484305920792, c20=0.31539156525252005,
            c22=0.5462742152960396, c3m3=0.5900435899266435, c3m2=2.890611442640554, c3m1=0.4570457994644658,
            c30=0.3731763325901154, c32=1.445305721320277)

f32 = np.float32


def level_table(log2_t: int):
    T = 1 << log2_t
    res = [int(np.floor(16.0 * 1.5 ** l)) for l in range(LEVELS)]
    dense = [(r + 1.0) ** 3 <= T for r in res]
    return T, res, dense


def records_to_arrays(rec: np.ndarray):
    """rec: (n, 16) float32 view of StrelkaNrcRecord rows."""
    return rec[:, 0:3], rec[:, 3:6], rec[:, 6:9], rec[:, 9], rec[:, 10:13]


def corners(pn, l, res, dense, T):
    """(n, 8) indices into the flattened grid (level-major) and weights."""
    r = res[l]
    x = pn * f32(r)
    i = np.clip(np.floor(x).astype(np.int64), 0, r - 1)
    f = np.clip(x - i.astype(f32), f32(0), f32(1)).astype(f32)
    idx = np.zeros((pn.shape[0], 8), np.uint64)
    w = np.zeros((pn.shape[0], 8), f32)
    for k in range(8):
        off = np.array([k & 1, (k >> 1) & 1, k >> 2])
        c = (i + off).astype(np.uint64)
        if dense[l]:
            s = np.uint64(r + 1)
            h = c[:, 0] + s * (c[:, 1] + s * c[:, 2])
        else:
            h = (c[:, 0] * np.uint64(1)) ^ (c[:, 1] * np.uint64(2654435761)) ^ (c[:, 2] * np.uint64(805459861))
            h = h & np.uint64(0xFFFFFFFF)
        idx[:, k] = (h & np.uint64(T - 1)) + np.uint64(l * T)
        wx = np.where(off[0], f[:, 0], f32(1) - f[:, 0]).astype(f32)
        wy = np.where(off[1], f[:, 1], f32(1) - f[:, 1]).astype(f32)
        wz = np.where(off[2], f[:, 2], f32(1) - f[:, 2]).astype(f32)
        w[:, k] = (wx * wy).astype(f32) * wz
    return idx, w


def sh16(d):
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    c = {k: f32(v) for k, v in SH_C.items()}
    xx, yy, zz = x * x, y * y, z * z
    o = [np.full_like(x, c["c00"]), -c["c1"] * y, c["c1"] * z, -c["c1"] * x,
         c["c2m2"] * x * y, -c["c2m2"] * y * z, c["c20"] * (f32(3) * zz - f32(1)), -c["c2m2"] * x * z,
         c["c22"] * (xx - yy),
         -c["c3m3"] * y * (f32(3) * xx - yy), c["c3m2"] * x * y * z, -c["c3m1"] * y * (f32(5) * zz - f32(1)),
         c["c30"] * z * (f32(5) * zz - f32(3)), -c["c3m1"] * x * (f32(5) * zz - f32(1)), c["c32"] * z * (xx - yy),
         -c["c3m3"] * x * (xx - f32(3) * yy)]
    return np.stack(o, 1).astype(f32)


def encode(rec, grid_half, bmin, bmax, log2_t):
    """Inputs (n, 64) float16 and the per-level corner tables."""
    T, res, dense = level_table(log2_t)
    pos, d, nrm, rough, _ = records_to_arrays(rec)
    binv = np.where(bmax - bmin > 0, f32(1) / (bmax - bmin).astype(f32), f32(0)).astype(f32)
    pn = np.clip((pos - bmin.astype(f32)) * binv, f32(0), f32(1)).astype(f32)
    g = grid_half.astype(f32).reshape(-1, 2)
    x = np.zeros((rec.shape[0], IN), np.float16)
    tabs = []
    for l in range(LEVELS):
        idx, w = corners(pn, l, res, dense, T)
        tabs.append((idx, w))
        f0 = np.zeros(rec.shape[0], f32)
        f1 = np.zeros(rec.shape[0], f32)
        for k in range(8):
            v = g[idx[:, k].astype(np.int64)]
            f0 = (f0 + w[:, k] * v[:, 0]).astype(f32)
            f1 = (f1 + w[:, k] * v[:, 1]).astype(f32)
        x[:, 2 * l] = f0.astype(np.float16)
        x[:, 2 * l + 1] = f1.astype(np.float16)
    x[:, 32:48] = sh16(d).astype(np.float16)
    x[:, 48:51] = (nrm * f32(0.5) + f32(0.5)).astype(np.float16)
    x[:, 51] = rough.astype(np.float16)
    x[:, 52] = np.float16(1.0)
    return x, tabs


def split_weights(mlp_half):
    Ws = [mlp_half[l * WIDTH * IN:(l + 1) * WIDTH * IN].reshape(WIDTH, IN) for l in range(4)]
    Ws.append(mlp_half[4 * WIDTH * IN:].reshape(OUT_PAD, IN))
    return [w.astype(np.float64) for w in Ws]


def forward(x, mlp_half, exact=False):
    """Returns y (n, 3) and the layer inputs [x, h1, h2, h3, h4] (FP16, or
    FP64 when exact)."""
    Ws = split_weights(mlp_half)
    acts = [x]
    a = x.astype(np.float64)
    for l in range(4):
        h = np.maximum(a @ Ws[l].T, 0.0)
        if not exact:
            h = h.astype(np.float16)
        acts.append(h)
        a = h.astype(np.float64)
    y = (a @ Ws[4].T)[:, :3]
    return (y if exact else y.astype(f32)), acts


def gradients(rec, mlp, grid, bmin, bmax, log2_t, exact=False):
    """Gradients of sum_i sum_c (y - t)^2 / (y^2 + 0.01) (with the kernel's
    clamp of dL/dy at +-1024), w.r.t. the FP32 master parameters, and the
    loss sum.  The denominator is treated as a constant (stop-gradient).
    exact=True drops every FP16 rounding and the clamp (for finite
    differences of the reference itself); the MLP input x stays as given."""
    mlp_half = mlp if exact else mlp.astype(np.float16)
    grid_half = grid if exact else grid.astype(np.float16)
    x, tabs = encode(rec, grid_half, bmin, bmax, log2_t)
    y, acts = forward(x, mlp_half, exact)
    t = rec[:, 10:13]
    if exact:
        den = y * y + 0.01
        diff = y - t
        loss = float(np.sum(diff ** 2 / den))
        g = 2 * diff / den * GRAD_SCALE
        d = np.zeros((rec.shape[0], OUT_PAD), np.float64)
        d[:, :3] = g
    else:
        den = (y * y + f32(0.01)).astype(f32)
        diff = (y - t).astype(f32)
        loss = float(np.sum(diff.astype(np.float64) ** 2 / den))
        g = np.clip(f32(2) * diff / den, -GRAD_CLAMP, GRAD_CLAMP) * f32(GRAD_SCALE)
        d = np.zeros((rec.shape[0], OUT_PAD), np.float16)
        d[:, :3] = g.astype(np.float16)
    Ws = split_weights(mlp_half)
    dW = [None] * 5
    dx = None
    for l in range(4, -1, -1):
        a_in = acts[l].astype(np.float64)
        dd = d.astype(np.float64)
        dW[l] = dd.T @ a_in
        din = dd @ Ws[l]
        if l > 0:
            mask = acts[l] > 0
            d = din * mask if exact else (din * mask).astype(np.float16)
        else:
            dx = din[:, :32]
    mlp_grad = np.concatenate([w.ravel() for w in dW]) / GRAD_SCALE
    grid_grad = np.zeros(grid.shape[0], np.float64)
    for l in range(LEVELS):
        idx, w = tabs[l]
        for k in range(8):
            ii = idx[:, k].astype(np.int64)
            np.add.at(grid_grad, 2 * ii, w[:, k] * dx[:, 2 * l])
            np.add.at(grid_grad, 2 * ii + 1, w[:, k] * dx[:, 2 * l + 1])
    return mlp_grad, grid_grad / GRAD_SCALE, loss


def infer(rec, mlp, grid, bmin, bmax, log2_t):
    x, _ = encode(rec, grid.astype(np.float16), bmin, bmax, log2_t)
    y, _ = forward(x, mlp.astype(np.float16))
    return y
