"""Helpers shared by the GPU parity tests."""
import numpy as np

F32 = np.float32


def relmse(x, y):
    """mean over pixels and channels of (x - y)^2 / (y^2 + 1e-2)."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    return float(np.mean((x - y) ** 2 / (y * y + 1e-2)))


def bits_equal_fraction(a, b):
    a = np.ascontiguousarray(a, F32).view(np.uint32)
    b = np.ascontiguousarray(b, F32).view(np.uint32)
    return float(np.mean(a == b))


def interior_rays(n, seed, lo=0.05, hi=0.95, tmax=1e9):
    rng = np.random.default_rng(seed)
    rays = np.zeros((n, 8), F32)
    rays[:, :3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = tmax
    return rays


def compare_closest(gpu_hits, orc_hits):
    """Closest-hit parity: identical records, except ties where the two hit
    distances agree within 1e-6 relative (both found)."""
    same = (gpu_hits == orc_hits).all(1)
    bad = np.nonzero(~same)[0]
    ties = 0
    for k in bad:
        g, o = gpu_hits[k], orc_hits[k]
        gi, oi = g[3] != 0xFFFFFFFF, o[3] != 0xFFFFFFFF
        assert gi and oi, f"ray {k}: found mismatch gpu={g} oracle={o}"
        tg = g[2:3].view(F32)[0]
        to = o[2:3].view(F32)[0]
        assert abs(tg - to) <= 1e-6 * abs(to), f"ray {k}: t {tg} vs {to}"
        ties += 1
    return ties
