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


def vertex_edge_rays(seed_origins=None):
    """Rays from points inside the unit Cornell box aimed at the vertices and
    edge midpoints of its 16x16 wall grid, where two or more triangles share
    the hit point and closest-hit ties in t are common."""
    g = np.concatenate([np.arange(17) / 16.0, (np.arange(16) + 0.5) / 16.0]).astype(F32)
    a, b = np.meshgrid(g, g)
    a, b = a.ravel(), b.ravel()
    targets = []
    for axis in range(3):
        others = [k for k in range(3) if k != axis]
        for val in (0.0, 1.0):
            t = np.zeros((a.size, 3), F32)
            t[:, axis] = val
            t[:, others[0]] = a
            t[:, others[1]] = b
            targets.append(t)
    targets = np.concatenate(targets)
    origins = np.array(seed_origins or [[0.5, 0.5, 0.5], [0.25, 0.5, 0.5], [0.5, 0.3, 0.7], [0.31, 0.62, 0.44]], F32)
    rays = []
    for o in origins:
        d = targets - o
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        r = np.zeros((targets.shape[0], 8), F32)
        r[:, :3] = o
        r[:, 3] = 1e9
        r[:, 4:7] = d
        rays.append(r)
    return np.concatenate(rays)


def chain_bvh(scene):
    """A chain-shaped BVH over the triangles of a one-instance identity scene
    (scenes.soup): inner node k has leaf k as its left child and inner node
    k + 1 as its right child, in the reference's flattened depth-first layout
    (inner k at index 2k, leaf k at 2k + 1, the last leaf at 2(n - 1)).  Its
    depth is n - 1; boxes enclose their subtrees, padded +1e-6 on the max
    corner like the builders."""
    import copy
    n = scene.num_triangles
    pos = scene.vb.view(F32).reshape(-1, 8)[:, :3]
    tri = pos[scene.ib.reshape(-1, 3)]  # (n, 3, 3)
    lo_t, hi_t = tri.min(1), tri.max(1) + F32(1e-6)
    N = 2 * n - 1
    f = np.zeros((N, 8), F32)
    u = f.view(np.int32)
    # suffix bounds: box of triangles k .. n-1
    slo = np.minimum.accumulate(lo_t[::-1], axis=0)[::-1]
    shi = np.maximum.accumulate(hi_t[::-1], axis=0)[::-1]
    for k in range(n - 1):
        i = 2 * k
        f[i, 0:3], f[i, 4:7] = slo[k], shi[k]
        u[i, 3] = -1
        u[i, 7] = -1                       # escape of every inner node: the end
        leaf = 2 * k + 1
        f[leaf, 0:3], f[leaf, 4:7] = lo_t[k], hi_t[k]
        u[leaf, 0] = k                     # minBounds[0] holds the triangle index bits
        u[leaf, 3] = 0                     # instance 0
        u[leaf, 7] = 2 * k + 2             # escape: the right sibling
    last = 2 * (n - 1)
    f[last, 0:3], f[last, 4:7] = lo_t[n - 1], hi_t[n - 1]
    u[last, 0] = n - 1
    u[last, 3] = 0
    u[last, 7] = -1
    c = copy.copy(scene)
    c.nodes = f.view(np.uint8).reshape(-1).copy()
    return c
