"""The host SAH builder emits the reference's flattened depth-first layout
(src/render/bvh.cpp:169-235), and stackless traversal over it finds the same
closest hit as a brute-force loop over every triangle."""
import numpy as np

import oracle
from strelka_b200 import scenes


def node_arrays(nodes_u8):
    n = nodes_u8.view(np.float32).reshape(-1, 8)
    i = nodes_u8.view(np.int32).reshape(-1, 8)
    return n, i


def check_layout(nodes_u8, num_tris):
    f, i = node_arrays(nodes_u8)
    N = f.shape[0]
    assert N == 2 * num_tris - 1
    leaves = i[:, 3] != -1
    assert leaves.sum() == num_tris
    # walk the implicit tree: inner node k has left child k+1 and right child
    # escape(k+1); escapes of the left child point to the right sibling
    seen = np.zeros(N, bool)
    stack = [(0, -1)]
    leaf_prims = []
    while stack:
        k, esc = stack.pop()
        assert not seen[k]
        seen[k] = True
        assert i[k, 7] == esc
        if leaves[k]:
            leaf_prims.append((i[k, 3], i[k, 0]))
            continue
        left = k + 1
        right = i[left, 7]
        assert 0 < right < N
        # parent bounds contain the children's bounds (inner children)
        for c in (left, right):
            if not leaves[c]:
                assert (f[c, 0:3] >= f[k, 0:3]).all() and (f[c, 4:7] <= f[k, 4:7]).all()
        stack.append((right, esc))
        stack.append((left, right))
    assert seen.all()
    assert len(set(leaf_prims)) == num_tris


def test_layout_soup():
    s = scenes.soup(3000, 11)
    check_layout(s.nodes, 3000)


def test_layout_cornell():
    s = scenes.cornell(32, 32, sphere_levels=2)
    check_layout(s.nodes, s.num_triangles)


def test_single_triangle_and_empty():
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    nodes = scenes.bvh_build(pos, np.zeros(3, np.uint32), np.zeros(3, np.uint32))
    i = nodes.view(np.int32).reshape(-1, 8)
    assert i.shape[0] == 1 and i[0, 3] == 0 and i[0, 7] == -1
    assert scenes.bvh_build(np.zeros((0, 3), np.float32), np.zeros(0, np.uint32), np.zeros(0, np.uint32)).size == 0


def test_identical_centroids_split():
    # every triangle identical: the builder falls back to median splits
    pos = np.tile(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), (17, 1))
    ids = np.repeat(np.arange(17, dtype=np.uint32), 3)
    nodes = scenes.bvh_build(pos, np.zeros(51, np.uint32), ids)
    check_layout(nodes, 17)


def test_deterministic():
    a = scenes.soup(20000, 2).nodes
    b = scenes.soup(20000, 2).nodes
    assert np.array_equal(a, b)


def world_triangles(s):
    """(T, 3, 3) float32 world-space corners, mul(M, float4(p, 1)) summed left
    to right in float32 like the kernels, plus (instId, primId) per triangle."""
    vb = s.vb.view(np.float32).reshape(-1, 8)[:, :3]
    inst = s.instances.view(np.float32).reshape(-1, 52)
    ii = s.instances.view(np.int32).reshape(-1, 52)
    tris, ids = [], []
    for k in range(inst.shape[0]):
        m = inst[k, :16]
        off, cnt = ii[k, 49], ii[k, 50]
        idx = s.ib[off:off + cnt].reshape(-1, 3)
        p = vb[idx]  # (t, 3, 3)
        w = np.empty_like(p)
        for r in range(3):
            w[..., r] = ((m[r] * p[..., 0] + m[4 + r] * p[..., 1]) + m[8 + r] * p[..., 2]) + m[12 + r] * np.float32(1)
        tris.append(w)
        ids += [(k, t) for t in range(idx.shape[0])]
    return np.concatenate(tris), ids


def brute_force_closest(s, rays):
    """Loop over all triangles with the oracle's own MT (raytracing.h:36-88):
    the minimum t with t < tmax."""
    import ctypes as C
    orc = oracle.load()
    tris, ids = world_triangles(s)
    out = []
    for r in rays:
        best = (np.float32(1e9), None)
        o = np.ascontiguousarray(r[:3])
        d = np.ascontiguousarray(r[4:7])
        for k in range(tris.shape[0]):
            v0 = np.ascontiguousarray(tris[k, 0])
            e0 = np.ascontiguousarray(tris[k, 1] - tris[k, 0])
            e1 = np.ascontiguousarray(tris[k, 2] - tris[k, 0])
            t, u, v = C.c_float(), C.c_float(), C.c_float()
            hit = orc.oracle_ray_triangle(o.ctypes.data, d.ctypes.data, v0.ctypes.data, e0.ctypes.data,
                                          e1.ctypes.data, C.byref(t), C.byref(u), C.byref(v))
            if hit and t.value < r[3] and np.float32(t.value) < best[0]:
                best = (np.float32(t.value), ids[k])
        out.append(best)
    return out


def test_traversal_equals_brute_force():
    s = scenes.cornell(16, 16, sphere_levels=1)
    v = oracle.SceneView(s)
    rng = np.random.default_rng(5)
    n = 300
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = rng.uniform(0.05, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = 1e9
    rays[:, 3][: n // 3] = 0.3  # some short rays
    hits, found, _ = oracle.trace(v, rays)
    bf = brute_force_closest(s, rays)
    nfound = 0
    for k, (t, prim) in enumerate(bf):
        assert found[k] == (prim is not None)
        if prim is not None:
            nfound += 1
            assert hits[k, 2].view(np.float32) == t
    assert nfound > 150
