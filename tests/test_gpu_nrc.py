"""Neural radiance cache kernels against the CPU reference (oracle/nrc_ref.py):
forward outputs, weight and hash-grid gradients, and that Adam training on
the GPU fits a radiance field."""
import ctypes as C

import numpy as np
import pytest

from oracle import nrc_ref
from strelka_b200 import abi
from strelka_b200.render import to_device

pytestmark = pytest.mark.gpu

LOG2_T = 14  # small tables keep the CPU reference fast; levels 0..2 dense, the rest hashed
BMIN = np.array([-1.0, -1.0, -1.0], np.float32)
BMAX = np.array([2.0, 1.5, 1.0], np.float32)


def make_nrc(seed=5, lr=1e-2, log2_t=LOG2_T):
    lib = abi.load()
    cfg = abi.StrelkaNrcConfig((C.c_float * 3)(*BMIN), (C.c_float * 3)(*BMAX), lr, seed, log2_t, (C.c_uint32 * 3)())
    h = C.c_void_p()
    abi.check(lib.strelka_nrc_create(C.byref(cfg), C.byref(h)))
    nm = C.c_uint32()
    ng = C.c_uint64()
    lib.strelka_nrc_info(h, C.byref(nm), C.byref(ng), None)
    return lib, h, nm.value, ng.value


def records(n, seed, target_fn=None):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 16), np.float32)
    r[:, 0:3] = rng.uniform(BMIN, BMAX, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3))
    r[:, 6:9] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    r[:, 9] = rng.uniform(0.05, 1.0, n)
    if target_fn is None:
        r[:, 10:13] = rng.gamma(1.0, 1.0, (n, 3))
    else:
        r[:, 10:13] = target_fn(r)
    return r


def params(lib, h, nm, ng):
    mlp = np.zeros(nm, np.float32)
    grid = np.zeros(ng, np.float32)
    abi.check(lib.strelka_nrc_get_params(h, mlp.ctypes.data, grid.ctypes.data))
    return mlp, grid


def test_forward_matches_reference(cuda):
    lib, h, nm, ng = make_nrc()
    assert nm == nrc_ref.PARAMS and ng == 16 * (1 << LOG2_T) * 2
    rng = np.random.default_rng(0)
    mlp, grid = params(lib, h, nm, ng)
    # a grid with visible structure so the encoding matters
    grid = rng.normal(0, 0.5, ng).astype(np.float32)
    abi.check(lib.strelka_nrc_set_params(h, None, grid.ctypes.data))
    rec = records(3000, 1)
    out = cuda.zeros(3000 * 3, dtype=cuda.float32, device="cuda")
    abi.check(lib.strelka_nrc_infer(h, to_device(rec).data_ptr(), 3000, out.data_ptr(), None))
    cuda.cuda.synchronize()
    got = out.cpu().numpy().reshape(-1, 3)
    ref = nrc_ref.infer(rec, mlp, grid, BMIN, BMAX, LOG2_T)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 2e-2 * scale, (np.abs(got - ref).max(), scale)
    status = C.c_uint32(123)
    abi.check(lib.strelka_nrc_get_device_status(h, None, C.byref(status)))
    assert status.value == 0  # no tensor-core wait ran out
    lib.strelka_nrc_destroy(h)


@pytest.mark.parametrize("log2_t", [LOG2_T, 19])
def test_gradients_match_reference(cuda, log2_t):
    # 2^19 is the table of the radiance-cache workload: levels 0-3 dense,
    # levels 4-15 hashed into 2^19 entries
    lib, h, nm, ng = make_nrc(seed=9, log2_t=log2_t)
    assert ng == 16 * (1 << log2_t) * 2
    rng = np.random.default_rng(1)
    mlp, _ = params(lib, h, nm, ng)
    grid = rng.normal(0, 0.3, ng).astype(np.float32)
    abi.check(lib.strelka_nrc_set_params(h, None, grid.ctypes.data))
    rec = records(2048, 2)
    gm = np.zeros(nm, np.float32)
    gg = np.zeros(ng, np.float32)
    loss = C.c_float()
    abi.check(lib.strelka_nrc_gradients(h, to_device(rec).data_ptr(), 2048, gm.ctypes.data, gg.ctypes.data,
                                        C.byref(loss), None))
    rm, rg, rloss = nrc_ref.gradients(rec, mlp, grid, BMIN, BMAX, log2_t)
    assert abs(loss.value - rloss) <= 1e-3 * abs(rloss)
    # per weight matrix: relative error of the gradient and its direction
    offs = [0, 4096, 8192, 12288, 16384, nm]
    for l in range(5):
        a, b = gm[offs[l]:offs[l + 1]].astype(np.float64), rm[offs[l]:offs[l + 1]]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        assert rel < 2e-2 and cos > 0.9995, (l, rel, cos)
    rel = np.linalg.norm(gg - rg) / np.linalg.norm(rg)
    cos = gg.astype(np.float64) @ rg / (np.linalg.norm(gg) * np.linalg.norm(rg))
    assert rel < 3e-2 and cos > 0.999, (rel, cos)
    lib.strelka_nrc_destroy(h)


def test_training_fits_a_radiance_field(cuda):
    lib, h, nm, ng = make_nrc(seed=3, lr=1e-2)

    def field(r):
        p, d = r[:, 0:3], r[:, 3:6]
        base = 1.0 + 0.5 * np.sin(3 * p[:, 0:1]) * np.cos(2 * p[:, 1:2]) + 0.3 * d[:, 2:3]
        return np.clip(base * np.array([1.0, 0.6, 0.3]), 0.0, None).astype(np.float32)

    test = records(4096, 77, field)
    losses = []
    for step in range(300):
        batch = records(8192, 1000 + step, field)
        loss = C.c_float()
        abi.check(lib.strelka_nrc_train(h, to_device(batch).data_ptr(), 8192, C.byref(loss), None))
        losses.append(loss.value)
    out = cuda.zeros(4096 * 3, dtype=cuda.float32, device="cuda")
    abi.check(lib.strelka_nrc_infer(h, to_device(test).data_ptr(), 4096, out.data_ptr(), None))
    cuda.cuda.synchronize()
    pred = out.cpu().numpy().reshape(-1, 3)
    t = test[:, 10:13]
    rel = np.mean((pred - t) ** 2 / (t * t + 1e-2))
    assert np.mean(losses[-20:]) < 0.05 * np.mean(losses[:5]), (losses[:5], losses[-5:])
    assert rel < 0.02, rel
    lib.strelka_nrc_destroy(h)


@pytest.mark.parametrize("n", [200, 1])
def test_gradients_partial_tile(cuda, n):
    # a batch that fills no whole 128-record tile: the padded rows of the last
    # tile contribute nothing
    lib, h, nm, ng = make_nrc(seed=4)
    rng = np.random.default_rng(6)
    mlp, _ = params(lib, h, nm, ng)
    grid = rng.normal(0, 0.3, ng).astype(np.float32)
    abi.check(lib.strelka_nrc_set_params(h, None, grid.ctypes.data))
    rec = records(n, 8)
    gm = np.zeros(nm, np.float32)
    gg = np.zeros(ng, np.float32)
    loss = C.c_float()
    abi.check(lib.strelka_nrc_gradients(h, to_device(rec).data_ptr(), n, gm.ctypes.data, gg.ctypes.data,
                                        C.byref(loss), None))
    rm, rg, rloss = nrc_ref.gradients(rec, mlp, grid, BMIN, BMAX, LOG2_T)
    assert abs(loss.value - rloss) <= 1e-3 * abs(rloss)
    a, b = gm.astype(np.float64), rm
    assert np.linalg.norm(a - b) <= 3e-2 * np.linalg.norm(b)
    assert np.linalg.norm(gg - rg) <= 3e-2 * np.linalg.norm(rg)
    status = C.c_uint32(1)
    abi.check(lib.strelka_nrc_get_device_status(h, None, C.byref(status)))
    assert status.value == 0
    lib.strelka_nrc_destroy(h)
