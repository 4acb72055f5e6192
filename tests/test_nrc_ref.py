"""The CPU reference of the radiance cache checks itself: its backward pass
against central finite differences of its own forward pass (exact mode, FP64,
stop-gradient denominator held fixed), and its encoding's invariants."""
import numpy as np

from oracle import nrc_ref

LOG2_T = 10
BMIN = np.array([0.0, 0.0, 0.0], np.float32)
BMAX = np.array([1.0, 1.0, 1.0], np.float32)


def _records(n, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 16), np.float32)
    r[:, 0:3] = rng.uniform(0, 1, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 6:9] = r[:, 3:6]
    r[:, 9] = 0.5
    r[:, 10:13] = rng.uniform(0.5, 2.0, (n, 3))
    return r


def _loss_fixed_den(rec, mlp, grid, den):
    x, _ = nrc_ref.encode(rec, grid, BMIN, BMAX, LOG2_T)
    y, _ = nrc_ref.forward(x, mlp, exact=True)
    return float(np.sum((y - rec[:, 10:13]) ** 2 / den))


def test_mlp_gradient_finite_differences():
    rng = np.random.default_rng(0)
    T = 1 << LOG2_T
    mlp = rng.normal(0, 0.2, nrc_ref.PARAMS)
    mlp[4 * 4096 + 3 * 64:] = 0.0
    grid = rng.normal(0, 0.5, 16 * T * 2)
    rec = _records(64, 1)
    g, _, _ = nrc_ref.gradients(rec, mlp, grid, BMIN, BMAX, LOG2_T, exact=True)
    x, _ = nrc_ref.encode(rec, grid, BMIN, BMAX, LOG2_T)
    y, _ = nrc_ref.forward(x, mlp, exact=True)
    den = y * y + 0.01
    for i in rng.choice(4 * 4096 + 192, 40, replace=False):
        e = np.zeros_like(mlp)
        e[i] = 1e-5
        fd = (_loss_fixed_den(rec, mlp + e, grid, den) - _loss_fixed_den(rec, mlp - e, grid, den)) / 2e-5
        assert abs(fd - g[i]) <= 1e-4 * max(1.0, abs(fd)), (i, fd, g[i])


def test_encoding_partition_of_unity():
    T, res, dense = nrc_ref.level_table(19)
    assert res[0] == 16 and res[15] == int(np.floor(16 * 1.5 ** 15))
    assert dense[0] and not dense[15]
    pn = np.random.default_rng(2).uniform(0, 1, (100, 3)).astype(np.float32)
    for l in (0, 7, 15):
        idx, w = nrc_ref.corners(pn, l, res, dense, T)
        assert np.allclose(w.sum(1), 1.0, atol=1e-6)
        assert (idx >= l * T).all() and (idx < (l + 1) * T).all()
