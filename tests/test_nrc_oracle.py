"""The radiance cache's CPU restatement (oracle/nrc_ref.py) checked against itself: its analytic
gradients against finite differences of the loss (the exact, unrounded network), the hash grid's
corner selection and weights, and the encoding's fixed entries. The reference has no radiance
cache, so nothing pins the network to it; the device kernels are checked against this module by
tests/test_gpu_nrc.py."""
import numpy as np
import pytest

from oracle import nrc_ref as R


def random_case(n=12, levels=4, log_t=12, seed=0):
    rng = np.random.default_rng(seed)
    grid = R.Grid(levels, log_t, 4, 64, [-1, -1, -1], [1, 1, 1])
    x = np.zeros((n, 13), np.float32)
    x[:, 0:3] = rng.uniform(-0.9, 0.9, (n, 3))
    x[:, 3] = rng.uniform(0, 1, n)
    x[:, 4:8] = rng.uniform(0, 1, (n, 4))
    x[:, 8:11] = rng.uniform(0, 1, (n, 3))
    x[:, 11] = rng.uniform(0, 1, n)
    x[:, 12] = rng.uniform(0, 1, n)
    mlp = np.zeros(R.MLP_PARAMS)
    mlp[:R.HIDDEN * 4096] = rng.uniform(-0.3, 0.3, R.HIDDEN * 4096)
    mlp[R.HIDDEN * 4096:R.HIDDEN * 4096 + 4 * 64] = rng.uniform(-0.3, 0.3, 4 * 64)
    table = rng.uniform(-1, 1, (levels, grid.entries, 2))
    y = rng.uniform(0, 2, (n, 4))
    return grid, x, mlp, table, y


@pytest.mark.parametrize("spectral", [False, True])
def test_gradients_match_finite_differences(spectral):
    grid, x, mlp, table, y = random_case()
    gm, gt, loss = R.gradients(x, y, mlp, table, grid, exact=True, spectral=spectral)
    den = R.denominators(x, mlp, table, grid, spectral=spectral)
    assert loss == pytest.approx(R.loss_sum(x, y, mlp, table, grid, den), rel=1e-12)
    rng = np.random.default_rng(1)
    h = 1e-6
    picks = list(rng.choice(R.HIDDEN * 4096, 12, replace=False)) + list(R.HIDDEN * 4096 + rng.choice(4 * 64, 4, replace=False))
    for i in picks:
        mp, mm = mlp.copy(), mlp.copy()
        mp[i] += h
        mm[i] -= h
        fd = (R.loss_sum(x, y, mp, table, grid, den) - R.loss_sum(x, y, mm, table, grid, den)) / (2 * h)
        assert gm[i] == pytest.approx(fd, rel=1e-5, abs=1e-7), i
    # Grid entries that the records touch.
    idx, _ = grid.corners(x[:, 0:3], 2)
    for e in idx[:4, 3]:
        for f in range(2):
            tp, tm = table.copy(), table.copy()
            tp[2, e, f] += h
            tm[2, e, f] -= h
            fd = (R.loss_sum(x, y, mlp, tp, grid, den) - R.loss_sum(x, y, mlp, tm, grid, den)) / (2 * h)
            assert gt[2, e, f] == pytest.approx(fd, rel=1e-5, abs=1e-7)


def test_corners_dense_and_hashed():
    grid = R.Grid(3, 12, 4, 64, [0, 0, 0], [1, 1, 1])
    # Level 0 (4 cells, 5^3 = 125 points) is dense; level 2 (64 cells) is hashed.
    assert grid.res == [4, 16, 64]
    pos = np.array([[0.3, 0.6, 0.9]], np.float32)
    idx, w = grid.corners(pos, 0)
    q = (pos - grid.lo) * grid.inv
    c = np.floor(q * 4).astype(int)[0]
    assert idx[0, 0] == c[0] + 5 * (c[1] + 5 * c[2])
    assert w.sum() == pytest.approx(1.0, abs=1e-6)
    idx2, _ = grid.corners(pos, 2)
    g = np.floor(q * 64).astype(np.uint64)[0]
    h = (int(g[0]) * 1) ^ ((int(g[1]) * 2654435761) & 0xffffffff) ^ ((int(g[2]) * 805459861) & 0xffffffff)
    assert idx2[0, 0] == h & (grid.entries - 1)


def test_encoding_fixed_entries():
    grid, x, mlp, table, y = random_case(n=5)
    e = R.encode(x, table, grid)
    assert np.all(e[:, 63] == 1.0)
    # One-blob: the kernel of the bin holding s is the largest (direction, wavelength number).
    assert np.all(np.argmax(e[:, 32:36], 1) == np.minimum((x[:, 4] * 4).astype(int), 3))
    assert np.all(np.argmax(e[:, 56:60], 1) == np.minimum((x[:, 12] * 4).astype(int), 3))
    # The frequency encoding of the normalised position.
    q = grid.position(x[:, 0:3]).astype(np.float64)
    assert np.abs(e[:, 60:63] - np.sin(2 * np.pi * q)).max() < 1e-3
    # fp16 values.
    assert np.all(e.astype(np.float16).astype(np.float64) == e)


def test_loss_scale_keeps_small_gradients():
    """The backward pass's fp16 values carry the loss gradient times LOSS_SCALE. With targets within
    1e-6 of the (fp16) prediction, the per-record gradients fall into fp16's subnormal range: without
    the scale they lose most of their precision, with it they stay close to a run whose scale leaves
    every value normal."""
    grid, x, mlp, table, _ = random_case(n=64, seed=3)
    p = R.predict(x, mlp, table, grid)
    y = p + 1e-6 * np.random.default_rng(4).standard_normal(p.shape)
    ref, _, _ = R.gradients(x, y, mlp, table, grid, loss_scale=4096.0)
    scaled, _, _ = R.gradients(x, y, mlp, table, grid)
    unscaled, _, _ = R.gradients(x, y, mlp, table, grid, loss_scale=1.0)
    n = R.HIDDEN * 4096
    e_scaled = np.abs(scaled[:n] - ref[:n]).max()
    e_unscaled = np.abs(unscaled[:n] - ref[:n]).max()
    assert e_scaled < 0.02 * np.abs(ref[:n]).max() and e_scaled < 0.1 * e_unscaled, (e_scaled, e_unscaled)
