"""The radiance cache on the device (nrc.cu, vt_render_nrc) against its CPU restatement
(oracle/nrc_ref.py), which rounds to fp16 where the kernels do and sums exactly where they
accumulate in fp32:
* inference: predictions within 5e-3 of the output range (fp16 ties may round apart);
* gradients: the weight and grid gradient sums within 1 % of each layer's largest, on records
  whose ReLUs are clear of zero;
* training: Adam on a smooth target cuts the loss tenfold;
* rendering: a trained cache's Cornell image (ReSTIR DI and MIS primaries, spectral) within 3 % of
  the plain path tracer's mean radiance, the cache's own bias being what the bound covers.
The reference has no radiance cache, so these parity bounds are against the restatement only."""
import numpy as np
import pytest

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import scenes, spectral_tables
from metal_vibe_tracer_b200.nrc import RadianceCache
from oracle import nrc_ref as R

pytestmark = pytest.mark.gpu


def random_inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 13), np.float32)
    x[:, 0:3] = rng.uniform(-0.95, 0.95, (n, 3))
    x[:, 3] = rng.uniform(0, 2, n)
    x[:, 4:8] = rng.uniform(0, 1, (n, 4))
    x[:, 8:11] = rng.uniform(0, 1, (n, 3))
    x[:, 11] = rng.uniform(0, 1, n)
    x[:, 12] = rng.uniform(0, 1, n)
    return x


def cache_with_params(ctx, seed, levels=8, log_t=14, spectral=False):
    cache = RadianceCache(ctx, [-1, -1, -1], [1, 1, 1], levels=levels, log2_table=log_t, base_resolution=8,
                          max_resolution=256, seed=seed, spectral=int(spectral))
    rng = np.random.default_rng(seed)
    mlp = np.zeros(R.MLP_PARAMS, np.float32)
    mlp[:R.HIDDEN * 4096] = rng.uniform(-0.25, 0.25, R.HIDDEN * 4096)
    mlp[R.HIDDEN * 4096:R.HIDDEN * 4096 + 4 * 64] = rng.uniform(-0.25, 0.25, 4 * 64)
    table = rng.uniform(-1, 1, cache.grid_params).astype(np.float32)
    cache.set_params(mlp, table)
    grid = R.Grid(levels, log_t, 8, 256, [-1, -1, -1], [1, 1, 1])
    return cache, grid, mlp, table.reshape(levels, 1 << log_t, 2)


def test_infer_matches_oracle(ctx):
    cache, grid, mlp, table = cache_with_params(ctx, 5)
    x = random_inputs(1000, 6)
    got = cache.infer(x)
    ref = R.predict(x, mlp, table, grid)
    scale = np.abs(ref).max()
    assert scale > 0.05
    err = np.abs(got - ref)
    assert err.max() <= 5e-3 * scale + 1e-5, (err.max(), scale)
    assert np.median(err) <= 1e-3 * scale
    cache.close()


@pytest.mark.parametrize("spectral", [False, True])
def test_gradients_match_oracle(ctx, spectral):
    cache, grid, mlp, table = cache_with_params(ctx, 7, spectral=spectral)
    x = random_inputs(2000, 8)
    # Records whose ReLUs are all clear of zero (a flipped ReLU changes a record's gradient).
    x = x[R.relu_margins(x, mlp, table, grid) > 5e-4][:1000]  # not a multiple of the 128-row tile
    assert len(x) == 1000
    y = np.random.default_rng(9).uniform(0, 2, (1000, 4)).astype(np.float32)
    gm, gg, loss = cache.gradients(x, y)
    rm, rg, rloss = R.gradients(x, y, mlp, table, grid, spectral=spectral)
    assert loss == pytest.approx(rloss, rel=2e-3)
    for l in range(R.HIDDEN + 1):
        a = gm[l * 4096:(l + 1) * 4096] if l < R.HIDDEN else gm[R.HIDDEN * 4096:]
        b = rm[l * 4096:(l + 1) * 4096] if l < R.HIDDEN else rm[R.HIDDEN * 4096:]
        assert np.abs(a - b).max() <= 1e-2 * np.abs(b).max(), (l, np.abs(a - b).max(), np.abs(b).max())
    assert np.all(gm[R.HIDDEN * 4096 + 4 * 64:] == 0.0)  # unused output rows
    rg = rg.ravel()
    assert np.abs(gg - rg).max() <= 1e-2 * np.abs(rg).max(), np.abs(gg - rg).max()
    assert np.count_nonzero(gg) > 0
    cache.close()


def test_training_fits_a_smooth_target(ctx):
    cache = RadianceCache(ctx, [-1, -1, -1], [1, 1, 1], log2_table=16, seed=11, learning_rate=5e-3)
    x = random_inputs(8192, 12)
    p = x[:, 0:3]
    y = np.stack([0.6 + 0.4 * np.sin(3 * p[:, 0]), 0.5 + 0.3 * np.cos(2 * p[:, 1]), 0.4 + 0.2 * p[:, 2] * x[:, 8],
                  np.zeros(len(x))], 1)
    first = cache.train(x, y)
    last = first
    for _ in range(300):
        last = cache.train(x, y)
    info = cache.info()
    assert info["steps"] == 301 and info["last_records"] == 8192
    assert np.isfinite(last) and last < 0.1 * first, (first, last)
    pred = cache.infer(x)
    assert np.mean(np.abs(pred - y)) < 0.05
    cache.close()


@pytest.fixture(scope="module")
def cornell_scene(ctx):
    faces, verts, mats, light, cam = scenes.cornell_box()
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, light, spectral_tables.load())
    yield mesh, scene, cam
    scene.close()
    mesh.close()


@pytest.mark.parametrize("mode", [1, 0])
def test_cached_cornell_matches_path_tracer(ctx, cornell_scene, mode):
    mesh, scene, cam = cornell_scene
    W = H = 64
    scene.reset()
    scene.render(vt.make_params(cam, W, H, 8, 1, True, 1), 1024)
    ref, _ = scene.readback()
    info = mesh.info()
    cache = RadianceCache(ctx, list(info.lo), list(info.hi), train_records=16384, seed=21, spectral=1)
    scene.reset()
    for f in range(120):  # training frames only
        cache.render(scene, vt.make_params(cam, W, H, 8, 1 + f, True, mode), 0, render=False)
    ci = cache.info()
    assert ci["steps"] == 120 and ci["last_records"] > 1000 and np.isfinite(ci["last_loss"])
    scene.reset()
    for f in range(16):
        cache.render(scene, vt.make_params(cam, W, H, 8, 5001 + 16 * f, True, mode), 16)
    img, n = scene.readback()
    assert n == 256 and np.isfinite(img).all()
    gm, rm = img.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(gm / rm - 1) < 0.03), (gm, rm)
    cache.close()


def test_render_nrc_rejects_other_modes(ctx, cornell_scene):
    mesh, scene, cam = cornell_scene
    info = mesh.info()
    cache = RadianceCache(ctx, list(info.lo), list(info.hi), train_records=1024, spectral=1)
    with pytest.raises(vt.MaterialLibraryError, match="sampling modes 0"):
        cache.render(scene, vt.make_params(cam, 16, 16, 8, 1, True, 2), 1)
    with pytest.raises(vt.MaterialLibraryError, match="transport"):
        cache.render(scene, vt.make_params(cam, 16, 16, 8, 1, False, 1), 1)
    with pytest.raises(vt.MaterialLibraryError, match="whole frames"):
        cache.render(scene, vt.make_params(cam, 16, 16, 8, 1, True, 1, pixel_stride=2), 1)
    with pytest.raises(vt.MaterialLibraryError, match="spread"):
        RadianceCache(ctx, list(info.lo), list(info.hi), query_vertex=0, spread=0.0)
    cache.close()


def test_cached_openpbr_cornell(ctx):
    """The OpenPBR variants of the cache's kernels (training paths, cache-terminated paths with MIS and
    ReSTIR DI primaries): a trained cache's image of the OpenPBR Cornell box within 4 % of the path
    tracer's mean radiance."""
    faces, verts, mats, light, cam = scenes.cornell_openpbr()
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, light, spectral_tables.load())
    W = H = 64
    scene.render(vt.make_params(cam, W, H, 8, 1, True, 1), 1024)
    ref, _ = scene.readback()
    info = mesh.info()
    for mode in (1, 0):
        cache = RadianceCache(ctx, list(info.lo), list(info.hi), train_records=16384, seed=5, spectral=1)
        scene.reset()
        for f in range(120):
            cache.render(scene, vt.make_params(cam, W, H, 8, 1 + f, True, mode), 0, render=False)
        scene.reset()
        for f in range(16):
            cache.render(scene, vt.make_params(cam, W, H, 8, 7001 + 16 * f, True, mode), 16)
        img, n = scene.readback()
        assert n == 256 and np.isfinite(img).all()
        gm, rm = img.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
        assert np.all(np.abs(gm / rm - 1) < 0.04), (mode, gm, rm)
        cache.close()
    scene.close()
    mesh.close()
