"""The procedural sky and sun of imported scenes (vt_scene_set_environment), and an environment image
(vt_scene_set_environment_map) with its compensated and original sampling tables, against the FP64 oracle,
which restates the same sky, sun-cone and cosine-lobe sampling and the MIS weights of escaped rays:
* images within 0.1 % of the oracle's mean radiance, most pixels identical to 1e-4, the per-pixel
  relMSE below a quarter of the estimator's own (as the other integrator parity tests);
* the estimator is consistent: light sampling only (mode 2) and BSDF sampling only (mode 3) agree
  with MIS (mode 1) in mean radiance, which holds only if the NEE density of the environment
  matches its sampling and escapes are weighed against it."""
import numpy as np
import pytest

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import scenes, spectral_tables

pytestmark = pytest.mark.gpu

MEAN_REL = 1e-3
SUN = {"intensity": 1.0, "sun_dir": (0.4, 0.6, -0.5), "sun_intensity": 30.0}


def relmse(a, b):
    return float(np.mean((a - b) ** 2 / (b ** 2 + 1e-2)))


def render(ctx, faces, verts, mats, cam, env, w, h, spp, spectral, mode=1, first=1):
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, None, spectral_tables.load() if spectral else None)
    scene.set_environment(**env)
    scene.render(vt.make_params(cam, w, h, 8, first, spectral, mode), spp)
    img, n = scene.readback()
    scene.close()
    mesh.close()
    assert n == spp and np.isfinite(img).all()
    return img


@pytest.mark.parametrize("emitter,spectral,sky", [(True, True, 0), (False, False, 1), (True, False, 2)])
def test_sky_scene_matches_oracle(ctx, oracle, emitter, spectral, sky):
    faces, verts, mats, cam = scenes.sky_scene(emitter=emitter)
    env = dict(SUN, sky_mode=sky)
    tables = spectral_tables.load() if spectral else None
    gpu = render(ctx, faces, verts, mats, cam, env, 96, 96, 16, spectral)
    ref = oracle.render(faces, verts, mats, None, cam, 96, 96, 16, spectral=tables, environment=env)
    other = oracle.render(faces, verts, mats, None, cam, 96, 96, 16, first_sample=1001, spectral=tables,
                          environment=env)
    gm, rm = gpu.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(gm / rm - 1) < MEAN_REL), (gm, rm)
    assert relmse(gpu, ref) < 0.25 * relmse(other, ref), (relmse(gpu, ref), relmse(other, ref))
    same = np.all(np.abs(gpu - ref) <= 1e-4 * np.maximum(np.abs(ref), 1e-3), axis=-1)
    assert same.mean() > 0.9, same.mean()


def test_light_and_bsdf_sampling_agree_with_mis(ctx):
    faces, verts, mats, cam = scenes.sky_scene(emitter=True)
    env = dict(SUN, sky_mode=1)
    # The sky seen directly and through one bounce: depth 2, so every estimator sums the same terms.
    means = {}
    for mode in (1, 2, 3):
        mesh = vt.Mesh(ctx, faces, verts)
        scene = vt.Scene(ctx, mesh, mats, None, None)
        scene.set_environment(**env)
        scene.render(vt.make_params(cam, 64, 64, 2, 1, False, mode), 1024)
        img, _ = scene.readback()
        scene.close()
        mesh.close()
        means[mode] = img.reshape(-1, 3).mean(0)
    assert np.all(np.abs(means[2] / means[1] - 1) < 0.02), means
    assert np.all(np.abs(means[3] / means[1] - 1) < 0.03), means


def test_environment_rejections(ctx):
    faces, verts, mats, cam = scenes.sky_scene(emitter=True)
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, None, None)
    scene.set_environment(**SUN)
    with pytest.raises(vt.MaterialLibraryError, match="sampling mode 0"):
        scene.render(vt.make_params(cam, 16, 16, 8, 1, False, 0), 1)
    with pytest.raises(vt.MaterialLibraryError, match="sky_mode"):
        scene.set_environment(intensity=1.0, sky_mode=3)
    scene.set_environment()  # removed: ReSTIR DI renders again
    scene.render(vt.make_params(cam, 16, 16, 8, 1, False, 0), 1)
    scene.close()
    cf, cv, cm, light, ccam = scenes.cornell_box()
    cmesh = vt.Mesh(ctx, cf, cv)
    quad = vt.Scene(ctx, cmesh, cm, light, None)
    with pytest.raises(vt.MaterialLibraryError, match="imported scene"):
        quad.set_environment(**SUN)
    quad.close()
    cmesh.close()
    mesh.close()


def test_batched_sky_scene_equals_single_render(ctx):
    """A scene with an environment in a batch (one persistent launch, then the captured graph) adds
    exactly the samples vt_render adds, beside a scene without one."""
    from metal_vibe_tracer_b200.render import Batch
    faces, verts, mats, cam = scenes.sky_scene(emitter=True)
    mesh = vt.Mesh(ctx, faces, verts)
    tables = spectral_tables.load()
    cf, cv, cm, light, ccam = scenes.cornell_box()
    cmesh = vt.Mesh(ctx, cf, cv)

    def make_sky():
        s = vt.Scene(ctx, mesh, mats, None, tables)
        s.set_environment(**dict(SUN, sky_mode=2))
        return s

    specs = [(make_sky, vt.make_params(cam, 48, 40, 8, 1, True, 1), 2),
             (lambda: vt.Scene(ctx, cmesh, cm, light), vt.make_params(ccam, 32, 32, 6, 1, False, 2), 3)]
    members = [make() for make, _, _ in specs]
    batch = Batch(ctx, members, [p for _, p, _ in specs], [s for _, _, s in specs])
    passes = 7
    for _ in range(passes):
        batch.render()
    for scene, (make, params, spp) in zip(members, specs):
        img, n = scene.readback()
        ref_scene = make()
        ref_scene.render(params, passes * spp)
        ref, m = ref_scene.readback()
        ref_scene.close()
        assert n == m == passes * spp and np.isfinite(img).all() and img.max() > 0
        np.testing.assert_allclose(img, ref, rtol=1e-12, atol=1e-12)
    batch.close()
    for s in members:
        s.close()
    cmesh.close()
    mesh.close()


def test_cached_sky_scene_matches_path_tracer(ctx):
    """The radiance cache on an open scene: training paths and cache-terminated paths that escape
    pick up the sky (MIS primaries, spectral). A trained cache's image within 4 % of the path
    tracer's mean radiance, the cache's own bias being what the bound covers."""
    from metal_vibe_tracer_b200.nrc import RadianceCache
    faces, verts, mats, cam = scenes.sky_scene(emitter=True)
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, None, spectral_tables.load())
    scene.set_environment(**dict(SUN, sky_mode=0))
    W = H = 64
    scene.render(vt.make_params(cam, W, H, 8, 1, True, 1), 1024)
    ref, _ = scene.readback()
    info = mesh.info()
    cache = RadianceCache(ctx, list(info.lo), list(info.hi), train_records=16384, seed=13, spectral=1)
    scene.reset()
    for f in range(120):
        cache.render(scene, vt.make_params(cam, W, H, 8, 1 + f, True, 1), 0, render=False)
    ci = cache.info()
    assert ci["last_records"] > 1000 and np.isfinite(ci["last_loss"])
    scene.reset()
    for f in range(16):
        cache.render(scene, vt.make_params(cam, W, H, 8, 9001 + 16 * f, True, 1), 16)
    img, n = scene.readback()
    assert n == 256 and np.isfinite(img).all()
    gm, rm = img.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(gm / rm - 1) < 0.04), (gm, rm)
    with pytest.raises(vt.MaterialLibraryError, match="sampling mode 0"):
        cache.render(scene, vt.make_params(cam, W, H, 8, 1, True, 0), 1)
    cache.close()
    scene.close()
    mesh.close()


def render_image_env(ctx, faces, verts, mats, cam, img, w, h, spp, spectral, mode=1, depth=8, wavefront=False,
                     rotation=0.7):
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, None, spectral_tables.load() if spectral else None)
    scene.set_environment_map(img, intensity=1.0, rotation=rotation)
    (scene.render_wavefront if wavefront else scene.render)(vt.make_params(cam, w, h, depth, 1, spectral, mode), spp)
    out, n = scene.readback()
    scene.close()
    mesh.close()
    assert n == spp and np.isfinite(out).all()
    return out


@pytest.mark.parametrize("emitter,spectral", [(True, True), (False, False)])
def test_image_environment_matches_oracle(ctx, oracle, emitter, spectral):
    """The image lookup (bilinear, rotated), the two sampling tables and the escaped rays' MIS weights
    against the oracle's double restatement (its tables built in double, so cells and densities
    differ at float rounding: the comparison is the mean and the per-pixel error against the
    estimator's own)."""
    faces, verts, mats, cam = scenes.sky_scene(emitter=emitter)
    img = scenes.environment_image(64, 32)
    tables = spectral_tables.load() if spectral else None
    gpu = render_image_env(ctx, faces, verts, mats, cam, img, 96, 96, 16, spectral)
    env = {"intensity": 1.0, "image": img, "rotation": 0.7}
    ref = oracle.render(faces, verts, mats, None, cam, 96, 96, 16, spectral=tables, environment=env)
    other = oracle.render(faces, verts, mats, None, cam, 96, 96, 16, first_sample=1001, spectral=tables,
                          environment=env)
    gm, rm = gpu.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(gm / rm - 1) < 5e-3), (gm, rm)
    assert relmse(gpu, ref) < 0.5 * relmse(other, ref), (relmse(gpu, ref), relmse(other, ref))


def test_image_light_and_bsdf_sampling_agree_with_mis(ctx):
    """Light sampling only (mode 2, the compensated table where a BSDF continuation follows, whose
    zero-density directions the BSDF hits then carry with full weight) and BSDF sampling only
    (mode 3) agree with MIS (mode 1) in mean radiance."""
    faces, verts, mats, cam = scenes.sky_scene(emitter=True)
    img = scenes.environment_image(64, 32)
    means = {m: render_image_env(ctx, faces, verts, mats, cam, img, 64, 64, 1024, False, mode=m, depth=2)
             .reshape(-1, 3).mean(0) for m in (1, 2, 3)}
    assert np.all(np.abs(means[2] / means[1] - 1) < 0.02), means
    assert np.all(np.abs(means[3] / means[1] - 1) < 0.03), means


def test_image_environment_wavefront_equals_megakernel(ctx):
    faces, verts, mats, cam = scenes.sky_scene(emitter=True)
    img = scenes.environment_image(64, 32)
    mega = render_image_env(ctx, faces, verts, mats, cam, img, 64, 64, 16, True)
    wave = render_image_env(ctx, faces, verts, mats, cam, img, 64, 64, 16, True, wavefront=True)
    same = np.all(np.abs(wave - mega) <= 1e-6 * np.maximum(np.abs(mega), 1e-3), axis=-1)
    assert same.mean() >= 0.995, same.mean()


def test_image_environment_rejections(ctx):
    faces, verts, mats, cam = scenes.sky_scene(emitter=True)
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, None, None)
    bad = scenes.environment_image(16, 8)
    bad[3, 4, 0] = np.nan
    with pytest.raises(vt.MaterialLibraryError, match="finite"):
        scene.set_environment_map(bad)
    with pytest.raises(vt.MaterialLibraryError, match="16384"):
        scene.set_environment_map(np.ones((8193, 1, 4), np.float32))
    scene.set_environment_map(scenes.environment_image(16, 8))
    with pytest.raises(vt.MaterialLibraryError, match="sampling mode 0"):
        scene.render(vt.make_params(cam, 16, 16, 8, 1, False, 0), 1)
    scene.set_environment_map(None)
    scene.render(vt.make_params(cam, 16, 16, 8, 1, False, 0), 1)
    scene.close()
    mesh.close()
