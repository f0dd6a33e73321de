"""The wavefront integrator (vt_render_wavefront) against the megakernel (vt_render) on the B200.

Both draw the same numbers from the same samplers and run the same device functions per vertex; the
wavefront's traversals are the persistent quantised-node kernels of traverse.cu (the megakernel
walks the 128-byte nodes), whose closest hit can differ only between triangles hit at exactly the
same distance. So the images agree pixel for pixel to FP64 summation order except on a handful of
pixels, and their means to well within the estimator's noise:
* Cornell box, spectral and RGB, sampling modes 1-3;
* the OpenPBR Cornell box (spectral), an imported scene under its light tree and an open scene with
  the procedural sky (shadow rays with the endpoint slack, MIS-weighted escapes);
* several passes (more samples than one pass's 4M paths hold) and a strided frame.
"""
import numpy as np
import pytest

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import scenes, spectral_tables

pytestmark = pytest.mark.gpu


def both(ctx, mesh, mats, light, params, spp, spectral, env=None):
    out = []
    for wavefront in (False, True):
        scene = vt.Scene(ctx, mesh, mats, light, spectral_tables.load() if spectral else None)
        if env:
            scene.set_environment(**env)
        (scene.render_wavefront if wavefront else scene.render)(params, spp)
        img, n = scene.readback()
        scene.close()
        assert n == spp and np.isfinite(img).all()
        out.append(img)
    return out


def assert_same(mega, wave, frac=0.995):
    same = np.all(np.abs(wave - mega) <= 1e-6 * np.maximum(np.abs(mega), 1e-3), axis=-1)
    assert same.mean() >= frac, same.mean()
    gm, wm = mega.reshape(-1, 3).mean(0), wave.reshape(-1, 3).mean(0)
    assert np.all(np.abs(wm / gm - 1) < 2e-3), (wm, gm)


@pytest.fixture(scope="module")
def cornell(ctx):
    faces, verts, mats, light, cam = scenes.cornell_box()
    mesh = vt.Mesh(ctx, faces, verts)
    yield mats, light, cam, mesh
    mesh.close()


@pytest.mark.parametrize("spectral,mode", [(True, 1), (False, 1), (True, 2), (True, 3)])
def test_cornell_equals_megakernel(ctx, cornell, spectral, mode):
    mats, light, cam, mesh = cornell
    mega, wave = both(ctx, mesh, mats, light, vt.make_params(cam, 96, 64, 8, 1, spectral, mode), 16, spectral)
    assert_same(mega, wave)


def test_openpbr_and_imported_scenes_equal_megakernel(ctx):
    faces, verts, mats, light, cam = scenes.cornell_openpbr()
    mesh = vt.Mesh(ctx, faces, verts)
    assert_same(*both(ctx, mesh, mats, light, vt.make_params(cam, 64, 64, 8, 1, True, 1), 16, True))
    mesh.close()
    faces, verts, mats, cam = scenes.cornell_emitters()
    mesh = vt.Mesh(ctx, faces, verts)
    assert_same(*both(ctx, mesh, mats, None, vt.make_params(cam, 64, 48, 8, 1, True, 1), 16, True))
    mesh.close()
    faces, verts, mats, cam = scenes.sky_scene(emitter=True)
    mesh = vt.Mesh(ctx, faces, verts)
    env = {"intensity": 1.0, "sun_dir": (0.4, 0.6, -0.5), "sun_intensity": 30.0, "sky_mode": 0}
    assert_same(*both(ctx, mesh, mats, None, vt.make_params(cam, 64, 64, 8, 1, True, 1), 16, True, env))
    mesh.close()


def test_passes_and_stride(ctx, cornell):
    mats, light, cam, mesh = cornell
    # 1024 x 1024 x 8 spp = 8M paths: two passes of 4M.
    mega, wave = both(ctx, mesh, mats, light, vt.make_params(cam, 1024, 1024, 4, 1, False, 1), 8, False)
    assert_same(mega, wave)
    mega, wave = both(ctx, mesh, mats, light, vt.make_params(cam, 96, 64, 8, 1, True, 1, pixel_stride=3), 8, True)
    assert_same(mega, wave)


def test_rejects_restir(ctx, cornell):
    mats, light, cam, mesh = cornell
    scene = vt.Scene(ctx, mesh, mats, light, None)
    with pytest.raises(vt.MaterialLibraryError, match="sampling modes 1-3"):
        scene.render_wavefront(vt.make_params(cam, 16, 16, 8, 1, False, 0), 1)
    scene.close()
