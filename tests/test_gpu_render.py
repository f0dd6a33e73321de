"""GPU path tracer against the FP64 oracle on the Cornell box.

Both consume the reference's PCG stream in the same order, so the GPU's fp32 paths follow the
oracle's fp64 paths except where rounding flips a discrete decision (a triangle edge, a roulette
threshold). The bars:
* mean radiance within 0.1 % per channel;
* per-pixel relMSE(GPU, oracle) far below the estimator's own: below a quarter of the relMSE
  between two independent oracle renders (different sample indices);
* most pixels identical to 1e-4 relative.
"""
import numpy as np
import pytest

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import scenes, spectral_tables

pytestmark = pytest.mark.gpu

MEAN_REL = 1e-3


def relmse(a, b):
    return float(np.mean((a - b) ** 2 / (b ** 2 + 1e-2)))


@pytest.fixture(scope="module")
def cornell(ctx):
    faces, verts, mats, light, cam = scenes.cornell_box()
    mesh = vt.Mesh(ctx, faces, verts)
    return faces, verts, mats, light, cam, mesh


def gpu_render(ctx, cornell, width, height, spp, spectral, depth=8, first=1, mode=1):
    faces, verts, mats, light, cam, mesh = cornell
    tables = spectral_tables.load() if spectral else None
    scene = vt.Scene(ctx, mesh, mats, light, tables)
    scene.render(vt.make_params(cam, width, height, depth, first, spectral, mode), spp)
    img, n = scene.readback()
    scene.close()
    assert n == spp
    return img


@pytest.mark.parametrize("spectral", [True, False])
def test_cornell_c1_matches_oracle(ctx, oracle, cornell, spectral):
    faces, verts, mats, light, cam, mesh = cornell
    tables = spectral_tables.load() if spectral else None
    gpu = gpu_render(ctx, cornell, 256, 256, 16, spectral)
    ref = oracle.render(faces, verts, mats, light, cam, 256, 256, 16, spectral=tables)
    other = oracle.render(faces, verts, mats, light, cam, 256, 256, 16, first_sample=1001, spectral=tables)
    gm, rm = gpu.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(gm / rm - 1) < MEAN_REL), (gm, rm)
    noise = relmse(other, ref)
    assert relmse(gpu, ref) < 0.25 * noise, (relmse(gpu, ref), noise)
    same = np.all(np.abs(gpu - ref) <= 1e-4 * np.maximum(np.abs(ref), 1e-3), axis=-1)
    assert same.mean() > 0.9, same.mean()
    assert np.isfinite(gpu).all()


@pytest.mark.parametrize("mode", [2, 3])
def test_sampling_modes_match_oracle_and_energy(ctx, oracle, cornell, mode):
    faces, verts, mats, light, cam, mesh = cornell
    gpu = gpu_render(ctx, cornell, 48, 32, 256, False, depth=3, mode=mode)
    ref = oracle.render(faces, verts, mats, light, cam, 48, 32, 256, max_depth=3, mode=mode)
    assert abs(gpu.mean() / ref.mean() - 1) < MEAN_REL
    mis = gpu_render(ctx, cornell, 48, 32, 256, False, depth=3, mode=1)
    assert abs(gpu.mean() / mis.mean() - 1) < (0.03 if mode == 2 else 0.12)


def test_accumulation_reset_and_resize(ctx, cornell):
    faces, verts, mats, light, cam, mesh = cornell
    scene = vt.Scene(ctx, mesh, mats, light, spectral_tables.load())
    scene.render(vt.make_params(cam, 64, 48, 8, 1, True), 4)
    scene.render(vt.make_params(cam, 64, 48, 8, 5, True), 4)
    a, n = scene.readback()
    assert n == 8
    b = gpu_render(ctx, cornell, 64, 48, 8, True)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    scene.reset()
    z, n = scene.readback()
    assert n == 0 and not z.any()
    scene.render(vt.make_params(cam, 32, 32, 8, 1, True), 2)   # a resize starts a new accumulation
    c, n = scene.readback()
    assert c.shape == (32, 32, 3) and n == 2
    scene.close()


def test_render_rejects_unsupported_input(ctx, cornell):
    faces, verts, mats, light, cam, mesh = cornell
    coloured = [dict(m) for m in mats]
    coloured[3] = {"type": 0, "albedo": (0.65, 0.05, 0.05), "emission": (0, 0, 0)}
    tables = spectral_tables.load()
    with pytest.raises(vt.MaterialLibraryError, match="colour model"):
        vt.Scene(ctx, mesh, coloured, light, dict(tables, uplift_w=np.zeros((1, 3)), uplift_cos=np.zeros(1)))
    scene = vt.Scene(ctx, mesh, coloured, light)   # RGB transport needs no tables
    with pytest.raises(vt.MaterialLibraryError, match="sampling_mode"):
        scene.render(vt.make_params(cam, 8, 8, 8, 1, False, mode=4), 1)
    with pytest.raises(vt.MaterialLibraryError, match="spectral tables"):
        scene.render(vt.make_params(cam, 8, 8, 8, 1, True), 1)
    scene.close()


@pytest.mark.parametrize("model", [0, 3])
def test_cornell_z_sampler_matches_oracle(ctx, oracle, cornell, model):
    faces, verts, mats, light, cam, mesh = cornell
    tables = spectral_tables.load()
    scene = vt.Scene(ctx, mesh, mats, light, tables)
    scene.render(vt.make_params(cam, 128, 128, 8, 1, True, sampler=1, z_temporal=model), 16)
    gpu, n = scene.readback()
    scene.close()
    ref = oracle.render(faces, verts, mats, light, cam, 128, 128, 16, spectral=tables, sampler=1, z_temporal=model)
    assert np.all(np.abs(gpu.reshape(-1, 3).mean(0) / ref.reshape(-1, 3).mean(0) - 1) < MEAN_REL)
    same = np.all(np.abs(gpu - ref) <= 1e-4 * np.maximum(np.abs(ref), 1e-3), axis=-1)
    assert same.mean() > 0.9, same.mean()
    # Z++ and PCG estimate the same image.
    pcg = oracle.render(faces, verts, mats, light, cam, 128, 128, 16, spectral=tables)
    assert abs(gpu.mean() / pcg.mean() - 1) < 0.02


def _parity(gpu, ref, other, same_frac=0.9):
    gm, rm = gpu.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(gm / rm - 1) < MEAN_REL), (gm, rm)
    assert relmse(gpu, ref) < 0.25 * relmse(other, ref), (relmse(gpu, ref), relmse(other, ref))
    same = np.all(np.abs(gpu - ref) <= 1e-4 * np.maximum(np.abs(ref), 1e-3), axis=-1)
    assert same.mean() > same_frac, same.mean()


@pytest.mark.parametrize("spectral", [False, True])
def test_thin_lens_matches_oracle(ctx, oracle, cornell, spectral):
    """lens_ray (main.swift:2210-2216): aperture 0.05, focus on the tall box."""
    faces, verts, mats, light, cam, mesh = cornell
    tables = spectral_tables.load() if spectral else None
    scene = vt.Scene(ctx, mesh, mats, light, tables)
    scene.render(vt.make_params(cam, 128, 128, 8, 1, spectral, aperture=0.05, focus_distance=3.0), 16)
    gpu, _ = scene.readback()
    scene.close()
    kw = dict(spectral=tables, aperture=0.05, focus_distance=3.0)
    ref = oracle.render(faces, verts, mats, light, cam, 128, 128, 16, **kw)
    other = oracle.render(faces, verts, mats, light, cam, 128, 128, 16, first_sample=1001, **kw)
    _parity(gpu, ref, other)
    pinhole = oracle.render(faces, verts, mats, light, cam, 128, 128, 16, spectral=tables)
    assert (np.abs(ref - pinhole).max(-1) > 0).mean() > 0.5   # the lens draws change the paths


@pytest.mark.parametrize("mode", [1, 0])
def test_smooth_normals_match_oracle(ctx, oracle, mode):
    """mesh_hit_attributes (main.swift:1587-1602): shading with interpolated vertex normals."""
    faces, verts, mats, light, cam = scenes.cornell_sphere()
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, light)
    scene.render(vt.make_params(cam, 128, 128, 8, 1, False, mode), 16)
    gpu, _ = scene.readback()
    scene.close()
    mesh.close()
    ref = oracle.render(faces, verts, mats, light, cam, 128, 128, 16, mode=mode)
    other = oracle.render(faces, verts, mats, light, cam, 128, 128, 16, first_sample=1001, mode=mode)
    gm, rm = gpu.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(gm / rm - 1) < (MEAN_REL if mode else 5e-3)), (gm, rm)
    assert relmse(gpu, ref) < (0.25 if mode else 1.0) * relmse(other, ref), (relmse(gpu, ref), relmse(other, ref))


@pytest.mark.parametrize("stride", [3, 8])
def test_pixel_stride_renders_the_frames_own_pixels(ctx, cornell, stride):
    """A strided render (vt_frame_params.pixel_stride) is the full frame's pixels (s i, s j): the same
    camera rays and sample streams, so the same FP64 sums up to summation order."""
    faces, verts, mats, light, cam, mesh = cornell
    tables = spectral_tables.load()
    full = gpu_render(ctx, cornell, 64, 48, 8, True)
    scene = vt.Scene(ctx, mesh, mats, light, tables)
    scene.render(vt.make_params(cam, 64, 48, 8, 1, True, 1, pixel_stride=stride), 8)
    img, n = scene.readback()
    assert n == 8 and img.shape == (-(-48 // stride), -(-64 // stride), 3)
    np.testing.assert_allclose(img, full[::stride, ::stride], rtol=1e-12, atol=1e-15)
    with pytest.raises(vt.MaterialLibraryError, match="pixel stride"):
        scene.render(vt.make_params(cam, 64, 48, 8, 1, True, 0, pixel_stride=stride), 1)
    scene.close()


def test_accumulation_save_and_restore_continue_a_render(ctx, cornell, tmp_path):
    """A render taken in two pieces through save_accumulation / restore_accumulation (vt_accum_restore)
    equals the same render in one piece: the FP64 sums and the sample count carry over."""
    faces, verts, mats, light, cam, mesh = cornell
    tables = spectral_tables.load()
    whole = gpu_render(ctx, cornell, 48, 48, 16, True)
    a = vt.Scene(ctx, mesh, mats, light, tables)
    p = vt.make_params(cam, 48, 48, 8, 1, True, 1, pixel_stride=2)
    a.render(p, 8)
    assert a.save_accumulation(tmp_path / "acc.npz", p) == 8
    a.close()
    b = vt.Scene(ctx, mesh, mats, light, tables)
    assert b.restore_accumulation(tmp_path / "acc.npz") == 8
    b.render(vt.make_params(cam, 48, 48, 8, 9, True, 1, pixel_stride=2), 8)
    img, n = b.readback()
    b.close()
    assert n == 16
    np.testing.assert_allclose(img, whole[::2, ::2], rtol=1e-12, atol=1e-15)
