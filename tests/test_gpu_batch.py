"""Batched scenes (config C4): one persistent launch per pass over many scenes, tuned and then
replayed as a captured CUDA graph.

A batch pass must add exactly the samples a vt_render call of the same frames adds: the same per
sample paths (the device-side frame jitter equals the host's), accumulated in FP64. The first six
passes try the launch shapes and the seventh onwards replays the graph; the per-scene completion
times lie within the pass.
"""
import numpy as np
import pytest

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import scenes, spectral_tables
from metal_vibe_tracer_b200.render import Batch

pytestmark = pytest.mark.gpu


def scene_specs(ctx):
    """(make_scene, params, spp) per batch member; make_scene builds a fresh, equivalent scene."""
    faces, verts, mats, light, cam = scenes.cornell_box()
    cornell = vt.Mesh(ctx, faces, verts)
    tables = spectral_tables.load()
    f2, v2, m2, c2 = scenes.sphere_grid(20_000, seed=3)
    grid = vt.Mesh(ctx, f2, v2)
    return [
        (lambda: vt.Scene(ctx, cornell, mats, light), vt.make_params(cam, 64, 48, 6, 1, False), 3),
        (lambda: vt.Scene(ctx, cornell, mats, light, tables), vt.make_params(cam, 40, 40, 8, 1, True), 2),
        (lambda: vt.Scene(ctx, grid, m2, None), vt.make_params(c2, 56, 32, 8, 1, False, mode=2), 4),
        (lambda: vt.Scene(ctx, grid, m2, None, light_tree=False), vt.make_params(c2, 24, 24, 5, 7, False), 1),
    ], (cornell, grid)


def test_batch_equals_single_renders(ctx):
    specs, meshes = scene_specs(ctx)
    batch_scenes = [make() for make, _, _ in specs]
    batch = Batch(ctx, batch_scenes, [p for _, p, _ in specs], [s for _, _, s in specs])
    passes = 8
    for k in range(passes):
        ms_pass = batch.render()
        st, ms = batch.stats()
        assert st.passes == k + 1 and st.tuned == (1 if k >= 5 else 0)
        assert st.items == sum(p.width * p.height for _, p, _ in specs)
        assert ms_pass > 0 and np.all(ms > 0) and np.all(ms <= ms_pass * 1.05 + 0.05), (ms, ms_pass)
    for scene, (make, params, spp) in zip(batch_scenes, specs):
        img, n = scene.readback()
        assert n == passes * spp
        ref_scene = make()
        ref_scene.render(params, passes * spp)
        ref, m = ref_scene.readback()
        ref_scene.close()
        assert m == n
        assert np.isfinite(img).all() and img.max() > 0
        # The same samples summed in another order (per pass, then across passes).
        np.testing.assert_allclose(img, ref, rtol=1e-12, atol=1e-12)
    batch.close()
    for sc in batch_scenes:
        sc.close()
    for m in meshes:
        m.close()


def test_batch_wavefront_equals_single_renders(ctx):
    """vt_batch_render_wavefront: per-scene queues on four streams; the first eight passes try queue
    size x block size x compaction frequency (every bounce, every second bounce with ended paths kept
    in place), and every pass adds exactly the samples vt_render_wavefront of the same frames adds (the
    same paths; only the FP64 summation order of the accumulation differs)."""
    specs, meshes = scene_specs(ctx)
    batch_scenes = [make() for make, _, _ in specs]
    batch = Batch(ctx, batch_scenes, [p for _, p, _ in specs], [s for _, _, s in specs])
    passes = 10
    seen = set()
    for k in range(passes):
        ms_pass = batch.render_wavefront()
        st, ms = batch.stats()
        assert st.wavefront == 1 and st.streams == 4 and st.passes == k + 1
        assert st.tuned == (1 if k >= 7 else 0)
        seen.add((st.queue_paths, st.block, st.compact_every))
        assert ms_pass > 0 and np.all(ms > 0) and np.all(ms <= ms_pass * 1.05 + 0.05), (ms, ms_pass)
    assert len(seen) == 8
    with pytest.raises(vt.MaterialLibraryError, match="wavefront"):
        batch.render()
    for scene, (make, params, spp) in zip(batch_scenes, specs):
        img, n = scene.readback()
        assert n == passes * spp
        ref_scene = make()
        ref_scene.render_wavefront(params, passes * spp)
        ref, m = ref_scene.readback()
        ref_scene.close()
        assert m == n
        assert np.isfinite(img).all() and img.max() > 0
        np.testing.assert_allclose(img, ref, rtol=1e-12, atol=1e-12)
    batch.close()
    for sc in batch_scenes:
        sc.close()
    for m in meshes:
        m.close()


def test_batch_rejects_bad_input(ctx):
    faces, verts, mats, light, cam = scenes.cornell_box()
    mesh = vt.Mesh(ctx, faces, verts)
    a, b = vt.Scene(ctx, mesh, mats, light), vt.Scene(ctx, mesh, mats, light)
    p = vt.make_params(cam, 16, 16, 4, 1, False)
    with pytest.raises(vt.MaterialLibraryError, match="twice"):
        Batch(ctx, [a, a], [p, p], [1, 1])
    with pytest.raises(vt.MaterialLibraryError, match="modes 1-3"):
        Batch(ctx, [a, b], [p, vt.make_params(cam, 16, 16, 4, 1, False, mode=0)], [1, 1])
    with pytest.raises(vt.MaterialLibraryError, match="spp"):
        Batch(ctx, [a, b], [p, p], [1, 0])
    a.close()
    b.close()
    mesh.close()
