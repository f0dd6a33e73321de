"""The oracle renderer's sampling options (CPU only): a pixel stride renders exactly the strided
pixels of the full image (each pixel's own camera ray and sample stream), and a hierarchy imported
from arrays (the device's build, here the oracle's own) renders the same image as the built one."""
import numpy as np

from metal_vibe_tracer_b200 import scenes


def test_stride_and_imported_bvh(oracle):
    faces, verts, mats, light, cam = scenes.cornell_box()
    full = oracle.render(faces, verts, mats, light, cam, 33, 25, 2)
    strided = oracle.render(faces, verts, mats, light, cam, 33, 25, 2, pixel_stride=4)
    assert strided.shape == (7, 9, 3)
    np.testing.assert_array_equal(strided, full[::4, ::4])
    built = oracle.Bvh.lbvh(faces, verts)
    info = built.info()
    imported = oracle.Bvh.from_arrays(built.nodes(), built.order(), faces, verts, info.depth)
    again = oracle.render(faces, verts, mats, light, cam, 33, 25, 2, bvh=imported)
    np.testing.assert_array_equal(again, full)
