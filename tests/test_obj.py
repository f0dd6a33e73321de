"""OBJ / MTL input (CPU): geometry, indices, fans and the MTL -> slot mapping of
Sources/OBJMaterials.swift:4-27 that this renderer supports."""
import math

import numpy as np
import pytest

from metal_vibe_tracer_b200 import obj

OBJ = """# a quad, a triangle with normals and uvs, and a pentagon with negative indices
mtllib box.mtl
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
vt 0 0
vt 1 0
vt 1 1
vn 0 0 1
usemtl red
f 1 2 3 4
usemtl metal
f 1/1/1 2/2/1 3/3/1
v 0 0 1
v 1 0 1
v 1 1 1
v 0 1 1
v 0.5 1.5 1
usemtl lamp
f -5 -4 -3 -2 -1
usemtl missing
f 1 3 4
"""
MTL = """newmtl red
Kd 0.65 0.05 0.05
Ks 0 0 0
illum 2
newmtl metal
Kd 0.9 0.8 0.3
Ks 0.9 0.9 0.9
Ns 200
illum 3
Ni 1.5
map_Kd gold.png
newmtl lamp
Ke 10 9 8
newmtl glass
Kd 1 1 1
illum 4
"""


@pytest.fixture
def scene(tmp_path):
    (tmp_path / "box.obj").write_text(OBJ)
    (tmp_path / "box.mtl").write_text(MTL)
    return obj.load_obj(tmp_path / "box.obj")


def test_geometry(scene):
    faces, verts, mats, report = scene
    # quad -> 2, triangle -> 1, pentagon -> 3, last triangle -> 1
    assert len(faces) == 7
    assert list(faces["tag"]) == [0, 0, 1, 2, 2, 2, 3]
    p = verts["p"]
    np.testing.assert_array_equal(p[faces["a"][0]], [0, 0, 0])
    np.testing.assert_array_equal(p[faces["c"][1]], [0, 1, 0])
    np.testing.assert_array_equal(p[faces["c"][5]], [0.5, 1.5, 1])  # -1 is the last vertex
    tri = faces[2]
    assert np.allclose(verts["n"][tri["a"]], [0, 0, 1]) and np.allclose(verts["uv"][tri["c"]], [1, 1])
    assert np.all(verts["n"][faces["a"][0]] == 0)  # no vn: flat shading


def test_materials(scene):
    faces, verts, mats, report = scene
    red, metal, lamp, missing = mats
    assert red["type"] == 0 and red["albedo"] == (0.65, 0.05, 0.05)
    assert metal["type"] == 4 and metal["metalness"] == pytest.approx(0.9) and metal["ior"] == 1.5
    assert metal["roughness"] == pytest.approx(math.sqrt(math.sqrt(2 / 202)))
    assert lamp["type"] == 3 and lamp["emission"] == (10.0, 9.0, 8.0)
    assert missing["type"] == 0 and missing["albedo"] == (0.8, 0.8, 0.8)
    assert any("texture maps" in r for r in report) and any("missing" in r for r in report)


def test_glass_and_specular_weight_are_reported():
    report = []
    m = obj.read_mtl(MTL + "newmtl plastic\nKd 0.5 0.5 0.5\nKs 0.5 0.5 0.5\nNs 10\n", report)
    slot = obj.material_slot("glass", m["glass"], report)
    assert slot["type"] == 0 and any("transparency" in r for r in report)
    p = obj.material_slot("plastic", m["plastic"], report)
    assert p["type"] == 4 and p["metalness"] == 0.0 and any("specular weight" in r for r in report)


def test_bad_index_raises(tmp_path):
    (tmp_path / "bad.obj").write_text("v 0 0 0\nv 1 0 0\nf 1 2 3\n")
    with pytest.raises(ValueError, match="out of range"):
        obj.load_obj(tmp_path / "bad.obj")
