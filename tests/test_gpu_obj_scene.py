"""An OBJ/MTL scene (the importer's path: obj.load_obj -> vt.Mesh -> vt.Scene as an imported scene,
Sources/OBJMaterials.swift:4-27 for the material mapping) rendered on the B200 against the FP64 oracle
on the same geometry and slots: a room of Lambert walls, a smooth-shaded metal block and a dielectric
block (OPENPBR slots from Ks / Ns / Ni / illum), lit by an emissive Ke quad under its light tree.
The bars are the integrator parity tests' own: mean radiance within 0.1 %, per-pixel relMSE below a
quarter of the estimator's own, and most pixels equal to 1e-4."""
import numpy as np
import pytest

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import obj, spectral_tables

pytestmark = pytest.mark.gpu

ROOM_OBJ = """# room 4 x 3 x 4 (open toward -z), two blocks, a lamp under the ceiling
mtllib room.mtl
v -2 0 -2
v 2 0 -2
v 2 0 2
v -2 0 2
v -2 3 -2
v 2 3 -2
v 2 3 2
v -2 3 2
usemtl white
f 1 4 3 2
f 5 6 7 8
f 4 8 7 3
usemtl red
f 1 5 8 4
usemtl green
f 2 3 7 6
v -0.4 2.99 -0.4
v 0.4 2.99 -0.4
v 0.4 2.99 0.4
v -0.4 2.99 0.4
usemtl lamp
f 9 10 11 12
v -1.3 0 -0.2
v -0.3 0 -0.2
v -0.3 0 0.8
v -1.3 0 0.8
v -1.3 1.4 -0.2
v -0.3 1.4 -0.2
v -0.3 1.4 0.8
v -1.3 1.4 0.8
vn 0 0 -1
vn 0 0 1
vn -1 0 0
vn 1 0 0
vn 0 1 0
usemtl gold
f 13//1 17//1 18//1 14//1
f 16//2 15//2 19//2 20//2
f 13//3 16//3 20//3 17//3
f 14//4 18//4 19//4 15//4
f 17//5 20//5 19//5 18//5
v 0.4 0 -0.6
v 1.2 0 -0.6
v 1.2 0 0.2
v 0.4 0 0.2
v 0.4 0.8 -0.6
v 1.2 0.8 -0.6
v 1.2 0.8 0.2
v 0.4 0.8 0.2
usemtl plastic
f 21 25 26 22
f 24 23 27 28
f 21 24 28 25
f 22 26 27 23
f 25 28 27 26
"""
ROOM_MTL = """newmtl white
Kd 0.73 0.73 0.73
newmtl red
Kd 0.63 0.065 0.05
newmtl green
Kd 0.14 0.45 0.091
newmtl lamp
Ke 12 10 8
newmtl gold
Kd 1.0 0.77 0.34
Ks 1.0 0.77 0.34
Ns 400
illum 3
newmtl plastic
Kd 0.2 0.3 0.6
Ks 0.04 0.04 0.04
Ns 90
Ni 1.45
illum 2
"""
CAMERA = {"pos": (0.0, 1.5, -6.0), "target": (0.0, 1.2, 0.0), "up": (0.0, 1.0, 0.0), "fov": 45.0}


def relmse(a, b):
    return float(np.mean((a - b) ** 2 / (b ** 2 + 1e-2)))


@pytest.mark.parametrize("spectral", [False, True])
def test_obj_scene_matches_oracle(ctx, oracle, tmp_path, spectral):
    (tmp_path / "room.obj").write_text(ROOM_OBJ)
    (tmp_path / "room.mtl").write_text(ROOM_MTL)
    faces, verts, mats, report = obj.load_obj(tmp_path / "room.obj")
    types = [m["type"] for m in mats]
    assert types.count(3) == 1 and types.count(4) == 2, types  # one emitter, two OPENPBR slots
    tables = spectral_tables.load() if spectral else None
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, None, tables)
    scene.render(vt.make_params(CAMERA, 96, 96, 6, 1, spectral, 1), 16)
    gpu, n = scene.readback()
    scene.close()
    mesh.close()
    assert n == 16 and np.isfinite(gpu).all() and gpu.mean() > 0
    ref = oracle.render(faces, verts, mats, None, CAMERA, 96, 96, 16, max_depth=6, spectral=tables)
    other = oracle.render(faces, verts, mats, None, CAMERA, 96, 96, 16, max_depth=6, first_sample=1001,
                          spectral=tables)
    gm, rm = gpu.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(gm / rm - 1) < 1e-3), (gm, rm)
    assert relmse(gpu, ref) < 0.25 * relmse(other, ref), (relmse(gpu, ref), relmse(other, ref))
    same = np.all(np.abs(gpu - ref) <= 1e-4 * np.maximum(np.abs(ref), 1e-3), axis=-1)
    assert same.mean() > 0.9, same.mean()
