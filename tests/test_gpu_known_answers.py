"""The reference's own device known answers (regression_checks, tests/GPUChecks.swift:14-37), checked
on the B200 against the integrator's device functions and its traversal.

* results[3]: power_heuristic(1e-10, 1e-10) = 0.5 within 1e-6;
* results[5]: the emission_weight truth table;
* results[2]: rand_f stays in [0, 1) over 100,000 draws from seed 17, and seed 890625759 (whose second
  PCG draw is exactly zero) gives a cosine sample above the grazing normal's tangent plane (> 1e-4);
* results[0..1]: a ray leaving the inside of a box exits at t = 1 through a back face whose normal,
  turned toward the ray, points along -x; a ray parallel to the box outside misses. The reference
  checks its analytic box primitive; the configs trace triangles, so the same rays are traced
  against a triangulated box.
* the scattering budget max(0, depth - 1) (scattering_limit, main.swift:3471-3473);
* results[4]: glass (IOR 1.52) met from inside beyond the critical angle reflects totally: the sample
  exists, goes back to z < 0 and weighs exactly 1 (sample_delta, the delta dielectric).
"""
import numpy as np
import pytest
import torch

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200.render import known_answers

pytestmark = pytest.mark.gpu


def test_device_known_answers(ctx):
    k = known_answers(ctx)
    assert abs(k[0] - 0.5) < 1e-6
    assert k[1] == 0.0 and k[2] == 1.0 and k[3] == 1.0
    assert k[4] == 0.0, "seed 890625759's second PCG draw must be exactly zero"
    assert k[5] > 1e-4, "the grazing cosine sample must stay above the tangent plane"
    assert 0.0 <= k[6] and k[7] < 1.0
    assert list(k[8:11]) == [0.0, 0.0, 7.0]
    # Glass, IOR 1.52, met from inside beyond the critical angle (GPUChecks.swift:32-34): the sample
    # exists, reflects to z < 0 and weighs exactly 1.
    assert k[11] == 1.0 and k[12] < 0.0 and list(k[13:16]) == [1.0, 1.0, 1.0]


def _box(lo, hi):
    """A closed box of 12 triangles wound counter-clockwise seen from outside (outward normals)."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    p = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float32)
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]
    tris = []
    for a, b, c, d in quads:
        tris += [(a, b, c), (a, c, d)]
    faces = np.zeros(len(tris), vt.FACE_DTYPE)
    for i, (a, b, c) in enumerate(tris):
        faces[i] = (a, b, c, 0)
    verts = np.zeros(len(p), vt.VERTEX_DTYPE)
    verts["p"] = p
    return faces, verts, p, tris


def test_box_exit_and_parallel_miss(ctx):
    faces, verts, p, tris = _box((-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))
    n = np.cross(p[[t[1] for t in tris]] - p[[t[0] for t in tris]], p[[t[2] for t in tris]] - p[[t[0] for t in tris]])
    assert (np.einsum("ij,ij->i", n, p[[t[0] for t in tris]]) > 0).all(), "outward winding"
    mesh = vt.Mesh(ctx, faces, verts)
    rays = np.zeros((2, 8), np.float32)
    rays[0] = [0, 0, 0, 0.001, 1, 0, 0, 100]     # inside, toward +x
    rays[1] = [2, 0, 0, 0.001, 0, 1, 0, 100]     # outside, parallel to the x = 1 face
    hits = mesh.closest(torch.from_numpy(rays).cuda()).cpu().numpy().view(vt.HIT_DTYPE).reshape(-1)
    assert abs(hits["t"][0] - 1.0) < 1e-5
    f = hits["prim"][0]
    ng = n[f] / np.linalg.norm(n[f])
    front = float(ng @ rays[0, 4:7]) < 0.0
    assert not front, "the exit is through a back face"
    turned = ng if front else -ng
    assert turned[0] < -0.99
    assert hits["prim"][1] == -1
    occ = mesh.occluded(torch.from_numpy(rays).cuda()).cpu().numpy()
    assert occ[0] == 1 and occ[1] == 0
    mesh.close()
