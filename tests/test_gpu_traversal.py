"""GPU traversal against the oracle.

* bit for bit (t, b1, b2, face) against the oracle's fp32 restatement on the same BVH;
* against the fp64 oracle: the same face on >= 99.99% of rays, t within 1e-5 relative;
* watertightness at the curved patch's shared edges and vertices (tests/Fix_accel.swift:244-297);
* any-hit against the oracle, host-buffer path equal to the device path, and edge cases.
"""
import math

import numpy as np
import pytest
import torch

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import scenes
from tests import fixtures_geometry as G

pytestmark = pytest.mark.gpu

REL_T = 1e-5       # t tolerance against the fp64 oracle (relative)
ID_AGREEMENT = 0.9999


def gpu_closest(mesh, rays):
    t = torch.from_numpy(np.ascontiguousarray(rays, np.float32).reshape(-1, 8)).cuda()
    out = mesh.closest(t)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(vt.HIT_DTYPE).reshape(-1)


def gpu_any(mesh, rays):
    t = torch.from_numpy(np.ascontiguousarray(rays, np.float32).reshape(-1, 8)).cuda()
    out = mesh.occluded(t)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def assert_bit_exact(a, b):
    diff = np.nonzero(a.view(np.uint32).reshape(-1, 4) != b.view(np.uint32).reshape(-1, 4))[0]
    assert diff.size == 0, f"{np.unique(diff).size} rays differ, first {a[diff[0]]} vs {b[diff[0]]}"


def assert_fp64_agreement(gpu, ref64):
    same = gpu["prim"] == ref64["prim"]
    assert same.mean() >= ID_AGREEMENT, f"face agreement {same.mean():.6f}"
    m = same & (ref64["prim"] >= 0)
    rel = np.abs(gpu["t"][m].astype(np.float64) - ref64["t"][m]) / np.abs(ref64["t"][m])
    assert rel.size == 0 or rel.max() <= REL_T, f"max rel t error {rel.max():.3e}"


def test_lcg_parity_protocol(ctx, oracle):
    rng = G.Lcg()
    faces, verts = G.lcg_soup(4000, rng)
    rays = G.lcg_rays(20_000, rng)
    mesh = vt.Mesh(ctx, faces, verts)
    ref = oracle.Bvh.lbvh(faces, verts)
    hits = gpu_closest(mesh, rays)
    assert_bit_exact(hits, ref.closest(rays))
    assert_bit_exact(hits, oracle.brute_closest(faces, verts, rays))
    assert_fp64_agreement(hits, oracle.brute_closest(faces, verts, rays, precision=64))
    assert np.array_equal(gpu_any(mesh, rays), ref.occluded(rays))


def test_patch_watertight_gpu(ctx, oracle):
    faces, verts, grid = G.patch(48)
    rays = G.patch_targets(grid)
    mesh = vt.Mesh(ctx, faces, verts)
    hits = gpu_closest(mesh, rays)
    assert (hits["prim"] >= 0).all(), f"{(hits['prim'] < 0).sum()} misses at shared edges/vertices"
    assert_bit_exact(hits, oracle.Bvh.lbvh(faces, verts).closest(rays))
    assert gpu_any(mesh, rays).all()


@pytest.mark.parametrize("leaf", [1, 2, 4])
def test_soup_sets_against_oracle(ctx, oracle, leaf):
    faces, verts = scenes.triangle_soup(200_000, seed=7)
    mesh = vt.Mesh(ctx, faces, verts, leaf_size=leaf)
    ref = oracle.Bvh.lbvh(faces, verts, leaf_size=leaf)
    coherent = scenes.coherent_rays_np(512, 512)[::3]
    incoherent = scenes.incoherent_rays_np(60_000, seed=3)
    for rays, coh in ((coherent, True), (incoherent, False)):
        hits = gpu_closest(mesh, rays)
        assert_bit_exact(hits, ref.closest(rays))
        assert_fp64_agreement(hits, ref.closest(rays, precision=64))
        shadow = scenes.shadow_tmax_np(rays, coh)
        assert np.array_equal(gpu_any(mesh, shadow), ref.occluded(shadow))


def test_full_size_sample_1m(ctx, oracle):
    faces, verts = scenes.triangle_soup(1_000_000, seed=0)
    mesh = vt.Mesh(ctx, faces, verts)
    ref = oracle.Bvh.lbvh(faces, verts)
    rays = np.concatenate([scenes.coherent_rays_np(4096, 4096, rows=slice(0, 4096, 64)),
                           scenes.incoherent_rays_np(100_000, seed=1)])
    hits = gpu_closest(mesh, rays)
    assert_bit_exact(hits, ref.closest(rays))
    assert_fp64_agreement(hits, ref.closest(rays, precision=64))
    shadow = np.concatenate([scenes.shadow_tmax_np(rays[:65536], True), scenes.shadow_tmax_np(rays[65536:], False)])
    assert np.array_equal(gpu_any(mesh, shadow), ref.occluded(shadow))


def test_host_path_equals_device_path(ctx):
    faces, verts = scenes.triangle_soup(50_000, seed=11, mu=math.log(0.01))
    mesh = vt.Mesh(ctx, faces, verts)
    # Three pipeline chunks (2^22 rays each, the last ragged), so both streams and both staging
    # slots are reused. numpy arrays are pageable: the call stages them through pinned buffers.
    rays = scenes.incoherent_rays_np((2 << 22) + 12345, seed=4)
    host = mesh.closest(rays)
    dev = gpu_closest(mesh, rays)
    assert_bit_exact(host, dev)
    shadow = scenes.shadow_tmax_np(rays, False)
    occ_dev = gpu_any(mesh, shadow)
    assert np.array_equal(mesh.occluded(shadow), occ_dev)
    # Pinned caller buffers take the direct asynchronous copies instead.
    pin_rays = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).pin_memory()
    pin_hits = torch.empty((rays.shape[0], 4), dtype=torch.float32).pin_memory()
    mesh.closest(pin_rays.numpy().view(vt.RAY_DTYPE).reshape(-1), pin_hits.numpy().view(vt.HIT_DTYPE).reshape(-1))
    assert_bit_exact(pin_hits.numpy().view(vt.HIT_DTYPE).reshape(-1), dev)
    pin_shadow = torch.from_numpy(np.ascontiguousarray(shadow).view(np.float32).reshape(-1, 8)).pin_memory()
    pin_occ = torch.empty((rays.shape[0],), dtype=torch.uint8).pin_memory()
    mesh.occluded(pin_shadow.numpy().view(vt.RAY_DTYPE).reshape(-1), pin_occ.numpy())
    assert np.array_equal(pin_occ.numpy(), occ_dev)
    # Mixed: pageable rays into a pinned output.
    mesh.closest(rays, pin_hits.numpy().view(vt.HIT_DTYPE).reshape(-1))
    assert_bit_exact(pin_hits.numpy().view(vt.HIT_DTYPE).reshape(-1), dev)


def test_edge_cases(ctx, oracle):
    # Empty mesh: every ray misses.
    empty = vt.Mesh(ctx, np.zeros(0, vt.FACE_DTYPE), np.zeros(0, vt.VERTEX_DTYPE))
    rays = scenes.incoherent_rays_np(1000)
    assert (gpu_closest(empty, rays)["prim"] == -1).all()
    assert not gpu_any(empty, rays).any()
    # Zero rays.
    faces, verts = scenes.triangle_soup(1000, seed=3, mu=math.log(0.05))
    mesh = vt.Mesh(ctx, faces, verts)
    assert gpu_closest(mesh, np.zeros((0, 8), np.float32)).shape == (0,)
    # Axis-parallel directions, tmin >= tmax, degenerate triangles.
    special = scenes.incoherent_rays_np(3000, seed=8)
    special[0:1000, 4:7] = np.array([[1, 0, 0], [0, -1, 0], [0, 0, 1]], np.float32)[np.arange(1000) % 3]
    special[1000:1500, 3] = special[1000:1500, 7] = 0.5
    f2 = faces.copy()
    v2 = verts.copy()
    v2["p"][3 * 10 + 2] = v2["p"][3 * 10 + 1]  # face 10 collapses to a segment
    for fs, vs in ((faces, verts), (f2, v2)):
        m = vt.Mesh(ctx, fs, vs)
        ref = oracle.Bvh.lbvh(fs, vs)
        hits = gpu_closest(m, special)
        assert_bit_exact(hits, ref.closest(special))
        assert (hits["prim"][1000:1500] == -1).all()
        assert np.array_equal(gpu_any(m, special), ref.occluded(special))


def test_traversal_counts_match_oracle(ctx, oracle):
    faces, verts = scenes.triangle_soup(100_000, seed=12)
    mesh = vt.Mesh(ctx, faces, verts)
    ref = oracle.Bvh.lbvh(faces, verts)
    rays = scenes.incoherent_rays_np(20_000, seed=6)
    assert mesh.count(rays, closest=True) == ref.count(rays, closest=True)
    shadow = scenes.shadow_tmax_np(rays, False)
    assert mesh.count(shadow, closest=False) == ref.count(shadow, closest=False)
