"""The oracle's two-level traversal (mesh_closest / mesh_occluded, main.swift:1840-1984) against
brute force over the flattened world triangles (CPU only).

Instances trace their meshes in object space (instance_ray, main.swift:1634-1637) while the brute
force intersects the transformed triangles, so the two agree up to rounding: the same (instance,
face) on nearly every ray and t to 1e-4 relative. The fp32 form (the CUDA kernel's arithmetic) must
agree with the fp64 form the same way.
"""
import numpy as np

from metal_vibe_tracer_b200 import scenes
from tests import fixtures_instances as FI


def _scene(oracle, grid=3, assets=2, sub=2, mirrored=0.4, seed=3):
    meshes, T, mesh_of, slots, _, _ = scenes.instanced_grid(grid=grid, assets=assets, subdivisions=sub, seed=seed,
                                                            mirrored_fraction=mirrored, nmat=7)
    obvh = [oracle.Bvh.lbvh(f, v) for f, v in meshes]
    infos = [b.info() for b in obvh]
    lo = np.array([list(i.lo) for i in infos], np.float32)
    hi = np.array([list(i.hi) for i in infos], np.float32)
    rec, grow, reach, bf, bv = FI.instance_setup(T, mesh_of, slots, [len(f) for f, _ in meshes], lo, hi)
    nodes = FI.oracle_tlas(oracle, bf, bv)
    return meshes, T, mesh_of, slots, obvh, rec, grow, reach, nodes, bv


def test_tlas_oracle_matches_brute_force(oracle):
    meshes, T, mesh_of, slots, obvh, rec, grow, reach, nodes, bv = _scene(oracle)
    assert rec["mirrored"].any() and not rec["mirrored"].all()
    p = bv["p"]
    rays = FI.probe_rays(p.min(0), p.max(0), 4000, seed=1)
    hits64, inst64 = oracle.tlas_trace(nodes, rec, obvh, grow, reach, rays, precision=64)
    hits32, inst32 = oracle.tlas_trace(nodes, rec, obvh, grow, reach, rays, precision=32)
    wf, wv = FI.flatten_world(meshes, T, mesh_of, slots)
    brute = oracle.brute_closest(wf, wv, rays, precision=64)
    base = rec["rendered_base"].astype(np.int64)
    tl_id = np.where(hits64["prim"] >= 0, base[np.minimum(inst64, len(rec) - 1)] + hits64["prim"], -1)
    hit = brute["prim"] >= 0
    assert hit.mean() > 0.3
    assert np.mean(tl_id == brute["prim"]) > 0.995
    both = hit & (tl_id == brute["prim"])
    assert np.allclose(hits64["t"][both], brute["t"][both], rtol=1e-4, atol=1e-6)
    # fp32 (the kernel's arithmetic) against fp64.
    same = (hits32["prim"] == hits64["prim"]) & (inst32 == inst64)
    assert same.mean() > 0.999
    h = same & (hits64["prim"] >= 0)
    assert np.allclose(hits32["t"][h], hits64["t"][h], rtol=1e-5, atol=1e-6)


def test_tlas_oracle_any_hit(oracle):
    meshes, T, mesh_of, slots, obvh, rec, grow, reach, nodes, bv = _scene(oracle, seed=5)
    p = bv["p"]
    rays = FI.probe_rays(p.min(0), p.max(0), 3000, seed=2)
    hits, _ = oracle.tlas_trace(nodes, rec, obvh, grow, reach, rays, precision=64)
    t = np.where(hits["prim"] >= 0, hits["t"], np.inf)
    rng = np.random.default_rng(4)
    short = rays.copy()
    short[:, 7] = np.where(np.isfinite(t), t * rng.choice([0.5, 1.5], len(t)), 10.0).astype(np.float32)
    occ = oracle.tlas_trace(nodes, rec, obvh, grow, reach, short, closest=False, precision=32)
    expect = np.isfinite(t) & (short[:, 7] > t)
    assert np.mean(occ.astype(bool) == expect) > 0.999
