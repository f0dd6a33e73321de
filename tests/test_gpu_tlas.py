"""The two-level hierarchy on the B200 (vt_tlas_*) against the oracle.

- The instance records (inverse, norms, rendered bases, mirror flags) and the TLAS nodes equal the
  host restatement and the oracle's LBVH over the same instance boxes, bit for bit.
- Closest hits and hit instances equal the oracle's fp32 two-level traversal bit for bit; any-hit
  flags equal it exactly (mesh_closest / mesh_occluded, main.swift:1840-1984).
- Against the fp64 form and the flattened mesh (vt_tlas_flatten) the hits agree up to rounding.
- Bad transforms and mesh indices are rejected with the reference's messages
  (Sources/Acceleration.swift:474-499).
"""
import numpy as np
import pytest

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import scenes
from tests import fixtures_instances as FI

pytestmark = pytest.mark.gpu


def _build(ctx, oracle, grid=4, assets=3, sub=3, mirrored=0.3, seed=11):
    meshes, T, mesh_of, slots, mats, cam = scenes.instanced_grid(grid=grid, assets=assets, subdivisions=sub, seed=seed,
                                                                 mirrored_fraction=mirrored, nmat=9)
    gm = [vt.Mesh(ctx, f, v) for f, v in meshes]
    tlas = vt.Tlas(ctx, gm, vt.instances_array(T, mesh_of, slots))
    infos = [m.info() for m in gm]
    lo = np.array([list(i.lo) for i in infos], np.float32)
    hi = np.array([list(i.hi) for i in infos], np.float32)
    rec, grow, reach, bf, bv = FI.instance_setup(T, mesh_of, slots, [len(f) for f, _ in meshes], lo, hi)
    obvh = [oracle.Bvh.lbvh(f, v) for f, v in meshes]
    return meshes, T, mesh_of, slots, mats, gm, tlas, rec, grow, reach, bf, bv, obvh


def test_tlas_build_matches_host_and_oracle(ctx, oracle):
    meshes, T, mesh_of, slots, _, gm, tlas, rec, grow, reach, bf, bv, _ = _build(ctx, oracle)
    info = tlas.info()
    assert info.instances == len(T) and info.meshes == len(meshes)
    assert info.rendered_triangles == sum(len(meshes[m][0]) for m in mesh_of)
    assert np.float32(info.grow) == np.float32(grow) and np.float32(info.reach) == np.float32(reach)
    got = tlas.records()
    for name in ("world", "local", "mesh", "slot_base", "rendered_base", "mirrored", "bound"):
        assert np.array_equal(got[name], rec[name]), name
    assert got["mirrored"].any()
    nodes = FI.oracle_tlas(oracle, bf, bv)
    assert np.array_equal(tlas.nodes().view(np.uint8), nodes.view(np.uint8))
    # Every instance's transformed vertices lie inside its leaf box.
    leaf_box = {}
    for nd in tlas.nodes():
        for k in range(4):
            if nd["child"][k] < 0:
                leaf_box[-nd["child"][k] - 1] = (np.array([nd["lox"][k], nd["loy"][k], nd["loz"][k]]),
                                                 np.array([nd["hix"][k], nd["hiy"][k], nd["hiz"][k]]))
    assert sorted(leaf_box) == list(range(len(T)))
    for i, mi in enumerate(mesh_of):
        p = meshes[mi][1]["p"].astype(np.float64) @ T[i, :, :3].T.astype(np.float64) + T[i, :, 3]
        lo, hi = leaf_box[i]
        assert np.all(p >= lo) and np.all(p <= hi)


def test_tlas_traversal_matches_oracle(ctx, oracle):
    meshes, T, mesh_of, slots, _, gm, tlas, rec, grow, reach, bf, bv, obvh = _build(ctx, oracle)
    nodes = tlas.nodes()
    p = bv["p"]
    rays = FI.probe_rays(p.min(0), p.max(0), 20000, seed=7)
    hits, inst = tlas.closest(rays)
    oh, oi = oracle.tlas_trace(nodes, tlas.records(), obvh, grow, reach, rays, precision=32)
    assert (hits["prim"] >= 0).mean() > 0.3
    assert np.array_equal(hits.view(np.uint32), oh.view(np.uint32))
    assert np.array_equal(inst, oi)
    # fp64 judge.
    h64, i64 = oracle.tlas_trace(nodes, tlas.records(), obvh, grow, reach, rays, precision=64)
    same = (h64["prim"] == hits["prim"]) & (i64 == inst)
    assert same.mean() > 0.999
    h = same & (hits["prim"] >= 0)
    assert np.allclose(hits["t"][h], h64["t"][h], rtol=1e-5, atol=1e-6)
    # Any hit, with tmax around the closest hit.
    t = np.where(hits["prim"] >= 0, hits["t"], np.inf)
    short = rays.copy()
    rng = np.random.default_rng(3)
    short[:, 7] = np.where(np.isfinite(t), t * rng.choice([0.5, 0.999, 1.001, 2.0], len(t)), 5.0).astype(np.float32)
    occ = tlas.occluded(short)
    oocc = oracle.tlas_trace(nodes, tlas.records(), obvh, grow, reach, short, closest=False, precision=32)
    assert np.array_equal(occ, oocc)


def test_tlas_flatten_matches_two_level(ctx, oracle):
    meshes, T, mesh_of, slots, _, gm, tlas, rec, grow, reach, bf, bv, obvh = _build(ctx, oracle)
    flat = tlas.flatten()
    fi = flat.info()
    assert fi.faces == tlas.info().rendered_triangles
    p = bv["p"]
    rays = FI.probe_rays(p.min(0), p.max(0), 20000, seed=9)
    hits, inst = tlas.closest(rays)
    fh = flat.closest(rays)
    base = rec["rendered_base"].astype(np.int64)
    tl_id = np.where(hits["prim"] >= 0, base[np.minimum(inst, len(rec) - 1)] + hits["prim"], -1)
    assert np.mean(tl_id == fh["prim"]) > 0.995
    both = (fh["prim"] >= 0) & (tl_id == fh["prim"])
    assert np.allclose(hits["t"][both], fh["t"][both], rtol=1e-4, atol=1e-6)
    # The flattened soup against brute force over the host-flattened triangles.
    wf, wv = FI.flatten_world(meshes, T, mesh_of, slots)
    brute = oracle.brute_closest(wf, wv, rays[:4000], precision=64)
    assert np.mean(brute["prim"] == fh["prim"][:4000]) > 0.995


def test_tlas_rejects_bad_instances(ctx, oracle):
    meshes, T, mesh_of, slots, _, gm, tlas, *_ = _build(ctx, oracle, grid=2, assets=1, sub=1)
    inst = vt.instances_array(T, mesh_of, slots)
    bad = inst.copy()
    bad["mesh"][0] = 99
    with pytest.raises(vt.MaterialLibraryError, match="names mesh"):
        vt.Tlas(ctx, gm, bad)
    bad = inst.copy()
    bad["world"][0, [0, 4, 8]] = 0.0  # first column zero
    with pytest.raises(vt.MaterialLibraryError, match="scale"):
        vt.Tlas(ctx, gm, bad)
    bad = inst.copy()
    bad["world"][0, 4:7] = bad["world"][0, 0:3]  # rows 0 and 1 equal: singular
    with pytest.raises(vt.MaterialLibraryError, match="Singular"):
        vt.Tlas(ctx, gm, bad)
    bad = inst.copy()
    bad["world"][0, 3] = 2e8
    with pytest.raises(vt.MaterialLibraryError, match="extent"):
        vt.Tlas(ctx, gm, bad)
    # The context stays usable.
    ok = vt.Tlas(ctx, gm, inst)
    assert ok.info().instances == len(inst)
