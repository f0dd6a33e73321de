"""The oracle against the reference's known answers and its own invariants (CPU only).

Pins: the PCG stream's known answer (seed 890625759 draws exactly zero second,
tests/GPUChecks.swift:24-27), rand_f's range over 10^5 draws from seed 17 (GPUChecks.swift:20-23),
watertightness at the shared edges and vertices of the curved patch (tests/Fix_accel.swift:244-
297: no misses, hits equal brute force), and BVH traversal equal to brute force on the parity
soup and rays (tests/Fix_accel.swift:216-243).
"""
import math

import numpy as np
import pytest

from metal_vibe_tracer_b200 import scenes
from tests import fixtures_geometry as G


def pcg_hash_py(v: int) -> int:
    """main.swift:91-95, restated in Python integers."""
    state = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & 0xFFFFFFFF
    return ((word >> 22) ^ word) & 0xFFFFFFFF


def test_pcg_matches_python_restatement(oracle):
    rng = np.random.default_rng(0)
    for v in [0, 1, 17, 0xFFFFFFFF, 890625759, *rng.integers(0, 2**32, 200).tolist()]:
        assert oracle.pcg_hash(v) == pcg_hash_py(v)


def test_pcg_known_answer_seed_890625759(oracle):
    # tests/GPUChecks.swift:24-27: "This seed makes the second PCG draw exactly zero."
    x, s = oracle.rand_f(890625759)
    y, s = oracle.rand_f(s)
    assert y == 0.0 and x > 0.0


def test_rand_f_bounded(oracle):
    s = 17
    lo, hi = 1.0, 0.0
    for _ in range(100_000):
        v, s = oracle.rand_f(s)
        lo, hi = min(lo, v), max(hi, v)
    assert lo >= 0.0 and hi < 1.0


def test_watertight_single_triangle(oracle):
    tri = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float32)
    hit, t, b1, b2 = oracle.intersect_f32([0.25, 0.25, 1.0, 0.0, 0, 0, -1, np.inf], tri)
    assert hit and t == 1.0 and b1 == 0.25 and b2 == 0.25
    # Two-sided, [tmin, tmax) half open.
    hit, t, _, _ = oracle.intersect_f32([0.25, 0.25, -1.0, 0.0, 0, 0, 1, np.inf], tri)
    assert hit and t == 1.0
    assert not oracle.intersect_f32([0.25, 0.25, 1.0, 0.0, 0, 0, -1, 1.0], tri)[0]
    assert oracle.intersect_f32([0.25, 0.25, 1.0, 1.0, 0, 0, -1, 1.5], tri)[0]
    # Edge and vertex hits count (edge value 0 is inside).
    assert oracle.intersect_f32([0.5, 0.0, 1.0, 0.0, 0, 0, -1, np.inf], tri)[0]
    assert oracle.intersect_f32([0.0, 0.0, 1.0, 0.0, 0, 0, -1, np.inf], tri)[0]
    assert not oracle.intersect_f32([0.6, 0.6, 1.0, 0.0, 0, 0, -1, np.inf], tri)[0]
    # A ray in the triangle's plane (det = 0) misses.
    assert not oracle.intersect_f32([-1, 0.25, 0, 0, 1, 0, 0, np.inf], tri)[0]
    # fp64 agrees.
    hit, t, b1, b2 = oracle.intersect_f64([0.25, 0.25, 1.0], [0, 0, -1], tri)
    assert hit and t == 1.0 and b1 == 0.25 and b2 == 0.25


@pytest.mark.parametrize("precision", [32, 64])
def test_patch_watertight(oracle, precision):
    faces, verts, grid = G.patch(48)
    rays = G.patch_targets(grid)
    for builder in ("lbvh", "wide"):
        bvh = oracle.Bvh.lbvh(faces, verts) if builder == "lbvh" else oracle.Bvh.widebvh(faces, verts)
        hits = bvh.closest(rays, precision=precision)
        assert (hits["prim"] >= 0).all(), f"{builder}: {(hits['prim'] < 0).sum()} misses at shared edges"
        brute = oracle.brute_closest(faces, verts, rays, precision=precision)
        same = hits["prim"] == brute["prim"]
        # At a shared edge both neighbours are the closest hit (equal t).
        tie = np.abs(hits["t"] - brute["t"]) <= 1e-6 * np.maximum(1.0, np.abs(brute["t"]))
        assert (same | tie).all()
        # Every target ray hits at (almost exactly) its target: t ~ length / 1.001.
        length = rays[:, 7] / np.float32(1.001)
        assert np.all(np.abs(hits["t"] - length) <= 1e-4 * length)


def test_lcg_soup_bvh_equals_brute_force(oracle):
    rng = G.Lcg()
    faces, verts = G.lcg_soup(1500, rng)
    rays = G.lcg_rays(4000, rng)
    brute = oracle.brute_closest(faces, verts, rays)
    for bvh in (oracle.Bvh.lbvh(faces, verts), oracle.Bvh.widebvh(faces, verts),
                oracle.Bvh.lbvh(faces, verts, treelet_size=-1), oracle.Bvh.lbvh(faces, verts, leaf_size=4)):
        hits = bvh.closest(rays)
        assert np.array_equal(hits.view(np.uint32), brute.view(np.uint32))
        occ = bvh.occluded(rays)
        assert np.array_equal(occ.astype(bool), brute["prim"] >= 0)
    b64 = oracle.brute_closest(faces, verts, rays, precision=64)
    agree = (b64["prim"] == brute["prim"]).mean()
    assert agree >= 0.9999
    m = (b64["prim"] >= 0) & (b64["prim"] == brute["prim"])
    assert np.all(np.abs(brute["t"][m] - b64["t"][m]) <= 1e-5 * np.abs(b64["t"][m]))


def _check_wide_tree(faces, verts, bvh, leaf_size):
    nodes, order = bvh.nodes(), bvh.order()
    n = len(faces)
    assert sorted(order.tolist()) == list(range(n))
    p = verts["p"]
    tri = np.stack([p[faces["a"]], p[faces["b"]], p[faces["c"]]], axis=1)
    lo, hi = tri.min(axis=1), tri.max(axis=1)
    seen = np.zeros(n, bool)
    referenced = np.zeros(len(nodes), int)
    for nd in nodes:
        for k in range(4):
            c = nd["child"][k]
            if c > 0:
                referenced[c] += 1
            elif c < 0:
                first, cnt = -c - 1, nd["count"][k]
                assert 1 <= cnt <= leaf_size
                items = order[first:first + cnt]
                assert not seen[first:first + cnt].any()
                seen[first:first + cnt] = True
                box_lo = np.array([nd["lox"][k], nd["loy"][k], nd["loz"][k]])
                box_hi = np.array([nd["hix"][k], nd["hiy"][k], nd["hiz"][k]])
                assert np.all(lo[items] >= box_lo) and np.all(hi[items] <= box_hi)
    assert seen.all()
    assert referenced[0] == 0 and np.all(referenced[1:] == 1)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 100, 3000])
def test_builds_well_formed(oracle, n):
    faces, verts = scenes.triangle_soup(n, seed=n, mu=math.log(0.05))
    for leaf in (1, 2, 4):
        _check_wide_tree(faces, verts, oracle.Bvh.lbvh(faces, verts, leaf_size=leaf), leaf)
        _check_wide_tree(faces, verts, oracle.Bvh.widebvh(faces, verts, leaf_size=leaf), leaf)


def test_widebvh_depth_limit_and_deferred_numbering(oracle):
    # n >= 65536 exercises the deferred subtrees (Sources/Acceleration.swift:312-350).
    faces, verts = scenes.triangle_soup(70_000, seed=4)
    w = oracle.Bvh.widebvh(faces, verts)
    assert w.info().depth <= 20
    _check_wide_tree(faces, verts, w, 2)
    # The result does not depend on the thread count.
    w1 = oracle.Bvh.widebvh(faces, verts, nthreads=1)
    assert np.array_equal(w.nodes().view(np.uint8), w1.nodes().view(np.uint8))
    assert np.array_equal(w.order(), w1.order())


def expand_bits_py(v):
    out = 0
    for b in range(10):
        out |= ((v >> b) & 1) << (3 * b)
    return out


def test_lbvh_morton_codes_restatement(oracle):
    faces, verts = scenes.triangle_soup(2000, seed=9, mu=math.log(0.03))
    bvh = oracle.Bvh.lbvh(faces, verts)
    codes, sorted_ = bvh.morton()
    p = verts["p"]
    tri = np.stack([p[faces["a"]], p[faces["b"]], p[faces["c"]]], axis=1)
    c = ((tri.min(axis=1) + tri.max(axis=1)) * np.float32(0.5)).astype(np.float32)
    clo, chi = c.min(axis=0), c.max(axis=0)
    ext = (chi - clo).astype(np.float32)
    scale = (np.float32(1024.0) / ext).astype(np.float32)
    f = ((c - clo).astype(np.float32) * scale).astype(np.float32)
    q = np.minimum(f, np.float32(1023)).astype(np.uint32)
    expect = [(expand_bits_py(int(a)) << 2) | (expand_bits_py(int(b)) << 1) | expand_bits_py(int(z)) for a, b, z in q]
    keys = sorted((e, i) for i, e in enumerate(expect))
    assert codes.tolist() == [k[0] for k in keys]
    assert sorted_.tolist() == [k[1] for k in keys]


def test_lbvh_refinement_lowers_sah(oracle):
    faces, verts = scenes.triangle_soup(20_000, seed=5)
    plain = oracle.Bvh.lbvh(faces, verts, treelet_size=-1)
    refined = oracle.Bvh.lbvh(faces, verts)
    wide = oracle.Bvh.widebvh(faces, verts)
    assert refined.info().sah_cost < plain.info().sah_cost
    # Within 5% of the reference's binned-SAH build.
    assert refined.info().sah_cost <= 1.05 * wide.info().sah_cost
    # Refinement keeps every binary node's box exact: the union of its children.
    ch, boxes = refined.binary()
    codes, sorted_ = refined.morton()
    p = verts["p"]
    tri = np.stack([p[faces["a"]], p[faces["b"]], p[faces["c"]]], axis=1)
    leaf_lo, leaf_hi = tri.min(axis=1)[sorted_], tri.max(axis=1)[sorted_]

    def box(c):
        return (boxes[c, :3], boxes[c, 3:]) if c >= 0 else (leaf_lo[-c - 1], leaf_hi[-c - 1])
    for i in range(len(ch)):
        (l0, h0), (l1, h1) = box(ch[i, 0]), box(ch[i, 1])
        assert np.array_equal(boxes[i, :3], np.minimum(l0, l1)) and np.array_equal(boxes[i, 3:], np.maximum(h0, h1))
