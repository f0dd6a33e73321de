"""Emitter-triangle lights on the B200: power sampling and the light tree.

The reference's own check (tests/Fix_light-tree.swift:38-176) restated on the device through
vt_light_estimate: a ceiling of small emitters (a 24 x 24 grid facing down in two emission slots, a
row facing up), 1024 threads x 64 light samples at each of five receivers. Per receiver:
* light samples and BSDF hits on the sampled triangle agree on the emitter pdf (no zero pdf,
  relative difference below 1e-3), for the tree and for power sampling;
* both selections estimate the emitted luminance of a quadrature reference (20 x 20 sub-triangles
  per emitter) within 5 standard errors + 1e-3;
* the tree rarely (<= 1 %) chooses an emitter facing away from the receiver, and lowers the variance
  below half of power sampling's where nearby lights dominate (receivers 1, 3, 4);
* one lamp (coincident triangles) renders through power sampling without a tree; eight separate
  lights build one.
Then images of an imported Cornell box lit by 36 emitter triangles against the FP64 oracle, with the
emitter list compared word for word with the oracle's restatement.
"""
import numpy as np
import pytest

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import scenes, spectral_tables
from oracle import light_tree as LT

pytestmark = pytest.mark.gpu

POINTS = np.array([(0, 0, 0), (-22, 0, -22), (15, 0.5, 5), (-3, 2.5, 7), (0, 5, 0)], np.float32)
PER_POINT, SAMPLES = 1024, 64
MEAN_REL = 1e-3


def quadrature(faces, verts, mats, p, k=20):
    """Luminance the front faces send to p (L cos_l / d^2 dA), 2 k^2 sub-triangle centroids."""
    pts = verts["p"].astype(np.float64)
    a, b, c = pts[faces["a"]], pts[faces["b"]], pts[faces["c"]]
    cr = np.cross(b - a, c - a)
    area = 0.5 * np.linalg.norm(cr, axis=1)
    n = cr / np.linalg.norm(cr, axis=1, keepdims=True)
    lum = np.array([0.2126 * m["emission"][0] + 0.7152 * m["emission"][1] + 0.0722 * m["emission"][2]
                    for m in mats])[faces["tag"]]
    uv = []
    for i in range(k):
        for j in range(k - i):
            for du, dv in ((1 / 3, 1 / 3), (2 / 3, 2 / 3)):
                if i + du + j + dv <= k:
                    uv.append(((i + du) / k, (j + dv) / k))
    uv = np.array(uv)
    q = a[:, None] + (b - a)[:, None] * uv[None, :, :1] + (c - a)[:, None] * uv[None, :, 1:]
    d = np.asarray(p, np.float64)[None, None] - q
    d2 = np.sum(d * d, -1)
    cos = np.maximum(0.0, np.sum(n[:, None] * d, -1) / np.sqrt(d2))
    return float(np.sum(lum[:, None] * cos / d2 * (area / (k * k))[:, None]))


def estimates(ctx, faces, verts, mats, tree):
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, None, light_tree=tree)
    out = scene.light_estimate(POINTS, PER_POINT, SAMPLES).reshape(len(POINTS), PER_POINT, 8)
    words = scene.emitter_words()
    scene.close()
    mesh.close()
    n = PER_POINT * SAMPLES
    res = []
    for k in range(len(POINTS)):
        o = out[k].astype(np.float64)
        mean = o[:, 0].sum() / n
        res.append({"mean": mean, "var": max(0.0, o[:, 1].sum() / n - mean * mean), "hits": o[:, 2].sum(),
                    "zero": o[:, 3].sum(), "error": o[:, 4].max(), "back": o[:, 5].sum()})
    return res, words


def test_ceiling_light_selection(ctx):
    faces, verts, mats = scenes.ceiling_lights()
    power, wp = estimates(ctx, faces, verts, mats, False)
    tree, wt = estimates(ctx, faces, verts, mats, True)
    ids, em = LT.scene_emitters(faces, verts, mats)
    assert np.array_equal(wt, LT.emitter_list(ids, em, True))
    assert np.array_equal(wp, LT.emitter_list(ids, em, False))
    assert wt[2 * len(faces) + 2] > 0 and wp[2 * len(faces) + 2] == 0
    n = PER_POINT * SAMPLES
    for k, p in enumerate(POINTS):
        t, w = tree[k], power[k]
        exact = quadrature(faces, verts, mats, p)
        assert t["zero"] == 0 and t["error"] < 1e-3 and w["zero"] == 0 and w["error"] < 1e-3, (k, t, w)
        assert exact == 0 or t["hits"] > 1000, (k, t)
        se_t, se_w = np.sqrt(t["var"] / n), np.sqrt(w["var"] / n)
        assert abs(t["mean"] - exact) <= 5 * se_t + 1e-3 * exact, (k, t["mean"], exact, se_t)
        assert abs(w["mean"] - exact) <= 5 * se_w + 1e-3 * exact, (k, w["mean"], exact, se_w)
        assert t["back"] <= 0.01 * n, (k, t["back"])
    for k in (1, 3, 4):
        assert tree[k]["var"] < 0.5 * power[k]["var"], (k, tree[k]["var"], power[k]["var"])


def test_lamp_uses_power_sampling_and_eight_lights_a_tree(ctx):
    faces, verts, mats = scenes.lamp()
    res, words = estimates(ctx, faces, verts, mats, True)
    assert int(words[0]) == 6 and words[2 * 6 + 2] == 0
    assert all(r["zero"] == 0 and r["error"] < 1e-3 for r in res)
    faces, verts, mats = scenes.ceiling_lights()
    res, words = estimates(ctx, faces[:8], verts, mats, True)
    assert words[2 * 8 + 2] > 1
    assert all(r["zero"] == 0 and r["error"] < 1e-3 for r in res)


def relmse(a, b):
    return float(np.mean((a - b) ** 2 / (b ** 2 + 1e-2)))


@pytest.mark.parametrize("tree,spectral", [(True, True), (False, True), (True, False)])
def test_imported_cornell_matches_oracle(ctx, oracle, tree, spectral):
    faces, verts, mats, cam = scenes.cornell_emitters()
    tables = spectral_tables.load() if spectral else None
    mesh = vt.Mesh(ctx, faces, verts)
    scene = vt.Scene(ctx, mesh, mats, None, tables, light_tree=tree)
    ids, em = LT.scene_emitters(faces, verts, mats)
    assert np.array_equal(scene.emitter_words(), LT.emitter_list(ids, em, tree))
    scene.render(vt.make_params(cam, 128, 128, 8, 1, spectral), 16)
    gpu, n = scene.readback()
    scene.close()
    mesh.close()
    assert n == 16 and np.isfinite(gpu).all()
    ref = oracle.render(faces, verts, mats, None, cam, 128, 128, 16, spectral=tables, light_tree=tree)
    other = oracle.render(faces, verts, mats, None, cam, 128, 128, 16, first_sample=1001, spectral=tables,
                          light_tree=tree)
    gm, rm = gpu.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(gm / rm - 1) < MEAN_REL), (gm, rm)
    assert relmse(gpu, ref) < 0.25 * relmse(other, ref), (relmse(gpu, ref), relmse(other, ref))
    same = np.all(np.abs(gpu - ref) <= 1e-4 * np.maximum(np.abs(ref), 1e-3), axis=-1)
    assert same.mean() > 0.9, same.mean()
