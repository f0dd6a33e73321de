"""The integrator's oracle and tables against the reference's own checks (CPU only).

* Spectral tables: the restatement of scripts/generate_spectral_tables.py reproduces the
  reference generator's XYZ -> sRGB matrix, normalised D65 and wavelength inverse CDF
  (golden fixture tests/golden/spectral_360_830.json, written by make_spectral_golden.py).
* Integrator energy (tests/Fix_integrator.swift:188-215): on the Cornell box, light sampling agrees
  with MIS within 3 %, BSDF sampling within 12 %, ReSTIR DI within 6 %, and each depth adds light.
* Spectral transport of a grey scene under D65 converges to the RGB render (D65 is the sRGB white).
"""
import json
from pathlib import Path

import numpy as np
import pytest

from metal_vibe_tracer_b200 import scenes, spectral_tables

GOLDEN = Path(__file__).resolve().parent / "golden" / "spectral_360_830.json"
HAVE_CIE = spectral_tables.have_reference_data()


@pytest.mark.skipif(not HAVE_CIE, reason="CIE datasets are read from the reference checkout")
def test_spectral_tables_match_reference_generator():
    g = json.loads(GOLDEN.read_text())
    t = spectral_tables.compute(g["lambda_min"], g["lambda_max"])
    np.testing.assert_allclose(np.array(t["xyz_to_rgb"]), np.array(g["xyz_to_rgb"]), rtol=0, atol=1e-15)
    for lam, v in g["d65_normalized"].items():
        assert t["illum"][int(lam) - g["lambda_min"]] == pytest.approx(v, rel=1e-14)
    for lam, v in g["density"].items():
        assert t["density"][int(lam) - g["lambda_min"]] == pytest.approx(v, rel=1e-14)
    for i, v in g["icdf_nodes"].items():
        assert t["icdf"][int(i)] == pytest.approx(v, rel=1e-14)


@pytest.mark.skipif(not HAVE_CIE, reason="CIE datasets are read from the reference checkout")
def test_render_range_tables():
    t = spectral_tables.compute(380, 780)
    cmf = np.array(t["cmf_rgb"])
    white = (cmf * np.array(t["illum"])[:, None]).sum(0)
    np.testing.assert_allclose(white, 1.0, atol=1e-12)   # D65 is the sRGB white
    icdf = np.array(t["icdf"])
    assert icdf[0] == 380 and icdf[-1] == 780 and np.all(np.diff(icdf) > 0) and len(icdf) == 1025


def spectral():
    if not spectral_tables.path().exists():
        if not HAVE_CIE:
            pytest.skip("no spectral tables")
        spectral_tables.generate()
    return spectral_tables.load()


def test_integrator_energy_reference_protocol(oracle):
    faces, verts, mats, light, cam = scenes.cornell_box()
    prev = 0.0
    for depth in (1, 2, 3):
        mis = oracle.render(faces, verts, mats, light, cam, 48, 32, 256, max_depth=depth, mode=1).mean()
        nee = oracle.render(faces, verts, mats, light, cam, 48, 32, 256, max_depth=depth, mode=2).mean()
        bsdf = oracle.render(faces, verts, mats, light, cam, 48, 32, 256, max_depth=depth, mode=3).mean()
        restir = oracle.render(faces, verts, mats, light, cam, 48, 32, 256, max_depth=depth, mode=0).mean()
        assert abs(nee / mis - 1) < 0.03 and abs(bsdf / mis - 1) < 0.12, (depth, mis, nee, bsdf)
        assert abs(restir / mis - 1) < 0.06, (depth, mis, restir)
        assert mis > prev
        prev = mis


def test_spectral_grey_scene_converges_to_rgb(oracle):
    faces, verts, mats, light, cam = scenes.cornell_box()
    rgb = oracle.render(faces, verts, mats, light, cam, 64, 64, 64).reshape(-1, 3).mean(0)
    spec = oracle.render(faces, verts, mats, light, cam, 64, 64, 64, spectral=spectral()).reshape(-1, 3).mean(0)
    np.testing.assert_allclose(spec, rgb, rtol=0.01)


def test_camera_sees_the_emitter(oracle):
    """RGB transport returns the emitter's radiance; spectral transport its four-wavelength estimate
    (emitter_rgb, main.swift:7467-7468), whose mean over the emitter's pixels is the radiance (D65
    is the sRGB white)."""
    faces, verts, mats, light, cam = scenes.cornell_box()
    rgb = oracle.render(faces, verts, mats, light, cam, 256, 256, 64)
    assert rgb.max() == pytest.approx(17.0)
    lit = np.all(rgb == 17.0, axis=-1)   # every sample of these pixels sees the emitter
    assert lit.sum() >= 20
    img = oracle.render(faces, verts, mats, light, cam, 256, 256, 64, spectral=spectral())
    np.testing.assert_allclose(img[lit].mean(0), 17.0, rtol=0.02)
    assert np.isfinite(img).all()


def test_imported_scene_tree_and_power_agree(oracle):
    """Light-tree and power selection estimate the same image of the emitter-lit Cornell box, and,
    without the wall lamps, the same image as the quad light (LightTree: unbiased selection)."""
    faces, verts, mats, cam = scenes.cornell_emitters()
    a = oracle.render(faces, verts, mats, None, cam, 48, 32, 256, light_tree=True)
    b = oracle.render(faces, verts, mats, None, cam, 48, 32, 256, light_tree=False)
    assert abs(a.mean() / b.mean() - 1) < 0.02
    faces, verts, mats, cam = scenes.cornell_emitters(lamps=False)
    c = oracle.render(faces, verts, mats, None, cam, 48, 32, 256)
    qf, qv, qm, light, _ = scenes.cornell_box()
    d = oracle.render(qf, qv, qm, light, cam, 48, 32, 256)
    assert abs(c.mean() / d.mean() - 1) < 0.02


def test_smooth_normals_shade_the_sphere(oracle):
    """Vertex normals change the sphere's shading (mesh_hit_attributes) but not the energy balance."""
    faces, verts, mats, light, cam = scenes.cornell_sphere()
    smooth = oracle.render(faces, verts, mats, light, cam, 64, 64, 64)
    flat_verts = verts.copy()
    flat_verts["n"] = 0.0
    flat = oracle.render(faces, flat_verts, mats, light, cam, 64, 64, 64)
    # Same sample streams: only the sphere's pixels (and what they light) differ.
    assert np.count_nonzero(np.abs(smooth - flat).max(-1) > 1e-6) > 100
    assert abs(smooth.mean() / flat.mean() - 1) < 0.05
