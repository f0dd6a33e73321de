"""OpenPBR (CPU): the reference's own BSDF, compiled from its vendored headers into oracle/_ref,
against the committed golden fixtures, and the FP64 oracle path tracer on OPENPBR slots.

The fixtures (tests/golden/openpbr_cases.json, metal_energy.json) were written from that library
by tests/golden/make_openpbr_golden.py; the CUDA restatement is checked against them on the B200
(tests/test_gpu_openpbr.py). Without the reference checkout the library cannot be built and the
checks that call it are skipped.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from metal_vibe_tracer_b200 import scenes
from oracle import openpbr_ref as R

GOLDEN = Path(__file__).resolve().parent / "golden"
needs_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref/libopenpbr_ref.so is not built")


@needs_ref
def test_reference_bsdf_reproduces_the_fixtures():
    cases = json.loads((GOLDEN / "openpbr_cases.json").read_text())["cases"]
    for c in cases[:200]:
        m = R.material(c["base"], c["metalness"], c["roughness"], c["ior"])
        f, pdf = R.evaluate(m, c["normal"], c["view"], c["light"])
        assert np.array_equal(f, np.float32(c["f_cos"])) and pdf == np.float32(c["pdf"])
        d, w, spdf, lobe = R.sample(m, c["normal"], c["view"], c["rand"])
        assert np.array_equal(d, np.float32(c["dir"])) and spdf == np.float32(c["sample_pdf"]) and lobe == c["lobe"]


@needs_ref
def test_reference_thin_film_reproduces_the_fixtures():
    """The thin-film fixtures (tests/golden/openpbr_thin_film_cases.json): iridescence at the case's
    three wavelengths (openpbr_thin_film_and_base_reflectance)."""
    cases = json.loads((GOLDEN / "openpbr_thin_film_cases.json").read_text())["cases"]
    for c in cases[:150]:
        m = R.material(c["base"], c["metalness"], c["roughness"], c["ior"], thin_film=c["thin_film"])
        f, pdf = R.evaluate(m, c["normal"], c["view"], c["light"], c["lambda"])
        assert np.array_equal(f, np.float32(c["f_cos"])) and pdf == np.float32(c["pdf"])
        d, w, spdf, lobe = R.sample(m, c["normal"], c["view"], c["rand"], c["lambda"])
        assert np.array_equal(d, np.float32(c["dir"])) and spdf == np.float32(c["sample_pdf"]) and lobe == c["lobe"]


@needs_ref
def test_reference_coat_reproduces_the_fixtures():
    """The coated fixtures (tests/golden/openpbr_coat_cases.json): the adapter's coat (roughness 0.12,
    IOR 1.6) at weights up to 1, some over a thin film, some seen from behind."""
    cases = json.loads((GOLDEN / "openpbr_coat_cases.json").read_text())["cases"]
    for c in cases[:150]:
        film = c["thin_film"] if c["thin_film"][0] > 0.0 else None
        m = R.material(c["base"], c["metalness"], c["roughness"], c["ior"], thin_film=film, coat=c["coat"])
        f, pdf = R.evaluate(m, c["normal"], c["view"], c["light"], c["lambda"])
        assert np.array_equal(f, np.float32(c["f_cos"])) and pdf == np.float32(c["pdf"])
        d, w, spdf, lobe = R.sample(m, c["normal"], c["view"], c["rand"], c["lambda"])
        assert np.array_equal(d, np.float32(c["dir"])) and spdf == np.float32(c["sample_pdf"]) and lobe == c["lobe"]


@needs_ref
def test_reference_fuzz_reproduces_the_fixtures():
    """The fuzzed fixtures (tests/golden/openpbr_fuzz_cases.json): the default fuzz (roughness 0.5,
    white) at weights up to 1, half of them under a coat."""
    cases = json.loads((GOLDEN / "openpbr_fuzz_cases.json").read_text())["cases"]
    for c in cases[:150]:
        m = R.material(c["base"], c["metalness"], c["roughness"], c["ior"], coat=c["coat"], fuzz=c["fuzz"])
        f, pdf = R.evaluate(m, c["normal"], c["view"], c["light"])
        assert np.array_equal(f, np.float32(c["f_cos"])) and pdf == np.float32(c["pdf"])
        d, w, spdf, lobe = R.sample(m, c["normal"], c["view"], c["rand"])
        assert np.array_equal(d, np.float32(c["dir"])) and spdf == np.float32(c["sample_pdf"]) and lobe == c["lobe"]


@needs_ref
def test_reference_anisotropy_reproduces_the_fixtures():
    """The anisotropic fixtures (tests/golden/openpbr_aniso_cases.json): specular_roughness_anisotropy
    about a unit tangent perpendicular to the normal, a third coated and a sixth fuzzed. The
    anisotropy changes the answer, and so does turning the tangent about the normal."""
    cases = json.loads((GOLDEN / "openpbr_aniso_cases.json").read_text())["cases"]
    changed = turned = 0
    for c in cases[:150]:
        args = (c["base"], c["metalness"], c["roughness"], c["ior"])
        m = R.material(*args, coat=c["coat"], fuzz=c["fuzz"], anisotropy=c["anisotropy"], tangent=c["tangent"])
        f, pdf = R.evaluate(m, c["normal"], c["view"], c["light"])
        assert np.array_equal(f, np.float32(c["f_cos"])) and pdf == np.float32(c["pdf"])
        d, w, spdf, lobe = R.sample(m, c["normal"], c["view"], c["rand"])
        assert np.array_equal(d, np.float32(c["dir"])) and spdf == np.float32(c["sample_pdf"]) and lobe == c["lobe"]
        iso = R.material(*args, coat=c["coat"], fuzz=c["fuzz"])
        changed += not np.allclose(R.evaluate(iso, c["normal"], c["view"], c["light"])[0], f, rtol=1e-2, atol=1e-6)
        bitangent = np.cross(np.float32(c["normal"]), np.float32(c["tangent"]))
        rot = R.material(*args, coat=c["coat"], fuzz=c["fuzz"], anisotropy=c["anisotropy"], tangent=bitangent)
        turned += not np.allclose(R.evaluate(rot, c["normal"], c["view"], c["light"])[0], f, rtol=1e-2, atol=1e-6)
    assert changed > 40 and turned > 40, (changed, turned)


@needs_ref
def test_oracle_renders_anisotropic_slots(oracle):
    """Anisotropic slots take their tangent from each triangle's first edge: the image changes with
    the anisotropy and stays finite."""
    faces, verts, mats, light, cam = scenes.cornell_openpbr()
    aniso = [dict(m, anisotropy=1.0) if m["type"] == 4 else m for m in mats]
    a = oracle.render(faces, verts, aniso, light, cam, 24, 24, 8, max_depth=4)
    b = oracle.render(faces, verts, mats, light, cam, 24, 24, 8, max_depth=4)
    assert np.isfinite(a).all() and a.mean() > 0.0
    assert not np.allclose(a, b)


@needs_ref
def test_reference_thin_film_changes_the_answer():
    """A film of weight 1 changes f |cos| on most cases; weight 0 gives the film-free answer."""
    cases = json.loads((GOLDEN / "openpbr_thin_film_cases.json").read_text())["cases"]
    changed = 0
    for c in cases[:60]:
        bare = R.material(c["base"], c["metalness"], c["roughness"], c["ior"])
        off = R.material(c["base"], c["metalness"], c["roughness"], c["ior"], thin_film=(0.0,) + tuple(c["thin_film"][1:]))
        f0, _ = R.evaluate(bare, c["normal"], c["view"], c["light"], c["lambda"])
        f1, _ = R.evaluate(off, c["normal"], c["view"], c["light"], c["lambda"])
        assert np.array_equal(f0, f1)
        changed += not np.allclose(f0, np.float32(c["f_cos"]), rtol=1e-2, atol=1e-6)
    assert changed > 20, changed


@needs_ref
def test_reference_metal_table_is_the_fixture():
    g = json.loads((GOLDEN / "metal_energy.json").read_text())
    t, a = R.metal_energy_table()
    assert np.array_equal(t[::8, ::8], np.float32(g["table"])) and np.array_equal(a, np.float32(g["average"]))


def test_fixture_cases_are_sane():
    """The reference's answers: f |cos|, pdfs and sampled weights nonnegative and finite, most
    samples valid (single samples of the one-sample MIS aggregate may weigh above one; the furnace
    test below bounds their mean)."""
    cases = json.loads((GOLDEN / "openpbr_cases.json").read_text())["cases"]
    fc = np.array([c["f_cos"] for c in cases])
    w = np.array([c["weight"] for c in cases])
    assert (fc >= 0).all() and all(c["pdf"] >= 0 for c in cases)
    ok = np.array([c["sample_pdf"] > 0 for c in cases])
    assert ok.mean() > 0.8
    assert np.isfinite(w[ok]).all() and (w[ok] >= 0).all()


@needs_ref
def test_reference_bsdf_is_energy_conserving():
    """White furnace: the mean sampled weight of a white metal and a white dielectric over diffuse
    stays below one and near it."""
    rng = np.random.default_rng(5)
    wo = [0.3, 0.0, 0.9539392]
    for metal in (0.0, 1.0):
        m = R.material([0.95, 0.95, 0.95], metal, 0.4, 1.5)
        acc = np.mean([R.sample(m, [0, 0, 1], wo, rng.random(3) * 0.9999)[1] for _ in range(4000)], axis=0)
        assert 0.85 < acc.min() and acc.max() < 1.0, acc


@needs_ref
def test_oracle_renders_openpbr_slots(oracle):
    faces, verts, mats, light, cam = scenes.cornell_openpbr()
    img = oracle.render(faces, verts, mats, light, cam, 24, 24, 8, max_depth=4)
    assert np.isfinite(img).all() and img.mean() > 0.0
    lambert = [dict(m, type=0) if m["type"] == 4 else m for m in mats]
    base = oracle.render(faces, verts, lambert, light, cam, 24, 24, 8, max_depth=4)
    assert not np.allclose(img, base)
