"""Ideal glass and mirrors in the FP64 oracle (CPU): the reference's DIELECTRIC and GLOSSY types
(sample_bsdf's delta branches, main.swift:3318-3352) and the bounce loop's rules for them.

* The delta Cornell box renders finite images in RGB and spectral transport, with both samplers and in
  every sampling mode; its mean radiance differs from the same box with those slots Lambert.
* A thin film on the mirror changes the spectral image (the reference's film over metal, through
  oracle/_ref), and leaves the RGB image alone (the film is a spectral-transport input).
* A GLOSSY slot of roughness 0.3 takes the OpenPBR BSDF with metalness 1: it renders as an OPENPBR slot
  of the same colour, roughness and metalness 1.
"""
import numpy as np
import pytest

from metal_vibe_tracer_b200 import scenes, spectral_tables
from oracle import openpbr_ref as R

needs_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref/libopenpbr_ref.so is not built")


@needs_ref
@pytest.mark.parametrize("spectral,sampler,mode", [(False, 0, 1), (True, 0, 1), (False, 1, 1), (False, 0, 0),
                                                   (False, 0, 2), (False, 0, 3)])
def test_delta_cornell_renders(oracle, spectral, sampler, mode):
    faces, verts, mats, light, cam = scenes.cornell_delta(film=spectral)
    tables = spectral_tables.load() if spectral else None
    img = oracle.render(faces, verts, mats, light, cam, 32, 32, 8, max_depth=8, spectral=tables, sampler=sampler, mode=mode)
    assert np.isfinite(img).all() and img.mean() > 0.0


@needs_ref
def test_delta_slots_change_the_mean():
    from oracle import vt_oracle as O
    faces, verts, mats, light, cam = scenes.cornell_delta()
    ref = O.render(faces, verts, mats, light, cam, 64, 64, 32, max_depth=8).reshape(-1, 3).mean(0)
    lam = O.render(faces, verts, [dict(m, type=0) if m["type"] in (1, 2) else m for m in mats], light, cam, 64, 64, 32,
                   max_depth=8).reshape(-1, 3).mean(0)
    assert np.abs(lam / ref - 1).max() > 0.06, (lam, ref)


@needs_ref
def test_mirror_film_is_spectral_only(oracle):
    faces, verts, mats, light, cam = scenes.cornell_delta(film=True)
    bare = [dict(m, thin_film_weight=0.0) for m in mats]
    tables = spectral_tables.load()
    a = oracle.render(faces, verts, mats, light, cam, 32, 32, 8, max_depth=8, spectral=tables)
    b = oracle.render(faces, verts, bare, light, cam, 32, 32, 8, max_depth=8, spectral=tables)
    assert np.abs(a - b).max() > 1e-3
    a = oracle.render(faces, verts, mats, light, cam, 32, 32, 8, max_depth=8)
    b = oracle.render(faces, verts, bare, light, cam, 32, 32, 8, max_depth=8)
    assert np.array_equal(a, b)


@needs_ref
def test_rough_glossy_is_openpbr_metal(oracle):
    faces, verts, mats, light, cam = scenes.cornell_delta()
    as_pbr = [dict(m, type=4, metalness=1.0) if m["type"] == 1 and m["roughness"] >= 0.02 else m for m in mats]
    a = oracle.render(faces, verts, mats, light, cam, 32, 32, 8, max_depth=8)
    b = oracle.render(faces, verts, as_pbr, light, cam, 32, 32, 8, max_depth=8)
    assert np.array_equal(a, b)
