"""The RGB -> spectrum uplift's oracle against the reference's generator and known answers
(CPU; the GPU uplift is checked against this oracle in tests/test_gpu_uplift.py).

Known answers restated from tests/Fix_spectral.swift:143-369: D65 is the sRGB white, every 8-bit code
round-trips within half an 8-bit step through the runtime conversion (sampled here), white emission
is D65 exactly and upsampled emitters keep a nonnegative spectrum.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from metal_vibe_tracer_b200 import spectral_tables
from oracle import vt_oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "fourier_srgb_lines.json"


@pytest.fixture(scope="module")
def tables():
    return spectral_tables.load()


@pytest.fixture(scope="module")
def uplift(tables):
    O.load()
    u = O.Uplift(tables["uplift_w"], tables["uplift_cos"])
    yield u
    u.close()


def srgb_oetf(v):
    v = np.clip(v, 0.0, 1.0)
    return np.where(v <= 0.0031308, 12.92 * v, 1.055 * np.power(v, 1 / 2.4) - 0.055)


def srgb_eotf(v):
    return np.where(v <= 0.04045, v / 12.92, np.power((v + 0.055) / 1.055, 2.4))


def test_d65_is_the_srgb_white(tables):
    """A white reflectance under D65 is linear sRGB (1, 1, 1) (Fix_spectral.swift:162)."""
    assert np.abs(tables["uplift_w"].sum(0) - 1.0).max() < 1e-12
    assert tables["uplift_cos"][0] == pytest.approx(-1.0) and tables["uplift_cos"][-1] == pytest.approx(1.0)


def test_grid_lines_match_the_reference_generator(uplift):
    """86 nodes on each of 16 (r, g) lines of FourierSRGB86.bin, as the generator solves them."""
    g = json.loads(GOLDEN.read_text())
    worst = 0.0
    for line in g["lines"]:
        i, j = line["r"] // 3, line["g"] // 3
        ref = np.asarray(line["moments"]).reshape(86, 3)
        mine = np.array([uplift.node(i, j, k) for k in range(86)])
        worst = max(worst, np.abs(mine.astype(np.float32).astype(np.float64) - ref).max())
    assert worst < 2e-8, worst


def test_lagrange_matches_the_generators_levinson():
    g = json.loads(GOLDEN.read_text())
    for check in g["lagrange3"]:
        L = O.fourier_lagrange(check["moments"])
        assert np.allclose(L, check["lagrange"], rtol=1e-9, atol=1e-9), (L, check["lagrange"])


def test_exact_solve_reproduces_its_code(uplift):
    for code in ([255, 0, 0], [0, 255, 0], [12, 200, 90], [250, 250, 10], [3, 3, 240]):
        m, L, err = uplift.solve_code(code)
        assert err < 1e-9
        rgb = uplift.rgb_of_lagrange(L)
        target = np.clip(srgb_eotf(np.asarray(code) / 255.0), 1e-4, 1 - 1e-4)
        assert np.abs(rgb - target).max() < 1e-9
        # The moments of the reconstruction give the multipliers back.
        assert np.allclose(O.fourier_lagrange(m), L, rtol=1e-6, atol=1e-6)


def test_sampled_codes_round_trip_within_half_a_step(uplift):
    """Through the runtime conversion (grid interpolation, refined cells exact)."""
    rng = np.random.default_rng(7)
    codes = rng.integers(0, 256, (400, 3))
    codes[:6] = [[255, 0, 0], [0, 255, 0], [0, 0, 255], [0, 255, 255], [255, 0, 255], [255, 255, 0]]
    lin = srgb_eotf(codes / 255.0)
    L = uplift.lagrange(lin)
    worst = 0.0
    for c, l4 in zip(codes, L):
        rgb = l4[0] * np.ones(3) if l4[3] == 2.0 else uplift.rgb_of_lagrange(l4[:3])
        worst = max(worst, np.abs(srgb_oetf(rgb) * 255.0 - c).max())
    assert worst <= 0.5, worst


def test_refined_cells_are_the_badly_interpolated_ones(uplift):
    """Saturated corners' cells need exact blocks; a mid-grey cell does not."""
    assert uplift.cell_refined([42, 42, 42]) is False
    flagged = [uplift.cell_refined(c) for c in ([84, 0, 0], [0, 84, 0], [0, 0, 84], [84, 84, 0], [0, 84, 84])]
    assert any(flagged)
    assert uplift.code_error([128, 128, 128]) == 0.0


def test_reflectance_is_bounded_and_greys_are_flat(uplift, tables):
    x = tables["cos_phase"].astype(np.float64)
    for rgb in ([0.9, 0.1, 0.05], [0.05, 0.6, 0.1], [0.02, 0.03, 0.9], [0.5, 0.5, 0.5]):
        L = uplift.lagrange(rgb)[0]
        rho = O.reflectance(L, x)
        assert np.all(rho > 0.0) and np.all(rho < 1.0)
        if L[3] == 2.0:
            assert np.all(rho == 0.5)


def emission_weights(e):
    """spectral_emission_weights (main.swift:917-927), restated for the known-answer check."""
    e = np.maximum(np.asarray(e, np.float64), 0.0)
    hi, lo = e.max(), e.min()
    mid = e.sum() - hi - lo
    p = 0 if e[0] == hi else 1 if e[1] == hi else 2
    s = 2 if p != 2 and e[2] == lo else 1 if p != 1 and e[1] == lo else 0
    return lo, max(mid - lo, 0.0), max(hi - mid, 0.0), s, p


def test_upsampled_emitters_keep_their_colour(uplift, tables):
    """e = lo + secondary basis + primary basis, the basis the saturated corners' spectra: white is
    D65 exactly, colours come back within half an 8-bit step and spectra stay nonnegative
    (Fix_spectral.swift:80-96)."""
    corners = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 1, 1], [1, 0, 1], [1, 1, 0]], np.float64)
    Ls = uplift.lagrange(corners)
    x = tables["uplift_cos"]
    basis = np.stack([O.reflectance(L, x) for L in Ls])  # (6, 471): R G B C M Y
    w = tables["uplift_w"]
    for e in ([1.0, 1.0, 1.0], [0.8, 0.2, 0.1], [0.1, 0.9, 0.3], [0.2, 0.3, 0.95], [0.6, 0.6, 0.05]):
        lo, sec, pri, si, pi = emission_weights(e)
        spec = lo + sec * basis[3 + si] + pri * basis[pi]
        rgb = spec @ w
        assert spec.min() >= 0.0
        if e == [1.0, 1.0, 1.0]:
            assert np.abs(rgb - 1.0).max() < 1e-12
        assert np.abs(srgb_oetf(rgb) * 255 - srgb_oetf(np.asarray(e)) * 255).max() <= 0.5, (e, rgb)
