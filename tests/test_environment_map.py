"""The environment image's sampling tables (vt_environment_tables, the host step of
vt_scene_set_environment_map) against a plain restatement of MaterialLibrary.environmentImportance
(Sources/StudioModel.swift:1300-1392) in float32 loops (CPU only): dilated luminance, the compensated
table max(0, L - mean L) sin(theta) and the original L sin(theta), normalised to CDFs whose last
entry is 1; a uniform map samples its luminance in both tables."""
import math

import numpy as np

from metal_vibe_tracer_b200 import scenes
from metal_vibe_tracer_b200.render import environment_tables


def restated_tables(img):
    h, w = img.shape[:2]
    f = np.float32
    lum = np.maximum(f(1e-6), f(0.2126) * img[..., 0] + f(0.7152) * img[..., 1] + f(0.0722) * img[..., 2]).astype(f)
    hor = np.maximum(lum, np.maximum(np.roll(lum, 1, axis=1), np.roll(lum, -1, axis=1)))
    mean_sum = angle_sum = 0.0
    pi = f(3.14159265)
    for y in range(h):
        st = float(max(f(1e-4), f(math.sin(f(pi * (f(y) + f(0.5))) / f(h)))))
        mean_sum += float(np.sum(lum[y].astype(np.float64))) * st
        angle_sum += st * w
    mean = f(mean_sum / angle_sum)
    rows = np.zeros((h, 2), f)
    cols = np.zeros((2, h, w), f)
    for y in range(h):
        st = max(f(1e-4), f(math.sin(f(pi * (f(y) + f(0.5))) / f(h))))
        dil = np.maximum(hor[max(y - 1, 0)], np.maximum(hor[y], hor[min(y + 1, h - 1)]))
        comp = (np.maximum(f(0), dil - mean) * st).astype(f)
        orig = (dil * st).astype(f)
        cols[0, y], cols[1, y] = comp, orig
        rows[y, 0] = np.sum(comp, dtype=np.float64)
        rows[y, 1] = np.sum(orig, dtype=np.float64)
    if not cols[0].sum() > 0:
        rows[:, 0], cols[0] = rows[:, 1], cols[1]

    def cdf(wt):
        total = max(float(np.sum(wt, dtype=np.float64)), 1e-12)
        c = np.cumsum(wt.astype(np.float64)) / total
        c[-1] = 1.0
        return c

    rc = np.stack([cdf(rows[:, t]) for t in range(2)], 1)
    cc = np.stack([[cdf(cols[t, y]) for y in range(h)] for t in range(2)])
    return rc, cc


def test_tables_match_restatement():
    img = scenes.environment_image(32, 16)
    rows, cols = environment_tables(img)
    rr, cc = restated_tables(img)
    # The library sums in float in the reference's order; the restatement in double: CDFs agree to
    # float rounding.
    np.testing.assert_allclose(rows, rr, atol=2e-6)
    np.testing.assert_allclose(cols, cc, atol=2e-6)
    assert np.all(np.diff(rows, axis=0) >= 0) and np.all(np.diff(cols, axis=2) >= 0)
    assert np.all(rows[-1] == 1.0) and np.all(cols[..., -1] == 1.0)
    # The compensated table leaves the texels at or below the mean to BSDF sampling.
    comp_cells = np.diff(np.concatenate([np.zeros((16, 1), np.float32), cols[0]], axis=1), axis=1)
    orig_cells = np.diff(np.concatenate([np.zeros((16, 1), np.float32), cols[1]], axis=1), axis=1)
    assert (comp_cells == 0).sum() > (orig_cells == 0).sum()


def test_uniform_map_samples_luminance_in_both_tables():
    img = np.ones((8, 16, 4), np.float32)
    rows, cols = environment_tables(img)
    np.testing.assert_array_equal(rows[:, 0], rows[:, 1])
    np.testing.assert_array_equal(cols[0], cols[1])
    # Rows weighted by sin(theta), columns uniform.
    np.testing.assert_allclose(cols[1, 3], (np.arange(16) + 1) / 16.0, atol=1e-6)
