"""Spectral transport tables: CIE 1931 CMFs as linear sRGB, the D65 illuminant and the wavelength
inverse CDF (restating scripts/generate_spectral_tables.py: `Data` :142-181, `sampling_density`
:490-500, `inverse_cdf` :510-530).

The CIE datasets are CC BY-SA 4.0 and are not part of this repository. `generate()` reads them
at build time from the reference's vendored copies (Vendor/Spectral/CIE) and writes the derived
tables to `data/spectral_<lo>_<hi>.bin` (git-ignored, shipped with the built library); `load()`
reads that file at run time. Every table is a 1 nm table over [lambda_min, lambda_max]:

* cmf_rgb[i]  linear-sRGB colour-matching functions M xyz(lambda_i), with M the XYZ -> linear sRGB
              matrix whose white point is the computed XYZ of D65 (so D65 maps to rgb (1, 1, 1));
* illum[i]    D65, normalised to luminance Y = 1 (1 nm sums over the range);
* icdf[n]     1025 nodes: lambda at u = n / 1024 of the piecewise-linear density
              0.9 D65 s / int(D65 s) + 0.1 s / int(s), s = |r| + |g| + |b| of the sRGB CMFs.

The renderer's default range is 380-780 nm (the traversal-path configs ask for four hero
wavelengths over 380-780 nm); the reference tabulates 360-830 nm, which `generate(360, 830)`
reproduces for the golden-vector check.

RGB -> spectrum uplift (scripts/generate_spectral_tables.py `Data` :142-181; main.swift:842-907): a
bounded colour's reflectance is the bounded MESE of three trigonometric moments on Peters' even XYZ
phase warp (Peters et al. 2019). The file also holds what the device needs to solve the moment grid
and to evaluate reflectances:

* uplift_w[i]   per nm over 360-830 (always that range, the colour model's): linear-sRGB CMFs times
                D65 normalised to Y = 1, float64 (reflectance -> linear sRGB is sum_i uplift_w[i] g_i);
* uplift_cos[i] cos(phi(lambda_i)) over 360-830, float64, phi the warp (XYZWarp.h
                applyXYZWarpEven: piecewise linear in 5 nm steps over 95 nodes);
* cos_phase[i]  cos(phi) at the render range's 1 nm bins, float32.

The warp's 95 nodes come from the reference's vendored copy of Peters' BSD code
(Vendor/Spectral/Peters2019/XYZWarp.h), read at build time like the CIE data.
"""
from __future__ import annotations

import csv
import math
import os
import struct
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
DATA_DIR = PKG / "data"
REFERENCE_ENV = "VT_REFERENCE_ROOT"


def reference_root() -> Path | None:
    """The checkout of the reference (gabinfor/metal-vibe-tracer) whose vendored data the build-time
    generators read, from the VT_REFERENCE_ROOT environment variable; None when it is unset. The
    build recipe (__graft_entry__.build) and the test set-up give it their default checkout path when
    unset. Run-time code never reads the reference: it loads the generated files under data/."""
    v = os.environ.get(REFERENCE_ENV)
    return Path(v) if v else None


def reference_cie() -> Path | None:
    r = reference_root()
    return r / "Vendor" / "Spectral" / "CIE" if r else None


def reference_warp() -> Path | None:
    r = reference_root()
    return r / "Vendor" / "Spectral" / "Peters2019" / "XYZWarp.h" if r else None


def have_reference_data() -> bool:
    c = reference_cie()
    return c is not None and (c / "CIE_xyz_1931_2deg.csv").exists()


def _need(path: Path | None, what: str) -> Path:
    if path is None:
        raise RuntimeError(f"{what}: set {REFERENCE_ENV} to the reference checkout (its vendored data is read at build time)")
    return path
UPLIFT_MIN, UPLIFT_MAX = 360, 830
SRGB_PRIMARIES = ((0.64, 0.33), (0.30, 0.60), (0.15, 0.06))
ICDF_SEGMENTS = 1024
DEFENSIVE = 0.1
MAGIC = b"VTSPEC02"


def _read(path: Path):
    with open(path, newline="") as f:
        return [[float(v) for v in row] for row in csv.reader(f) if row]


def _resample(rows, col, wavelengths):
    pts = [(r[0], r[col]) for r in rows]
    out, j = [], 0
    for lam in wavelengths:
        if lam < pts[0][0] or lam > pts[-1][0]:
            out.append(0.0)
            continue
        while pts[j + 1][0] < lam:
            j += 1
        (x0, y0), (x1, y1) = pts[j], pts[j + 1]
        out.append(y0 + (y1 - y0) * (lam - x0) / (x1 - x0))
    return out


def _inv3(m):
    (a, b, c), (d, e, f), (g, h, i) = m
    det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g)
    return [[(e * i - f * h) / det, (c * h - b * i) / det, (b * f - c * e) / det],
            [(f * g - d * i) / det, (a * i - c * g) / det, (c * d - a * f) / det],
            [(d * h - e * g) / det, (b * g - a * h) / det, (a * e - b * d) / det]]


def _apply(m, v):
    return [m[r][0] * v[0] + m[r][1] * v[1] + m[r][2] * v[2] for r in range(3)]


def compute(lambda_min: int, lambda_max: int, cie_dir: Path | None = None) -> dict:
    cie_dir = _need(cie_dir or reference_cie(), "CIE datasets")
    """All tables in float64 (lists), from the CIE CSVs."""
    wl = list(range(lambda_min, lambda_max + 1))
    cmf_rows = _read(cie_dir / "CIE_xyz_1931_2deg.csv")
    cmf = [tuple(r[1:4]) for r in cmf_rows if lambda_min <= r[0] <= lambda_max]
    assert len(cmf) == len(wl)
    spd = _resample(_read(cie_dir / "CIE_std_illum_D65.csv"), 1, wl)
    y = sum(s * c[1] for s, c in zip(spd, cmf))
    d65 = [s / y for s in spd]
    white = [sum(s * c[k] for s, c in zip(d65, cmf)) for k in range(3)]
    primaries = [[x / yy for x, yy in SRGB_PRIMARIES], [1.0, 1.0, 1.0],
                 [(1 - x - yy) / yy for x, yy in SRGB_PRIMARIES]]
    scale = _apply(_inv3(primaries), white)
    rgb_to_xyz = [[primaries[r][k] * scale[k] for k in range(3)] for r in range(3)]
    xyz_to_rgb = _inv3(rgb_to_xyz)
    cmf_rgb = [_apply(xyz_to_rgb, c) for c in cmf]
    s = [abs(v[0]) + abs(v[1]) + abs(v[2]) for v in cmf_rgb]

    def normalized(values):
        total = sum(0.5 * (values[i] + values[i + 1]) for i in range(len(values) - 1))
        return [v / total for v in values]
    a, b = normalized([p * q for p, q in zip(d65, s)]), normalized(s)
    density = [(1.0 - DEFENSIVE) * x + DEFENSIVE * yv for x, yv in zip(a, b)]
    icdf = inverse_cdf(density, lambda_min, lambda_max)
    return {"lambda_min": lambda_min, "lambda_max": lambda_max, "cmf_xyz": cmf, "cmf_rgb": cmf_rgb,
            "illum": d65, "icdf": icdf, "xyz_to_rgb": xyz_to_rgb, "density": density}


def read_warp(path: Path | None = None) -> list:
    path = _need(path or reference_warp(), "XYZ warp")
    """The 95 nodes of Peters' even XYZ phase warp (-pi at 360 nm ... 0 at 830 nm, 5 nm apart)."""
    text = path.read_text()
    key = "pXYZWarpEven[] = {"
    start = text.index(key) + len(key)
    values = [float(v.strip().rstrip("f")) for v in text[start:text.index("}", start)].split(",")]
    if len(values) != 95:
        raise RuntimeError(f"{path}: expected 95 warp nodes, found {len(values)}")
    return values


def warp_phase(warp, lam: float) -> float:
    """phi(lambda): linear between the 5 nm nodes (XYZWarp.h applyXYZWarpEven)."""
    t = (lam - 360.0) * 0.2
    i = min(max(int(math.floor(t)), 0), 93)
    f = t - i
    return warp[i] * (1.0 - f) + warp[i + 1] * f


def uplift_model(cie_dir: Path | None = None, warp_path: Path | None = None) -> dict:
    cie_dir = _need(cie_dir or reference_cie(), "CIE datasets")
    warp_path = _need(warp_path or reference_warp(), "XYZ warp")
    """The uplift's colour model over 360-830 nm in float64: per nm weights (rgb CMF x D65, Y = 1)
    and cos of the warped phase."""
    t = compute(UPLIFT_MIN, UPLIFT_MAX, cie_dir)
    w = [[c[k] * s for k in range(3)] for c, s in zip(t["cmf_rgb"], t["illum"])]
    warp = read_warp(warp_path)
    cos_phi = [math.cos(warp_phase(warp, lam)) for lam in range(UPLIFT_MIN, UPLIFT_MAX + 1)]
    return {"weights": w, "cos": cos_phi, "warp": warp}


def inverse_cdf(density, lambda_min, lambda_max, segments=ICDF_SEGMENTS):
    """Wavelengths at u = i / segments of the CDF of a piecewise-linear 1 nm density (exact)."""
    cdf = [0.0]
    for i in range(len(density) - 1):
        cdf.append(cdf[-1] + 0.5 * (density[i] + density[i + 1]))
    total = cdf[-1]
    out = [float(lambda_min)]
    j = 0
    for n in range(1, segments):
        yv = total * n / segments
        while cdf[j + 1] < yv:
            j += 1
        p0, p1, rest = density[j], density[j + 1], yv - cdf[j]
        dp = p1 - p0
        if abs(dp) < 1e-12 * max(p0, 1e-30):
            t = rest / p0
        else:
            t = (-p0 + math.sqrt(max(p0 * p0 + 2.0 * dp * rest, 0.0))) / dp
        out.append(lambda_min + j + min(max(t, 0.0), 1.0))
    out.append(float(lambda_max))
    for i in range(1, len(out)):
        if out[i] <= out[i - 1]:
            out[i] = math.nextafter(out[i - 1], math.inf)
    return out


def path(lambda_min: int = 380, lambda_max: int = 780) -> Path:
    return DATA_DIR / f"spectral_{lambda_min}_{lambda_max}.bin"


def generate(lambda_min: int = 380, lambda_max: int = 780, cie_dir: Path | None = None,
             warp_path: Path | None = None) -> Path:
    cie_dir = _need(cie_dir or reference_cie(), "CIE datasets")
    warp_path = _need(warp_path or reference_warp(), "XYZ warp")
    """Write the table file (build time; needs the CIE CSVs and the warp)."""
    t = compute(lambda_min, lambda_max, cie_dir)
    u = uplift_model(cie_dir, warp_path)
    n = lambda_max - lambda_min + 1
    DATA_DIR.mkdir(parents=True, exist_ok=True)
    out = path(lambda_min, lambda_max)
    blob = MAGIC + struct.pack("<iiii", lambda_min, lambda_max, n, ICDF_SEGMENTS)
    blob += np.asarray(t["cmf_rgb"], np.float32).tobytes()
    blob += np.asarray(t["illum"], np.float32).tobytes()
    blob += np.asarray(t["icdf"], np.float32).tobytes()
    blob += np.asarray(t["xyz_to_rgb"], np.float64).tobytes()
    blob += np.asarray(u["weights"], np.float64).tobytes()
    blob += np.asarray(u["cos"], np.float64).tobytes()
    cos_bins = [math.cos(warp_phase(u["warp"], float(lam))) for lam in range(lambda_min, lambda_max + 1)]
    blob += np.asarray(cos_bins, np.float32).tobytes()
    tmp = out.with_suffix(".tmp")
    tmp.write_bytes(blob)
    tmp.replace(out)
    return out


def load(lambda_min: int = 380, lambda_max: int = 780) -> dict:
    """float32 tables from the generated file (no CIE input needed)."""
    p = path(lambda_min, lambda_max)
    if not p.exists():
        raise RuntimeError(f"{p} is missing: it is generated at build time from the CIE datasets "
                           "(metal_vibe_tracer_b200.spectral_tables.generate)")
    b = p.read_bytes()
    if b[:8] != MAGIC:
        raise RuntimeError(f"{p}: bad header")
    lo, hi, n, seg = struct.unpack("<iiii", b[8:24])
    off = 24
    cmf_rgb = np.frombuffer(b, np.float32, 3 * n, off).reshape(n, 3); off += 12 * n
    illum = np.frombuffer(b, np.float32, n, off); off += 4 * n
    icdf = np.frombuffer(b, np.float32, seg + 1, off); off += 4 * (seg + 1)
    m = np.frombuffer(b, np.float64, 9, off).reshape(3, 3); off += 72
    nu = UPLIFT_MAX - UPLIFT_MIN + 1
    uw = np.frombuffer(b, np.float64, 3 * nu, off).reshape(nu, 3); off += 24 * nu
    uc = np.frombuffer(b, np.float64, nu, off); off += 8 * nu
    cos_phase = np.frombuffer(b, np.float32, n, off)
    return {"lambda_min": lo, "lambda_max": hi, "n": n, "segments": seg, "cmf_rgb": cmf_rgb.copy(),
            "illum": illum.copy(), "icdf": icdf.copy(), "xyz_to_rgb": m.copy(),
            "uplift_w": np.ascontiguousarray(uw), "uplift_cos": uc.copy(), "cos_phase": cos_phase.copy()}
