"""Writes tests/golden/openpbr_cases.json and tests/golden/metal_energy.json from the reference's
own OpenPBR BSDF (oracle/_ref/libopenpbr_ref.so, compiled from the reference's vendored Adobe
openpbr-bsdf headers and Shaders/MetalEnergy.metal by oracle/openpbr_ref/Makefile).

Cases: seeded opaque OPENPBR materials (base colour uniform, metalness 0, 1 or uniform, roughness
uniform in [0, 1] (the adapter clamps at 0.03), IOR uniform in [1.3, 1.8], specular weight 1),
random unit shading normals, views mostly on the normal's side (some behind it), light directions
uniform on the sphere and three uniform random numbers: each with the reference's f |cos| and pdf
at the light direction and its sample (direction, weight, pdf). The metal table: every 8th node of
the 129 x 129 table and all 129 averages. Thin-film cases (tests/golden/openpbr_thin_film_cases.json): the
same with thin-film iridescence (weight, thickness, film IOR) at three given wavelengths. Coated cases
(tests/golden/openpbr_coat_cases.json): the same with the adapter's coat (weight; roughness 0.12, IOR
1.6), a third of them with a thin film under it. Fuzzed cases (tests/golden/openpbr_fuzz_cases.json): the
same with the fuzz (weight; roughness 0.5, white), half of them under a coat as well. Anisotropic
cases (tests/golden/openpbr_aniso_cases.json): the same with specular_roughness_anisotropy in (0, 1]
about a unit tangent perpendicular to the normal (as the adapter's mat.tangent is), a third of them
coated and a sixth fuzzed.
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import openpbr_ref as R  # noqa: E402


def unit(v):
    return v / np.linalg.norm(v)


rng = np.random.default_rng(20261203)
cases = []
for i in range(600):
    base = rng.random(3)
    metal = [0.0, 1.0, float(rng.random())][i % 3]
    rough = float(rng.random())
    ior = float(1.3 + 0.5 * rng.random())
    n = unit(rng.normal(size=3))
    wo = unit(rng.normal(size=3))
    if (np.dot(wo, n) < 0) != (i % 10 == 9):
        wo = -wo
    wi = unit(rng.normal(size=3))
    if i % 4 != 3 and np.dot(wi, n) < 0:
        wi = -wi
    r = rng.random(3).astype(np.float32)
    f32 = lambda x: [float(v) for v in np.asarray(x, np.float32)]
    m = R.material(base, metal, rough, ior)
    f, pdf = R.evaluate(m, f32(n), f32(wo), f32(wi))
    d, w, spdf, lobe = R.sample(m, f32(n), f32(wo), f32(r))
    cases.append({"base": f32(base), "metalness": metal, "roughness": rough, "ior": ior, "normal": f32(n), "view": f32(wo),
                  "light": f32(wi), "rand": f32(r), "f_cos": f32(f), "pdf": float(pdf), "dir": f32(d), "weight": f32(w),
                  "sample_pdf": float(spdf), "lobe": lobe})
# Thin-film cases (their own stream, after the opaque ones): weight 1 or uniform, thickness uniform in
# [0, 1] micrometres (below 0.03 the film fades out), film IOR uniform in [1.2, 2.4], the three
# wavelengths uniform in [380, 780] nm, metalness 0, 1 or uniform.
rng = np.random.default_rng(20261204)
film_cases = []
for i in range(300):
    base = rng.random(3)
    metal = [0.0, 1.0, float(rng.random())][i % 3]
    rough = float(rng.random())
    ior = float(1.3 + 0.5 * rng.random())
    film = (1.0 if i % 2 == 0 else float(rng.random()), float(rng.random()), float(1.2 + 1.2 * rng.random()))
    lam = [float(x) for x in np.asarray(380.0 + 400.0 * rng.random(3), np.float32)]
    n = unit(rng.normal(size=3))
    wo = unit(rng.normal(size=3))
    if (np.dot(wo, n) < 0) != (i % 10 == 9):
        wo = -wo
    wi = unit(rng.normal(size=3))
    if i % 4 != 3 and np.dot(wi, n) < 0:
        wi = -wi
    r = rng.random(3).astype(np.float32)
    f32 = lambda x: [float(v) for v in np.asarray(x, np.float32)]
    m = R.material(base, metal, rough, ior, thin_film=film)
    f, pdf = R.evaluate(m, f32(n), f32(wo), f32(wi), lam)
    d, w, spdf, lobe = R.sample(m, f32(n), f32(wo), f32(r), lam)
    film_cases.append({"base": f32(base), "metalness": metal, "roughness": rough, "ior": ior, "normal": f32(n),
                       "view": f32(wo), "light": f32(wi), "rand": f32(r), "thin_film": f32(film), "lambda": lam,
                       "f_cos": f32(f), "pdf": float(pdf), "dir": f32(d), "weight": f32(w), "sample_pdf": float(spdf),
                       "lobe": lobe})
# Coated cases (their own stream, after the thin-film ones): coat weight 1 or uniform, every third with
# a thin film at three wavelengths (the others at the upstream RGB wavelengths), one in ten seen from
# behind (where only the base counts).
rng = np.random.default_rng(20261205)
coat_cases = []
for i in range(300):
    base = rng.random(3)
    metal = [0.0, 1.0, float(rng.random())][i % 3]
    rough = float(rng.random())
    ior = float(1.3 + 0.5 * rng.random())
    coat = 1.0 if i % 2 == 0 else float(rng.random())
    film = (1.0, float(0.1 + 0.8 * rng.random()), float(1.2 + 1.2 * rng.random())) if i % 3 == 1 else None
    lam = [float(x) for x in np.asarray(380.0 + 400.0 * rng.random(3), np.float32)] if film else [620.0, 540.0, 450.0]
    n = unit(rng.normal(size=3))
    wo = unit(rng.normal(size=3))
    if (np.dot(wo, n) < 0) != (i % 10 == 9):
        wo = -wo
    wi = unit(rng.normal(size=3))
    if i % 4 != 3 and np.dot(wi, n) < 0:
        wi = -wi
    r = rng.random(3).astype(np.float32)
    f32 = lambda x: [float(v) for v in np.asarray(x, np.float32)]
    m = R.material(base, metal, rough, ior, thin_film=film, coat=coat)
    f, pdf = R.evaluate(m, f32(n), f32(wo), f32(wi), lam)
    d, w, spdf, lobe = R.sample(m, f32(n), f32(wo), f32(r), lam)
    coat_cases.append({"base": f32(base), "metalness": metal, "roughness": rough, "ior": ior, "normal": f32(n),
                       "view": f32(wo), "light": f32(wi), "rand": f32(r), "thin_film": f32(film) if film else [0.0, 0.0, 1.4],
                       "lambda": lam, "coat": float(np.float32(coat)), "f_cos": f32(f), "pdf": float(pdf), "dir": f32(d),
                       "weight": f32(w), "sample_pdf": float(spdf), "lobe": lobe})
# Fuzzed cases (their own stream): fuzz weight 1 or uniform, every other one also coated.
rng = np.random.default_rng(20261206)
fuzz_cases = []
for i in range(300):
    base = rng.random(3)
    metal = [0.0, 1.0, float(rng.random())][i % 3]
    rough = float(rng.random())
    ior = float(1.3 + 0.5 * rng.random())
    fuzz = 1.0 if i % 4 < 2 else float(rng.random())
    coat = 0.0 if i % 2 == 0 else float(rng.random())
    n = unit(rng.normal(size=3))
    wo = unit(rng.normal(size=3))
    if (np.dot(wo, n) < 0) != (i % 10 == 9):
        wo = -wo
    wi = unit(rng.normal(size=3))
    if i % 4 != 3 and np.dot(wi, n) < 0:
        wi = -wi
    r = rng.random(3).astype(np.float32)
    f32 = lambda x: [float(v) for v in np.asarray(x, np.float32)]
    m = R.material(base, metal, rough, ior, coat=coat, fuzz=fuzz)
    f, pdf = R.evaluate(m, f32(n), f32(wo), f32(wi))
    d, w, spdf, lobe = R.sample(m, f32(n), f32(wo), f32(r))
    fuzz_cases.append({"base": f32(base), "metalness": metal, "roughness": rough, "ior": ior, "normal": f32(n),
                       "view": f32(wo), "light": f32(wi), "rand": f32(r), "coat": float(np.float32(coat)),
                       "fuzz": float(np.float32(fuzz)), "f_cos": f32(f), "pdf": float(pdf), "dir": f32(d), "weight": f32(w),
                       "sample_pdf": float(spdf), "lobe": lobe})
# Anisotropic cases (their own stream): anisotropy 1 or uniform, a tangent perpendicular to the normal.
rng = np.random.default_rng(20261207)
aniso_cases = []
for i in range(300):
    base = rng.random(3)
    metal = [0.0, 1.0, float(rng.random())][i % 3]
    rough = float(rng.random())
    ior = float(1.3 + 0.5 * rng.random())
    aniso = 1.0 if i % 5 == 0 else float(rng.random())
    coat = float(rng.random()) if i % 3 == 1 else 0.0
    fuzz = float(rng.random()) if i % 6 == 2 else 0.0
    n = unit(rng.normal(size=3))
    t = rng.normal(size=3)
    t = unit(t - n * np.dot(t, n))
    wo = unit(rng.normal(size=3))
    if (np.dot(wo, n) < 0) != (i % 10 == 9):
        wo = -wo
    wi = unit(rng.normal(size=3))
    if i % 4 != 3 and np.dot(wi, n) < 0:
        wi = -wi
    r = rng.random(3).astype(np.float32)
    f32 = lambda x: [float(v) for v in np.asarray(x, np.float32)]
    m = R.material(base, metal, rough, ior, coat=coat, fuzz=fuzz, anisotropy=aniso, tangent=f32(t))
    f, pdf = R.evaluate(m, f32(n), f32(wo), f32(wi))
    d, w, spdf, lobe = R.sample(m, f32(n), f32(wo), f32(r))
    aniso_cases.append({"base": f32(base), "metalness": metal, "roughness": rough, "ior": ior, "normal": f32(n),
                        "view": f32(wo), "light": f32(wi), "rand": f32(r), "coat": float(np.float32(coat)),
                        "fuzz": float(np.float32(fuzz)), "anisotropy": float(np.float32(aniso)), "tangent": f32(t),
                        "f_cos": f32(f), "pdf": float(pdf), "dir": f32(d), "weight": f32(w), "sample_pdf": float(spdf),
                        "lobe": lobe})
here = Path(__file__).resolve().parent
(here / "openpbr_aniso_cases.json").write_text(json.dumps({"source": "oracle/_ref/libopenpbr_ref.so (reference OpenPBR BSDF, "
                                                           "specular anisotropy about a tangent)", "cases": aniso_cases}) + "\n")
(here / "openpbr_fuzz_cases.json").write_text(json.dumps({"source": "oracle/_ref/libopenpbr_ref.so (reference OpenPBR BSDF, "
                                                          "the default fuzz)", "cases": fuzz_cases}) + "\n")
(here / "openpbr_coat_cases.json").write_text(json.dumps({"source": "oracle/_ref/libopenpbr_ref.so (reference OpenPBR BSDF, "
                                                          "the adapter's coat)", "cases": coat_cases}) + "\n")
(here / "openpbr_cases.json").write_text(json.dumps({"source": "oracle/_ref/libopenpbr_ref.so (reference OpenPBR BSDF)",
                                                     "cases": cases}) + "\n")
(here / "openpbr_thin_film_cases.json").write_text(json.dumps({"source": "oracle/_ref/libopenpbr_ref.so (reference OpenPBR BSDF, "
                                                               "thin-film iridescence at given wavelengths)",
                                                               "cases": film_cases}) + "\n")
t, a = R.metal_energy_table()
(here / "metal_energy.json").write_text(json.dumps({"source": "Shaders/MetalEnergy.metal via oracle/_ref",
                                                    "step": 8, "table": t[::8, ::8].astype(float).tolist(),
                                                    "average": a.astype(float).tolist()}) + "\n")
print("wrote", len(cases), "cases,", len(film_cases), "thin-film,", len(coat_cases), "coated,", len(fuzz_cases), "fuzzed and",
      len(aniso_cases), "anisotropic cases")
