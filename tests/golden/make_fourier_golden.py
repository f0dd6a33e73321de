"""Writes tests/golden/fourier_srgb_lines.json from the reference's own table generator.

Run in a container that has the reference checked out: it imports scripts/generate_spectral_tables.py
and solves whole (r, g) lines of the 86^3 moment grid exactly as that script builds
FourierSRGB86.bin (`_coarse_line`: Levenberg-Marquardt warm-started along b, moments by the 1024-node
midpoint rule), stored as the float32 values the file holds. Nothing is written into the reference
tree. Lines: the four that hold the six saturated corners, plus twelve seeded ones. Also the
generator's Lagrange multipliers (`lagrange3`) of a few lines' nodes. Values derive from the CIE 1931
2-degree CMFs and D65 (CIE 2019, CC BY-SA 4.0) and Peters' warp (BSD); only a small sample is stored.
"""
import json
import random
import struct
import sys
from pathlib import Path

REF = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
sys.path.insert(0, str(REF / "scripts"))
import generate_spectral_tables as G  # noqa: E402

G._init_worker()
rng = random.Random(20261203)
lines = [(0, 0), (255, 0), (0, 255), (255, 255)]
while len(lines) < 16:
    r, g = 3 * rng.randrange(86), 3 * rng.randrange(86)
    if (r, g) not in lines:
        lines.append((r, g))
out = {"source": "scripts/generate_spectral_tables.py _coarse_line (FourierSRGB86.bin entries as float32)",
       "codes_b": G.COARSE_CODES, "lines": []}
for r, g in lines:
    blob, worst = G._coarse_line((r, g))
    vals = struct.unpack("<%dd" % (len(blob) // 8), blob)
    f32 = [struct.unpack("<f", struct.pack("<f", v))[0] for v in vals]
    out["lines"].append({"r": r, "g": g, "moments": f32, "worst_residual": worst})
    print("line", r, g, "worst", worst, flush=True)
checks = []
for line in out["lines"][:4]:
    for b in (0, 12, 43, 85):
        c = line["moments"][3 * b:3 * b + 3]
        checks.append({"moments": c, "lagrange": G.lagrange3(*G.clamp_moments(c))})
out["lagrange3"] = checks
dest = Path(__file__).resolve().parent / "fourier_srgb_lines.json"
dest.write_text(json.dumps(out) + "\n")
print("wrote", dest)
