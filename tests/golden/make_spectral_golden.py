"""Writes tests/golden/spectral_360_830.json from the reference's own table generator.

Run in a container that has the reference checked out (it imports
scripts/generate_spectral_tables.py from it); the fixture it writes is committed so the check
runs without the reference. Values are derived from the CIE 1931 2-degree colour-matching
functions and CIE standard illuminant D65 (CIE 2019, DOIs 10.25039/CIE.DS.xvudnb9b and
10.25039/CIE.DS.hjfjmt59, CC BY-SA 4.0); only a handful of derived numbers are stored.
"""
import json
import sys
from pathlib import Path

REF = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
sys.path.insert(0, str(REF / "scripts"))
import generate_spectral_tables as G  # noqa: E402

data = G.Data(REF / "Vendor" / "Spectral")
d65 = 1  # index of D65 in G.ILLUMINANTS
icdf = G.inverse_cdf(G.sampling_density(data, d65))
density = G.sampling_density(data, d65)
picks = [400, 450, 500, 555, 560, 600, 650, 700]
golden = {
    "source": "scripts/generate_spectral_tables.py (Data, sampling_density, inverse_cdf), 360-830 nm",
    "lambda_min": G.LAMBDA_MIN, "lambda_max": G.LAMBDA_MAX, "segments": G.ICDF_SEGMENTS,
    "xyz_to_rgb": data.xyz_to_rgb,
    "d65_white_xyz": data.white,
    "d65_normalized": {str(l): data.illuminants[d65][l - G.LAMBDA_MIN] for l in picks},
    "density": {str(l): density[l - G.LAMBDA_MIN] for l in picks},
    "icdf_nodes": {str(i): icdf[i] for i in range(0, G.ICDF_SEGMENTS + 1, 64)},
}
out = Path(__file__).resolve().parent / "spectral_360_830.json"
out.write_text(json.dumps(golden, indent=1) + "\n")
print("wrote", out)
