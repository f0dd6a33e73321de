"""OpenPBR data: the opaque-dielectric energy complement tables of the Adobe openpbr-bsdf library
the reference vendors (Vendor/OpenPBR/impl/data, Apache-2.0), which the diffuse base lobe and the
coat use (impl/openpbr_diffuse_lobe.h, impl/openpbr_coating_lobe.h), and the fuzz lobe's LTC table
(openpbr_ltc_data.h: Zeltner, Burley and Chiang's sheen fit, Apache-2.0).

They are library data, not part of this repository: `generate()` reads them at build time from the
reference's vendored headers (32^3 and 32^2 unorm16 values) and writes
`data/openpbr_energy.bin` (git-ignored, shipped with the built library); `load()` reads that file
at run time and `set_tables(ctx)` hands them to the device. The dense metal table the reference
substitutes for the library's (Shaders/MetalEnergy.metal) is solved on the device instead
(vt_openpbr_energy_table).
"""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
DATA = PKG / "data" / "openpbr_energy.bin"


def reference_data() -> Path | None:
    """The vendored OpenPBR data directory of the reference checkout named by VT_REFERENCE_ROOT (see
    spectral_tables.reference_root); None when unset."""
    from .spectral_tables import reference_root
    r = reference_root()
    return r / "Vendor" / "OpenPBR" / "impl" / "data" if r else None
MAGIC = b"VTPBR002"
N = 32


def _read_values(path: Path) -> np.ndarray:
    text = "\n".join(line for line in path.read_text().splitlines() if not line.lstrip().startswith("//"))
    return np.array([int(v) for v in re.findall(r"\d+", text)], np.uint16)


def _read_ltc(path: Path) -> np.ndarray:
    """The fuzz lobe's LTC table (openpbr_ltc_data.h: 32 x 32 entries of (a_inv, b_inv, R), rows by
    roughness, columns by cos theta) as float32, each decimal literal rounded as a C++ compiler does
    (to double, then to float)."""
    text = "\n".join(line for line in path.read_text().splitlines() if not line.lstrip().startswith("//"))
    num = r"\s*([-\d.eE+]+)\s*"
    vals = re.findall(r"vec3\(" + num + "," + num + "," + num + r"\)", text)
    return np.array([[float(x) for x in v] for v in vals], np.float64).astype(np.float32).reshape(-1)


def generate(data_dir: Path | None = None) -> Path:
    data_dir = data_dir or reference_data()
    if data_dir is None:
        raise RuntimeError("OpenPBR data: set VT_REFERENCE_ROOT to the reference checkout")
    energy = _read_values(data_dir / "openpbr_opaque_dielectric_energy_complement_data.h")
    average = _read_values(data_dir / "openpbr_opaque_dielectric_avg_energy_complement_data.h")
    ltc = _read_ltc(data_dir / "openpbr_ltc_data.h")
    if energy.size != N ** 3 or average.size != N ** 2 or ltc.size != 3 * N * N:
        raise RuntimeError(f"unexpected OpenPBR table sizes {energy.size}, {average.size}, {ltc.size}")
    DATA.parent.mkdir(parents=True, exist_ok=True)
    tmp = DATA.with_suffix(".tmp")
    tmp.write_bytes(MAGIC + energy.tobytes() + average.tobytes() + ltc.tobytes())
    tmp.replace(DATA)
    return DATA


def load() -> dict:
    if not DATA.exists():
        raise RuntimeError(f"{DATA} is missing: it is generated at build time from the reference's vendored "
                           "OpenPBR data (metal_vibe_tracer_b200.openpbr_tables.generate)")
    b = DATA.read_bytes()
    if b[:8] != MAGIC:
        raise RuntimeError(f"{DATA}: bad header")
    energy = np.frombuffer(b, np.uint16, N ** 3, 8).copy()
    average = np.frombuffer(b, np.uint16, N ** 2, 8 + 2 * N ** 3).copy()
    ltc = np.frombuffer(b, np.float32, 3 * N * N, 8 + 2 * N ** 3 + 2 * N ** 2).copy()
    return {"opaque_energy": energy, "opaque_average": average, "ltc": ltc}
