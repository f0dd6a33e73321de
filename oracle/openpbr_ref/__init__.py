"""ctypes binding of oracle/_ref/libopenpbr_ref.so: the reference's own OpenPBR BSDF compiled for the
CPU from its vendored headers (test infrastructure only; see openpbr_ref.cpp)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent.parent / "_ref" / "libopenpbr_ref.so"
F3 = C.c_float * 3


class Material(C.Structure):
    _fields_ = [("type", C.c_int32), ("albedo", C.c_float * 3), ("roughness", C.c_float), ("metalness", C.c_float),
                ("ior", C.c_float), ("coat", C.c_float), ("anisotropy", C.c_float), ("fuzz", C.c_float),
                ("transmission", C.c_float), ("thin_film_weight", C.c_float), ("thin_film_thickness", C.c_float),
                ("thin_film_ior", C.c_float), ("inside", C.c_int32), ("tangent", C.c_float * 3), ("pad", C.c_float)]


_lib = None


def available() -> bool:
    return LIB.exists()


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(f"{LIB} is missing: build it with `make -C oracle/openpbr_ref` where the reference is checked out")
        _lib = C.CDLL(str(LIB))
        _lib.ref_metal_energy.restype = C.c_float
        _lib.ref_metal_energy.argtypes = [C.c_float, C.c_float]
        _lib.ref_metal_average_energy.restype = C.c_float
        _lib.ref_metal_average_energy.argtypes = [C.c_float]
    return _lib


def material(base, metalness, roughness, ior, type_=4, thin_film=None, coat=0.0, fuzz=0.0, anisotropy=0.0, tangent=None):
    """A reference material; `thin_film` = (weight, thickness in micrometres, IOR) or None; `coat`:
    the coat weight (the adapter's coat: roughness 0.12, default IOR and colour); `fuzz`: the fuzz
    weight (default roughness and colour); `anisotropy`: specular_roughness_anisotropy, oriented by the
    unit `tangent` (the adapter's mat.tangent; None: the basis from the normal alone)."""
    m = Material()
    m.type = type_
    m.albedo[:] = [float(x) for x in base]
    m.roughness, m.metalness, m.ior = float(roughness), float(metalness), float(ior)
    m.coat = float(coat)
    m.fuzz = float(fuzz)
    m.anisotropy = float(anisotropy)
    if tangent is not None:
        m.tangent[:] = [float(x) for x in tangent]
    if thin_film is not None:
        m.thin_film_weight, m.thin_film_thickness, m.thin_film_ior = (float(x) for x in thin_film)
    return m


def evaluate(m, n, wo, wi, lambda_nm=None):
    """(f |cos| (3), pdf) of the reference BSDF (at three wavelengths in nm; None: its RGB ones)."""
    f, pdf = F3(), C.c_float()
    lam = F3(*lambda_nm) if lambda_nm is not None else None
    load().ref_openpbr_eval(C.byref(m), F3(*n), F3(*wo), F3(*wi), lam, f, C.byref(pdf))
    return np.array(f, np.float32), np.float32(pdf.value)


def sample(m, n, wo, rand, lambda_nm=None):
    """(direction, weight f |cos| / pdf, pdf, lobe type bits) of one reference sample."""
    d, w, pdf, lobe = F3(), F3(), C.c_float(), C.c_int32()
    lam = F3(*lambda_nm) if lambda_nm is not None else None
    load().ref_openpbr_sample(C.byref(m), F3(*n), F3(*wo), F3(*rand), lam, d, w, C.byref(pdf), C.byref(lobe))
    return np.array(d, np.float32), np.array(w, np.float32), np.float32(pdf.value), int(lobe.value)


def metal_energy_table():
    """The reference's dense metal table (Shaders/MetalEnergy.metal): (129, 129) and (129,)."""
    t = np.empty(129 * 129, np.float32)
    a = np.empty(129, np.float32)
    load().ref_metal_energy_table(t.ctypes.data_as(C.c_void_p), a.ctypes.data_as(C.c_void_p))
    return t.reshape(129, 129), a
