"""ctypes binding of libvt_b200.so (the C ABI declared in include/vt.h).

The library is loaded from the package's ``lib/`` folder. There is no fallback: if the library is
missing or fails to load, every entry point raises, so no result can silently come from anything
but the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libvt_b200.so"

# ---- record layouts (numpy dtypes mirror the C structs byte for byte) -------------------------
FACE_DTYPE = np.dtype([("a", "<u4"), ("b", "<u4"), ("c", "<u4"), ("tag", "<u4")])
VERTEX_DTYPE = np.dtype([("p", "<f4", 3), ("n", "<f4", 3), ("uv", "<f4", 2)])
WIDE_NODE_DTYPE = np.dtype([
    ("lox", "<f4", 4), ("loy", "<f4", 4), ("loz", "<f4", 4),
    ("hix", "<f4", 4), ("hiy", "<f4", 4), ("hiz", "<f4", 4),
    ("child", "<i4", 4), ("count", "<i4", 4),
])
RAY_DTYPE = np.dtype([("o", "<f4", 3), ("tmin", "<f4"), ("d", "<f4", 3), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("b1", "<f4"), ("b2", "<f4"), ("prim", "<i4")])
EMITTER_DTYPE = np.dtype([("a", "<f4", 3), ("b", "<f4", 3), ("c", "<f4", 3), ("pad", "<f4"),
                          ("power", "<f8"), ("cos_emission", "<f8")])
assert EMITTER_DTYPE.itemsize == 56
assert FACE_DTYPE.itemsize == 16 and VERTEX_DTYPE.itemsize == 32
assert WIDE_NODE_DTYPE.itemsize == 128 and RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 16
INSTANCE_DTYPE = np.dtype([("world", "<f4", 12), ("mesh", "<u4"), ("slot_base", "<u4"), ("reserved", "<u4", 2)])
INSTANCE_RECORD_DTYPE = np.dtype([("world", "<f4", 12), ("local", "<f4", 12), ("mesh", "<u4"), ("slot_base", "<u4"),
                                  ("rendered_base", "<u4"), ("mirrored", "<u4"), ("bound", "<f4", 4)])
assert INSTANCE_DTYPE.itemsize == 64 and INSTANCE_RECORD_DTYPE.itemsize == 128


class BuildOptions(C.Structure):
    _fields_ = [("leaf_size", C.c_int32), ("treelet_size", C.c_int32),
                ("refine_rounds", C.c_int32), ("max_depth", C.c_int32)]


class MeshInfo(C.Structure):
    _fields_ = [("faces", C.c_uint32), ("wide_nodes", C.c_uint32), ("binary_nodes", C.c_uint32),
                ("depth", C.c_uint32), ("sah_cost", C.c_float), ("build_ms", C.c_float),
                ("lo", C.c_float * 3), ("hi", C.c_float * 3)]


class TlasInfo(C.Structure):
    _fields_ = [("instances", C.c_uint32), ("meshes", C.c_uint32), ("nodes", C.c_uint32), ("depth", C.c_uint32),
                ("rendered_triangles", C.c_uint64), ("lo", C.c_float * 3), ("hi", C.c_float * 3),
                ("grow", C.c_float), ("reach", C.c_float), ("build_ms", C.c_float), ("pad", C.c_float)]


class LightTreeInfo(C.Structure):
    _fields_ = [("node_count", C.c_uint32), ("depth", C.c_uint32), ("count", C.c_uint32), ("pad", C.c_uint32),
                ("grid_lo", C.c_float * 3), ("grid_hi", C.c_float * 3)]


class SpectralGridInfo(C.Structure):
    _fields_ = [("built", C.c_uint32), ("refined_cells", C.c_uint32), ("flagged_cells", C.c_uint32),
                ("pad", C.c_uint32), ("max_residual", C.c_double)]


class OpenPBRTables(C.Structure):
    _fields_ = [("opaque_energy", C.c_void_p), ("opaque_average", C.c_void_p), ("ltc", C.c_void_p)]


class OpenPBRCase(C.Structure):
    _fields_ = [("base_color", C.c_float * 3), ("metalness", C.c_float), ("roughness", C.c_float), ("ior", C.c_float),
                ("specular_weight", C.c_float), ("diffuse_roughness", C.c_float), ("normal", C.c_float * 3),
                ("view", C.c_float * 3), ("light", C.c_float * 3), ("rand", C.c_float * 3),
                ("thin_film_weight", C.c_float), ("thin_film_thickness", C.c_float), ("thin_film_ior", C.c_float),
                ("lambda_nm", C.c_float * 3), ("coat", C.c_float), ("fuzz", C.c_float),
                ("anisotropy", C.c_float), ("tangent", C.c_float * 3)]


class OpenPBRResult(C.Structure):
    _fields_ = [("f_cos", C.c_float * 3), ("pdf", C.c_float), ("dir", C.c_float * 3), ("weight", C.c_float * 3),
                ("sample_pdf", C.c_float), ("ok", C.c_float)]


class OpenPBRParams(C.Structure):
    _fields_ = [("roughness", C.c_float), ("metalness", C.c_float), ("ior", C.c_float), ("diffuse_roughness", C.c_float),
                ("thin_film_weight", C.c_float), ("thin_film_thickness", C.c_float), ("thin_film_ior", C.c_float),
                ("coat", C.c_float), ("fuzz", C.c_float), ("anisotropy", C.c_float), ("pad", C.c_float * 2)]


assert C.sizeof(OpenPBRCase) == 128 and C.sizeof(OpenPBRResult) == 48 and C.sizeof(OpenPBRParams) == 48


class BatchStats(C.Structure):
    _fields_ = [("scenes", C.c_uint32), ("passes", C.c_uint32), ("items", C.c_ulonglong), ("last_ms", C.c_float),
                ("tuned", C.c_uint32), ("block", C.c_uint32), ("chunk", C.c_uint32), ("wavefront", C.c_uint32),
                ("queue_paths", C.c_uint32), ("compact_every", C.c_uint32), ("streams", C.c_uint32)]


class Environment(C.Structure):
    _fields_ = [("intensity", C.c_float), ("sun_dir", C.c_float * 3), ("sun_intensity", C.c_float),
                ("sky_mode", C.c_uint32), ("pad", C.c_uint32 * 2)]


class NRCConfig(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("log2_table", C.c_uint32), ("base_resolution", C.c_uint32),
                ("max_resolution", C.c_uint32), ("train_records", C.c_uint32), ("train_paths", C.c_uint32),
                ("query_vertex", C.c_uint32), ("seed", C.c_uint32), ("learning_rate", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("epsilon", C.c_float), ("spread", C.c_float),
                ("spectral", C.c_uint32)]


class NRCInput(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("roughness", C.c_float), ("direction", C.c_float * 2),
                ("normal", C.c_float * 2), ("diffuse", C.c_float * 3), ("specular", C.c_float),
                ("wavelength", C.c_float), ("pad", C.c_float * 3)]


class NRCInfo(C.Structure):
    _fields_ = [("mlp_params", C.c_ulonglong), ("grid_params", C.c_ulonglong), ("steps", C.c_uint32),
                ("last_records", C.c_uint32), ("last_loss", C.c_float), ("pad", C.c_uint32)]


VT_OK = 0
STATUS_NAMES = {0: "VT_OK", 1: "VT_ERR_INVALID", 2: "VT_ERR_CUDA", 3: "VT_ERR_MEMORY",
                4: "VT_ERR_LIMIT", 5: "VT_ERR_DEVICE"}

# Every symbol include/vt.h declares, with (restype, argtypes).
_P = C.c_void_p
_U32 = C.c_uint32
_I32 = C.c_int32
SIGNATURES = {
    "vt_abi_version": (_U32, []),
    "vt_ctx_create": (_I32, [_I32, C.POINTER(_P)]),
    "vt_ctx_destroy": (_I32, [_P]),
    "vt_last_error": (C.c_char_p, [_P]),
    "vt_sync": (_I32, [_P]),
    "vt_mesh_build": (_I32, [_P, _P, _U32, _P, _U32, C.POINTER(BuildOptions), C.POINTER(_P)]),
    "vt_mesh_build_device": (_I32, [_P, _P, _U32, _P, _U32, C.POINTER(BuildOptions), C.POINTER(_P)]),
    "vt_mesh_destroy": (_I32, [_P, _P]),
    "vt_mesh_get_info": (_I32, [_P, _P, C.POINTER(MeshInfo)]),
    "vt_mesh_get_order": (_I32, [_P, _P, _P, _U32]),
    "vt_mesh_get_nodes": (_I32, [_P, _P, _P, _U32]),
    "vt_mesh_get_morton": (_I32, [_P, _P, _P, _P, _U32]),
    "vt_mesh_get_binary": (_I32, [_P, _P, _P, _P, _U32]),
    "vt_trace_closest": (_I32, [_P, _P, _P, _U32, _P, _P]),
    "vt_trace_any": (_I32, [_P, _P, _P, _U32, _P, _P]),
    "vt_trace_closest_host": (_I32, [_P, _P, _P, _U32, _P]),
    "vt_trace_any_host": (_I32, [_P, _P, _P, _U32, _P]),
    "vt_trace_count": (_I32, [_P, _P, _P, _U32, _I32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "vt_tlas_build": (_I32, [_P, _P, _U32, _P, _U32, C.POINTER(_P)]),
    "vt_tlas_destroy": (_I32, [_P, _P]),
    "vt_tlas_get_info": (_I32, [_P, _P, C.POINTER(TlasInfo)]),
    "vt_tlas_get_nodes": (_I32, [_P, _P, _P, _U32]),
    "vt_tlas_get_instances": (_I32, [_P, _P, _P, _U32]),
    "vt_tlas_trace_closest": (_I32, [_P, _P, _P, _U32, _P, _P, _P]),
    "vt_tlas_trace_any": (_I32, [_P, _P, _P, _U32, _P, _P]),
    "vt_tlas_flatten": (_I32, [_P, _P, C.POINTER(BuildOptions), C.POINTER(_P)]),
    "vt_mesh_build_noalloc": (_I32, [_P, _U32, _P, _U32, C.POINTER(BuildOptions), _P, _U32, _P, _P,
                                     C.POINTER(MeshInfo), _P, C.c_char_p, _U32]),
    "vt_scene_create": (_I32, [_P, _P, _P, _U32, _P, _P, C.POINTER(_P)]),
    "vt_scene_destroy": (_I32, [_P, _P]),
    "vt_render": (_I32, [_P, _P, _P, _U32, _P]),
    "vt_render_wavefront": (_I32, [_P, _P, _P, _U32, _P]),
    "vt_accum_reset": (_I32, [_P, _P]),
    "vt_accum_readback": (_I32, [_P, _P, _P, _U32, C.POINTER(_U32)]),
    "vt_accum_restore": (_I32, [_P, _P, _U32, _U32, _U32, _P, _U32, _U32]),
    "vt_sampler_frame": (_I32, [_P, _U32, _U32, _U32, _U32, _U32, _U32, _U32, _U32, _P]),
    "vt_known_answers": (_I32, [_P, _P, _U32]),
    "vt_light_tree_build": (_I32, [_P, _P, _U32, _U32, C.c_double, C.POINTER(_P)]),
    "vt_light_tree_destroy": (_I32, [_P, _P]),
    "vt_light_tree_get_info": (_I32, [_P, _P, C.POINTER(LightTreeInfo)]),
    "vt_light_tree_get_words": (_I32, [_P, _P, _P, _U32]),
    "vt_light_tree_get_order": (_I32, [_P, _P, _P, _P, _U32]),
    "vt_emitter_list_pack": (_I32, [_P, _P, _P, _U32, _U32, _P, _U32, C.POINTER(_U32)]),
    "vt_scene_create_imported": (_I32, [_P, _P, _P, _U32, _P, _U32, C.POINTER(_P)]),
    "vt_scene_emitter_words": (_I32, [_P, _P, _P, _U32, C.POINTER(_U32)]),
    "vt_light_estimate": (_I32, [_P, _P, _P, _U32, _U32, _U32, _P]),
    "vt_scene_di_weights": (_I32, [_P, _P, _P, _U32]),
    "vt_scene_gi_weights": (_I32, [_P, _P, _P, _U32]),
    "vt_batch_create": (_I32, [_P, _P, _P, _P, _U32, C.POINTER(_P)]),
    "vt_batch_render": (_I32, [_P, _P, _P]),
    "vt_batch_render_wavefront": (_I32, [_P, _P, _P]),
    "vt_batch_stats": (_I32, [_P, _P, C.POINTER(BatchStats), _P, _U32]),
    "vt_batch_destroy": (_I32, [_P, _P]),
    "vt_spectral_grid_build": (_I32, [_P, _P]),
    "vt_spectral_grid_get_info": (_I32, [_P, C.POINTER(SpectralGridInfo)]),
    "vt_spectral_grid_read": (_I32, [_P, _P, _U32]),
    "vt_spectral_lagrange": (_I32, [_P, _P, _U32, _P]),
    "vt_spectral_round_trip": (_I32, [_P, C.POINTER(C.c_float), C.POINTER(_U32)]),
    "vt_openpbr_tables_set": (_I32, [_P, C.POINTER(OpenPBRTables)]),
    "vt_openpbr_energy_table": (_I32, [_P, _P, _P]),
    "vt_openpbr_evaluate": (_I32, [_P, _P, _U32, _P]),
    "vt_scene_set_openpbr": (_I32, [_P, _P, _P, _U32]),
    "vt_scene_set_environment": (_I32, [_P, _P, C.POINTER(Environment)]),
    "vt_scene_set_environment_map": (_I32, [_P, _P, _P, _U32, _U32, C.c_float, C.c_float]),
    "vt_environment_tables": (_I32, [_P, _U32, _U32, _P, _P]),
    "vt_nrc_config_default": (_I32, [C.POINTER(NRCConfig)]),
    "vt_nrc_create": (_I32, [_P, C.POINTER(NRCConfig), _P, _P, C.POINTER(_P)]),
    "vt_nrc_destroy": (_I32, [_P, _P]),
    "vt_nrc_get_info": (_I32, [_P, _P, C.POINTER(NRCInfo)]),
    "vt_nrc_get_params": (_I32, [_P, _P, _P, _P]),
    "vt_nrc_set_params": (_I32, [_P, _P, _P, _P]),
    "vt_nrc_infer": (_I32, [_P, _P, _P, _U32, _P]),
    "vt_nrc_gradients": (_I32, [_P, _P, _P, _P, _U32, _P, _P, C.POINTER(C.c_double)]),
    "vt_nrc_train": (_I32, [_P, _P, _P, _P, _U32, C.POINTER(C.c_float)]),
    "vt_render_nrc": (_I32, [_P, _P, _P, _P, _U32, _U32, _P]),
}
NOALLOC_MAX_FACES = 32768
KNOWN_ANSWERS = 16

_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Load libvt_b200.so (once) and declare every C-ABI signature. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m metal_vibe_tracer_b200.build` "
            "(or __graft_entry__.build()). There is no CPU fallback.")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(SIGNATURES)
