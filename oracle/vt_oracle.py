"""ctypes binding of the oracle library (oracle/lib/libvt_oracle.so).

Test infrastructure only: the checker for the CUDA path (see vt_oracle.h for the reference
functions each routine restates, with file:line).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "libvt_oracle.so"

FACE_DTYPE = np.dtype([("a", "<u4"), ("b", "<u4"), ("c", "<u4"), ("tag", "<u4")])
VERTEX_DTYPE = np.dtype([("p", "<f4", 3), ("n", "<f4", 3), ("uv", "<f4", 2)])
WIDE_NODE_DTYPE = np.dtype([
    ("lox", "<f4", 4), ("loy", "<f4", 4), ("loz", "<f4", 4),
    ("hix", "<f4", 4), ("hiy", "<f4", 4), ("hiz", "<f4", 4),
    ("child", "<i4", 4), ("count", "<i4", 4),
])
RAY_DTYPE = np.dtype([("o", "<f4", 3), ("tmin", "<f4"), ("d", "<f4", 3), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("b1", "<f4"), ("b2", "<f4"), ("prim", "<i4")])


class BvhInfo(C.Structure):
    _fields_ = [("faces", C.c_uint32), ("wide_nodes", C.c_uint32), ("binary_nodes", C.c_uint32),
                ("depth", C.c_uint32), ("sah_cost", C.c_float), ("lo", C.c_float * 3), ("hi", C.c_float * 3)]


_P, _U32, _I32 = C.c_void_p, C.c_uint32, C.c_int32
_SIGS = {
    "vto_pcg_hash": (_U32, [_U32]),
    "vto_rand_f": (C.c_float, [C.POINTER(_U32)]),
    "vto_intersect_f32": (_I32, [_P, _P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "vto_intersect_f64": (_I32, [_P, _P, C.c_double, C.c_double, C.POINTER(C.c_double),
                                 C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "vto_lbvh_build": (_P, [_P, _U32, _P, _U32, _I32, _I32, _I32]),
    "vto_widebvh_build": (_P, [_P, _U32, _P, _U32, _I32, _I32, _I32]),
    "vto_bvh_free": (None, [_P]),
    "vto_bvh_import": (_P, [_P, _U32, _P, _U32, _P, _P, _U32]),
    "vto_bvh_get_info": (None, [_P, C.POINTER(BvhInfo)]),
    "vto_bvh_get_nodes": (None, [_P, _P]),
    "vto_bvh_get_order": (None, [_P, _P]),
    "vto_bvh_get_morton": (None, [_P, _P, _P]),
    "vto_bvh_get_binary": (None, [_P, _P, _P]),
    "vto_trace_closest": (None, [_P, _P, _U32, _P, _I32, _I32]),
    "vto_trace_any": (None, [_P, _P, _U32, _P, _I32, _I32]),
    "vto_brute_closest": (None, [_P, _U32, _P, _P, _U32, _P, _I32, _I32]),
    "vto_trace_count": (None, [_P, _P, _U32, _I32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), _I32]),
    "vto_tlas_trace": (None, [_P, _P, _P, C.c_float, C.c_float, _P, _U32, _P, _P, _P, _I32, _I32, _I32]),
}

_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off)."""
    res = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def threads() -> int:
    return max(1, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count() or 1)


def _faces(f):
    f = np.ascontiguousarray(f)
    assert f.dtype == FACE_DTYPE
    return f


def _verts(v):
    v = np.ascontiguousarray(v)
    assert v.dtype == VERTEX_DTYPE
    return v


def _rays(r):
    r = np.ascontiguousarray(r)
    if r.dtype != RAY_DTYPE:
        r = np.ascontiguousarray(r, dtype=np.float32).view(RAY_DTYPE).reshape(-1)
    return r


def pcg_hash(v: int) -> int:
    return int(load().vto_pcg_hash(v & 0xFFFFFFFF))


def rand_f(seed: int) -> tuple[float, int]:
    s = C.c_uint32(seed & 0xFFFFFFFF)
    x = load().vto_rand_f(C.byref(s))
    return float(x), int(s.value)


def intersect_f32(ray, tri) -> tuple[bool, float, float, float]:
    r = _rays(np.asarray(ray, np.float32).reshape(1, 8))
    t9 = np.ascontiguousarray(tri, np.float32).reshape(9)
    t, b1, b2 = C.c_float(), C.c_float(), C.c_float()
    hit = load().vto_intersect_f32(r.ctypes.data, t9.ctypes.data, C.byref(t), C.byref(b1), C.byref(b2))
    return bool(hit), t.value, b1.value, b2.value


def intersect_f64(o, d, tri, tmin=0.0, tmax=np.inf) -> tuple[bool, float, float, float]:
    r = np.ascontiguousarray(np.concatenate([o, d]), np.float64)
    t9 = np.ascontiguousarray(tri, np.float64).reshape(9)
    t, b1, b2 = C.c_double(), C.c_double(), C.c_double()
    hit = load().vto_intersect_f64(r.ctypes.data, t9.ctypes.data, tmin, tmax, C.byref(t), C.byref(b1), C.byref(b2))
    return bool(hit), t.value, b1.value, b2.value


class Bvh:
    """An oracle BVH (LBVH restatement or the reference's binned-SAH WideBVH)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def lbvh(cls, faces, verts, leaf_size=2, treelet_size=7, rounds=2):
        f, v = _faces(faces), _verts(verts)
        return cls(load().vto_lbvh_build(f.ctypes.data, f.shape[0], v.ctypes.data, v.shape[0],
                                         leaf_size, treelet_size, rounds))

    @classmethod
    def from_arrays(cls, nodes, order, faces, verts, depth):
        """A hierarchy built elsewhere (the device's 4-wide nodes, leaf order and depth) over the same
        faces and vertices."""
        nd = np.ascontiguousarray(nodes, WIDE_NODE_DTYPE)
        od = np.ascontiguousarray(order, np.int32)
        f, v = _faces(faces), _verts(verts)
        return cls(load().vto_bvh_import(nd.ctypes.data, nd.shape[0], od.ctypes.data, od.shape[0], f.ctypes.data,
                                         v.ctypes.data, int(depth)))

    @classmethod
    def widebvh(cls, faces, verts, leaf_size=2, max_depth=20, nthreads=None):
        f, v = _faces(faces), _verts(verts)
        return cls(load().vto_widebvh_build(f.ctypes.data, f.shape[0], v.ctypes.data, v.shape[0],
                                            leaf_size, max_depth, nthreads or threads()))

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                load().vto_bvh_free(self._h)
                self._h = None
        except Exception:
            pass

    def info(self) -> BvhInfo:
        out = BvhInfo()
        load().vto_bvh_get_info(self._h, C.byref(out))
        return out

    def nodes(self) -> np.ndarray:
        out = np.empty(self.info().wide_nodes, WIDE_NODE_DTYPE)
        load().vto_bvh_get_nodes(self._h, out.ctypes.data)
        return out

    def order(self) -> np.ndarray:
        out = np.empty(self.info().faces, np.int32)
        load().vto_bvh_get_order(self._h, out.ctypes.data)
        return out

    def morton(self):
        n = self.info().faces
        codes, sorted_ = np.empty(n, np.uint32), np.empty(n, np.int32)
        load().vto_bvh_get_morton(self._h, codes.ctypes.data, sorted_.ctypes.data)
        return codes, sorted_

    def binary(self):
        n = self.info().binary_nodes
        ch, boxes = np.empty((n, 2), np.int32), np.empty((n, 6), np.float32)
        load().vto_bvh_get_binary(self._h, ch.ctypes.data, boxes.ctypes.data)
        return ch, boxes

    def closest(self, rays, precision=32, nthreads=None):
        r = _rays(rays)
        out = np.empty(r.shape[0], HIT_DTYPE)
        load().vto_trace_closest(self._h, r.ctypes.data, r.shape[0], out.ctypes.data, precision,
                                 nthreads or threads())
        return out

    def occluded(self, rays, precision=32, nthreads=None):
        r = _rays(rays)
        out = np.empty(r.shape[0], np.uint8)
        load().vto_trace_any(self._h, r.ctypes.data, r.shape[0], out.ctypes.data, precision,
                             nthreads or threads())
        return out

    def count(self, rays, closest=True, nthreads=None):
        r = _rays(rays)
        a, b = C.c_uint64(), C.c_uint64()
        load().vto_trace_count(self._h, r.ctypes.data, r.shape[0], 1 if closest else 0, C.byref(a), C.byref(b),
                               nthreads or threads())
        return int(a.value), int(b.value)


def tlas_trace(nodes, records, meshes, grow, reach, rays, closest=True, precision=32, nthreads=None):
    """Two-level traversal over oracle meshes (Bvh), the TLAS nodes and instance records of a vt_tlas:
    (hits, instances) for closest, else occluded flags."""
    r = _rays(rays)
    nodes = np.ascontiguousarray(nodes, WIDE_NODE_DTYPE)
    records = np.ascontiguousarray(records)
    handles = (C.c_void_p * len(meshes))(*[m._h for m in meshes])
    n = r.shape[0]
    hits = np.empty(n, HIT_DTYPE)
    inst = np.empty(n, np.uint32)
    occ = np.empty(n, np.uint8)
    load().vto_tlas_trace(nodes.ctypes.data, records.ctypes.data, handles, C.c_float(grow), C.c_float(reach),
                          r.ctypes.data, n, hits.ctypes.data, inst.ctypes.data, occ.ctypes.data, 1 if closest else 0,
                          precision, nthreads or threads())
    return (hits, inst) if closest else occ


def brute_closest(faces, verts, rays, precision=32, nthreads=None):
    f, v, r = _faces(faces), _verts(verts), _rays(rays)
    out = np.empty(r.shape[0], HIT_DTYPE)
    load().vto_brute_closest(f.ctypes.data, f.shape[0], v.ctypes.data, r.ctypes.data, r.shape[0],
                             out.ctypes.data, precision, nthreads or threads())
    return out


# ---- path tracer -------------------------------------------------------------------------------
class Material(C.Structure):
    _fields_ = [("type", C.c_int32), ("albedo", C.c_float * 3), ("emission", C.c_float * 3), ("pad", C.c_float)]


class QuadLight(C.Structure):
    _fields_ = [("corner", C.c_float * 3), ("su", C.c_float * 3), ("sv", C.c_float * 3), ("normal", C.c_float * 3),
                ("emission", C.c_float * 3), ("pad", C.c_float)]


class FrameParams(C.Structure):
    _fields_ = [("camera_pos", C.c_float * 3), ("fov_deg", C.c_float), ("camera_target", C.c_float * 3),
                ("max_depth", C.c_uint32), ("camera_up", C.c_float * 3), ("sampling_mode", C.c_uint32),
                ("width", C.c_uint32), ("height", C.c_uint32), ("first_sample", C.c_uint32),
                ("spectral", C.c_uint32), ("sampler", C.c_uint32), ("z_temporal", C.c_uint32),
                ("first_frame", C.c_uint32), ("di_candidates", C.c_uint32),
                ("aperture", C.c_float), ("focus_distance", C.c_float), ("pixel_stride", C.c_uint32)]


class Environment(C.Structure):
    _fields_ = [("intensity", C.c_float), ("sun_dir", C.c_float * 3), ("sun_intensity", C.c_float),
                ("sky_mode", C.c_uint32), ("pad", C.c_uint32 * 2)]


class PtInputs(C.Structure):
    _fields_ = [("faces", C.c_void_p), ("nfaces", C.c_uint32), ("verts", C.c_void_p), ("nverts", C.c_uint32),
                ("materials", C.c_void_p), ("nmat", C.c_uint32), ("light", QuadLight),
                ("cmf_rgb", C.c_void_p), ("illum", C.c_void_p), ("icdf", C.c_void_p),
                ("nbins", C.c_uint32), ("segments", C.c_uint32), ("lambda_min", C.c_float),
                ("emitters", C.c_void_p), ("nemitter_words", C.c_uint32), ("imported", C.c_uint32),
                ("uplift", C.c_void_p), ("cos_phase", C.c_void_p),
                ("pbr_params", C.c_void_p), ("pbr_eval", C.c_void_p), ("pbr_sample", C.c_void_p),
                ("environment", Environment), ("env_rgba", C.c_void_p), ("env_w", C.c_uint32), ("env_h", C.c_uint32),
                ("env_rot", C.c_float), ("bvh", C.c_void_p), ("pbr_film_mirror", C.c_void_p)]


_SIGS["vto_render"] = (None, [C.POINTER(PtInputs), C.POINTER(FrameParams), _U32, _P, _I32])


def render(faces, verts, materials, light, camera, width, height, spp, max_depth=8, first_sample=1,
           spectral=None, nthreads=None, mode=1, sampler=0, z_temporal=3, first_frame=1, light_tree=True,
           emitter_words=None, di_candidates=0, aperture=0.0, focus_distance=1.0, environment=None,
           pixel_stride=1, bvh=None):
    """FP64 oracle render: (height, width, 3) mean linear-sRGB radiance over `spp` frames (with a
    pixel stride s, modes 1-3: (ceil(height / s), ceil(width / s), 3) for every s-th pixel). `bvh`: a
    prebuilt hierarchy over the faces (Bvh.from_arrays), else the renderer builds its LBVH.

    light=None renders an imported scene lit by its emissive faces; its emitter list is the
    pure-Python restatement's (oracle/light_tree.py) unless `emitter_words` is given. An imported
    scene may also have an `environment` (dict: intensity, sun_dir, sun_intensity, sky_mode; or intensity,
    image (height, width, 4) float32 lat-long pixels and rotation in radians)."""
    lib = load()
    if not hasattr(lib.vto_render, "_typed"):
        lib.vto_render.restype, lib.vto_render.argtypes = _SIGS["vto_render"]
        lib.vto_render._typed = True
    f, v = _faces(faces), _verts(verts)
    mats = (Material * len(materials))()
    for i, m in enumerate(materials):
        mats[i].type = int(m["type"])
        mats[i].albedo[:] = [float(x) for x in m["albedo"]]
        mats[i].emission[:] = [float(x) for x in m["emission"]]
    q = QuadLight()
    if light is not None:
        for k in ("corner", "su", "sv", "normal", "emission"):
            getattr(q, k)[:] = [float(x) for x in light[k]]
    inp = PtInputs(f.ctypes.data, f.shape[0], v.ctypes.data, v.shape[0], C.cast(mats, C.c_void_p), len(materials), q,
                   None, None, None, 0, 0, 0.0, None, 0, 0, None, None, None, None, None)
    keep = []
    if any(int(m["type"]) in (1, 2, 4) for m in materials):
        # OPENPBR, GLOSSY and DIELECTRIC slots: their lobe parameters, and the reference's own BSDF
        # and mirror film (oracle/openpbr_ref).
        from . import openpbr_ref
        ref = openpbr_ref.load()
        params = np.array([[float(m.get("roughness", 0.5)), float(m.get("metalness", 0.0)), float(m.get("ior", 1.5)),
                            float(m.get("diffuse_roughness", 0.0)), float(m.get("thin_film_weight", 0.0)),
                            float(m.get("thin_film_thickness", 0.0)), float(m.get("thin_film_ior", 1.4)), float(m.get("coat", 0.0)),
                            float(m.get("fuzz", 0.0)), float(m.get("anisotropy", 0.0)), 0.0, 0.0]
                           for m in materials], np.float32)
        keep.append(params)
        inp.pbr_params = params.ctypes.data
        inp.pbr_eval = C.cast(ref.ref_openpbr_eval, C.c_void_p).value
        inp.pbr_sample = C.cast(ref.ref_openpbr_sample, C.c_void_p).value
        inp.pbr_film_mirror = C.cast(ref.ref_thin_film_mirror, C.c_void_p).value
    if light is None and environment is not None and float(environment.get("intensity", 0.0)) > 0.0:
        env = inp.environment
        env.intensity = float(environment["intensity"])
        env.sun_dir[:] = [float(x) for x in environment.get("sun_dir", (0.0, 1.0, 0.0))]
        env.sun_intensity = float(environment.get("sun_intensity", 0.0))
        env.sky_mode = int(environment.get("sky_mode", 0))
        if environment.get("image") is not None:
            img = np.ascontiguousarray(np.clip(np.asarray(environment["image"], np.float32), 0.0, None))
            keep.append(img)
            inp.env_rgba, inp.env_h, inp.env_w = img.ctypes.data, img.shape[0], img.shape[1]
            inp.env_rot = float(environment.get("rotation", 0.0))
    if light is None:
        if emitter_words is None:
            from . import light_tree as LT
            emitter_words = LT.emitter_list(*LT.scene_emitters(faces, verts, materials), light_tree=light_tree)
        words = np.ascontiguousarray(emitter_words, np.uint32)
        keep.append(words)
        inp.emitters, inp.nemitter_words, inp.imported = words.ctypes.data, len(words), 1
    if spectral is not None:
        cmf = np.ascontiguousarray(spectral["cmf_rgb"], np.float32)
        ill = np.ascontiguousarray(spectral["illum"], np.float32)
        icdf = np.ascontiguousarray(spectral["icdf"], np.float32)
        keep += [cmf, ill, icdf]
        inp.cmf_rgb, inp.illum, inp.icdf = cmf.ctypes.data, ill.ctypes.data, icdf.ctypes.data
        inp.nbins, inp.segments, inp.lambda_min = cmf.shape[0], icdf.shape[0] - 1, float(spectral["lambda_min"])
        cosp = np.ascontiguousarray(spectral["cos_phase"], np.float32)
        up = uplift_for(spectral)
        keep += [cosp, up]
        inp.uplift, inp.cos_phase = up._p, cosp.ctypes.data
    p = FrameParams()
    p.camera_pos[:] = [float(x) for x in camera["pos"]]
    p.camera_target[:] = [float(x) for x in camera["target"]]
    p.camera_up[:] = [float(x) for x in camera["up"]]
    p.fov_deg = float(camera["fov"])
    p.max_depth, p.sampling_mode, p.width, p.height = max_depth, mode, width, height
    p.first_sample, p.spectral = first_sample, 1 if spectral is not None else 0
    p.sampler, p.z_temporal, p.first_frame = sampler, z_temporal, first_frame
    p.di_candidates = di_candidates
    p.aperture, p.focus_distance = aperture, focus_distance
    stride = max(1, int(pixel_stride))
    p.pixel_stride = stride
    if bvh is not None:
        inp.bvh = bvh._h
        keep.append(bvh)
    oh, ow = (height, width) if mode == 0 else (-(-height // stride), -(-width // stride))
    out = np.empty(3 * ow * oh, np.float64)
    lib.vto_render(C.byref(inp), C.byref(p), spp, out.ctypes.data, nthreads or threads())
    return out.reshape(oh, ow, 3)


_SIGS["vto_z_sequences"] = (None, [_U32, _U32, _P, _P])
_SIGS["vto_z_shuffles"] = (None, [_U32, _U32, _U32, _P])
_SIGS["vto_sampler_frame"] = (None, [_U32, _U32, _I32, _U32, _U32, _U32, _U32, _U32, _P])


def _fn(name):
    fn = getattr(load(), name)
    fn.restype, fn.argtypes = _SIGS[name]
    return fn


def z_sequences(seed: int, n: int):
    """(O2m3 points (n, 3) uint32, Sobol' points (n, 2) uint32) as 0.32 fixed point."""
    o, q = np.empty((n, 3), np.uint32), np.empty((n, 2), np.uint32)
    _fn("vto_z_sequences")(seed, n, o.ctypes.data, q.ctypes.data)
    return o, q


def z_shuffles(base: int, dimension: int, n: int):
    out = np.empty(n, np.uint32)
    _fn("vto_z_shuffles")(base & 0xFFFFFFFF, dimension & 0xFFFFFFFF, n, out.ctypes.data)
    return out


def sampler_frame(width, height, z, model, sample_index, frame_index, vertex, stream):
    """(height, width, 6): rand_f, rand_f2 (2), rand_f3 (3) of one event per pixel."""
    out = np.empty((height, width, 6), np.float32)
    _fn("vto_sampler_frame")(width, height, 1 if z else 0, model, sample_index, frame_index, vertex, stream,
                             out.ctypes.data)
    return out


# ---- RGB -> spectrum uplift (spectral_uplift.cpp) ---------------------------------------------
_SIGS["vto_uplift_create"] = (_P, [_P, _P, _U32])
_SIGS["vto_uplift_destroy"] = (None, [_P])
_SIGS["vto_fourier_lagrange"] = (None, [_P, _P])
_SIGS["vto_uplift_solve_code"] = (C.c_double, [_P, _P, _P, _P])
_SIGS["vto_uplift_rgb_of_lagrange"] = (None, [_P, _P, _P])
_SIGS["vto_uplift_moments_of_lagrange"] = (None, [_P, _P])
_SIGS["vto_uplift_node"] = (None, [_P, _U32, _U32, _U32, _P])
_SIGS["vto_uplift_code_error"] = (C.c_double, [_P, _P])
_SIGS["vto_uplift_cell_refined"] = (_I32, [_P, _P])
_SIGS["vto_spectral_lagrange"] = (None, [_P, _P, _U32, _P])


def fourier_lagrange(c) -> np.ndarray:
    """Bounded-MESE Lagrange multipliers of three moments (with the biasing of invalid ones)."""
    c = np.ascontiguousarray(c, np.float64)
    out = np.empty(3, np.float64)
    _fn("vto_fourier_lagrange")(c.ctypes.data, out.ctypes.data)
    return out


def moments_of_lagrange(L) -> np.ndarray:
    L = np.ascontiguousarray(L, np.float64)
    out = np.empty(3, np.float64)
    _fn("vto_uplift_moments_of_lagrange")(L.ctypes.data, out.ctypes.data)
    return out


class Uplift:
    """The uplift's colour model (spectral_tables.load()['uplift_w'], ['uplift_cos']) with the
    lazily solved moment grid."""

    def __init__(self, weights, cos_phi):
        self._w = np.ascontiguousarray(weights, np.float64)
        self._c = np.ascontiguousarray(cos_phi, np.float64)
        self._p = _fn("vto_uplift_create")(self._w.ctypes.data, self._c.ctypes.data, self._c.shape[0])

    def solve_code(self, code):
        code = np.ascontiguousarray(code, np.uint32)
        m, L = np.empty(3, np.float64), np.empty(3, np.float64)
        err = _fn("vto_uplift_solve_code")(self._p, code.ctypes.data, m.ctypes.data, L.ctypes.data)
        return m, L, err

    def rgb_of_lagrange(self, L):
        L = np.ascontiguousarray(L, np.float64)
        out = np.empty(3, np.float64)
        _fn("vto_uplift_rgb_of_lagrange")(self._p, L.ctypes.data, out.ctypes.data)
        return out

    def node(self, i, j, k):
        out = np.empty(3, np.float64)
        _fn("vto_uplift_node")(self._p, i, j, k, out.ctypes.data)
        return out

    def code_error(self, code):
        code = np.ascontiguousarray(code, np.uint32)
        return _fn("vto_uplift_code_error")(self._p, code.ctypes.data)

    def cell_refined(self, cell):
        cell = np.ascontiguousarray(cell, np.uint32)
        return bool(_fn("vto_uplift_cell_refined")(self._p, cell.ctypes.data))

    def lagrange(self, rgb):
        """spectral_lagrange of linear colours (n, 3) -> (n, 4): L0, L1, L2, flag (2 = flat L0)."""
        rgb = np.ascontiguousarray(np.atleast_2d(rgb), np.float64)
        out = np.empty((rgb.shape[0], 4), np.float64)
        _fn("vto_spectral_lagrange")(self._p, rgb.ctypes.data, rgb.shape[0], out.ctypes.data)
        return out

    def close(self):
        if getattr(self, "_p", None):
            _fn("vto_uplift_destroy")(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reflectance(L4, cos_phi):
    """Eq. 11 at cos(phi) values; a flat quadruple (flag 2) gives its value."""
    L4 = np.asarray(L4, np.float64)
    x = np.asarray(cos_phi, np.float64)
    if L4[3] == 2.0:
        return np.full(x.shape, L4[0])
    return np.arctan(L4[0] + 2.0 * L4[1] * x + 2.0 * L4[2] * (2.0 * x * x - 1.0)) / np.pi + 0.5


_UPLIFTS = {}


def uplift_for(spectral) -> "Uplift":
    """One oracle uplift per colour model (its solved grid nodes are kept between renders)."""
    key = (np.asarray(spectral["uplift_w"], np.float64).tobytes(), np.asarray(spectral["uplift_cos"], np.float64).tobytes())
    key = hash(key)
    if key not in _UPLIFTS:
        _UPLIFTS[key] = Uplift(spectral["uplift_w"], spectral["uplift_cos"])
    return _UPLIFTS[key]
