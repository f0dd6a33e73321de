"""Path tracing on the B200: scenes, frames and the FP64 accumulation (host side of include/vt.h).

The roles of the reference's renderer: `MaterialLibrary` resources and bind (main.swift:9432-9449),
`renderFrame(output:samples:)` / `encodeSample` (main.swift:10978, 11214-11708) for the MIS
integrator (shading_kernel, main.swift:7370-7914), and the accumulation read back as linear sRGB.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .accel import Context, MaterialLibraryError, Mesh, _check

VT_MAT_DIFFUSE, VT_MAT_GLOSSY, VT_MAT_DIELECTRIC, VT_MAT_EMISSIVE, VT_MAT_OPENPBR = 0, 1, 2, 3, 4


class Material(C.Structure):
    _fields_ = [("type", C.c_int32), ("albedo", C.c_float * 3), ("emission", C.c_float * 3), ("pad", C.c_float)]


class QuadLight(C.Structure):
    _fields_ = [("corner", C.c_float * 3), ("su", C.c_float * 3), ("sv", C.c_float * 3), ("normal", C.c_float * 3),
                ("emission", C.c_float * 3), ("pad", C.c_float)]


class SpectralTables(C.Structure):
    _fields_ = [("cmf_rgb", C.c_void_p), ("illuminant", C.c_void_p), ("icdf", C.c_void_p),
                ("nbins", C.c_uint32), ("segments", C.c_uint32), ("lambda_min", C.c_float), ("pad", C.c_uint32),
                ("cos_phase", C.c_void_p), ("uplift_weights", C.c_void_p), ("uplift_cos", C.c_void_p),
                ("uplift_n", C.c_uint32), ("pad2", C.c_uint32)]


def spectral_struct(spectral: dict):
    """vt_spectral_tables for a spectral_tables.load() dict, with the arrays it points to (keep
    them alive as long as the struct is used)."""
    arrays = [np.ascontiguousarray(spectral["cmf_rgb"], np.float32), np.ascontiguousarray(spectral["illum"], np.float32),
              np.ascontiguousarray(spectral["icdf"], np.float32), np.ascontiguousarray(spectral["cos_phase"], np.float32),
              np.ascontiguousarray(spectral["uplift_w"], np.float64), np.ascontiguousarray(spectral["uplift_cos"], np.float64)]
    cmf, ill, icdf, cosp, uw, uc = arrays
    if uw.shape != (uc.shape[0], 3) or cosp.shape[0] != cmf.shape[0] or ill.shape[0] != cmf.shape[0]:
        raise ValueError("spectral tables: uplift_w must be (len(uplift_cos), 3) and cos_phase / illum one per bin")
    s = SpectralTables(cmf.ctypes.data, ill.ctypes.data, icdf.ctypes.data, cmf.shape[0], icdf.shape[0] - 1,
                       float(spectral["lambda_min"]), 0, cosp.ctypes.data, uw.ctypes.data, uc.ctypes.data, uc.shape[0], 0)
    return s, arrays


class FrameParams(C.Structure):
    _fields_ = [("camera_pos", C.c_float * 3), ("fov_deg", C.c_float), ("camera_target", C.c_float * 3),
                ("max_depth", C.c_uint32), ("camera_up", C.c_float * 3), ("sampling_mode", C.c_uint32),
                ("width", C.c_uint32), ("height", C.c_uint32), ("first_sample", C.c_uint32),
                ("spectral", C.c_uint32), ("sampler", C.c_uint32), ("z_temporal", C.c_uint32),
                ("first_frame", C.c_uint32), ("di_candidates", C.c_uint32),
                ("aperture", C.c_float), ("focus_distance", C.c_float), ("pixel_stride", C.c_uint32)]


assert C.sizeof(Material) == 32 and C.sizeof(QuadLight) == 64 and C.sizeof(FrameParams) == 92


def make_materials(materials) -> C.Array:
    arr = (Material * len(materials))()
    for i, m in enumerate(materials):
        arr[i].type = int(m["type"])
        arr[i].albedo[:] = [float(x) for x in m["albedo"]]
        arr[i].emission[:] = [float(x) for x in m["emission"]]
    return arr


def make_light(light) -> QuadLight:
    q = QuadLight()
    for k in ("corner", "su", "sv", "normal", "emission"):
        getattr(q, k)[:] = [float(x) for x in light[k]]
    return q


def make_params(camera, width, height, max_depth=8, first_sample=1, spectral=True, mode=1, sampler=0, z_temporal=3,
                first_frame=0, di_candidates=0, aperture=0.0, focus_distance=1.0, pixel_stride=1) -> FrameParams:
    p = FrameParams()
    p.camera_pos[:] = [float(x) for x in camera["pos"]]
    p.camera_target[:] = [float(x) for x in camera["target"]]
    p.camera_up[:] = [float(x) for x in camera["up"]]
    p.fov_deg = float(camera["fov"])
    p.max_depth = int(max_depth)
    p.sampling_mode = int(mode)  # 0 ReSTIR DI, 1 MIS, 2 light sampling, 3 BSDF sampling (Uniforms.samplingMode)
    p.width, p.height = int(width), int(height)
    p.first_sample = int(first_sample)
    p.spectral = 1 if spectral else 0
    p.sampler = int(sampler)          # 0 PCG, 1 Z++
    p.z_temporal = int(z_temporal)    # Z++ temporal model (the reference's default: 3, reshuffled)
    p.first_frame = int(first_frame)  # 0: continue the scene's accumulation
    p.di_candidates = int(di_candidates)  # ReSTIR DI candidates (0: the reference's 4)
    p.aperture, p.focus_distance = float(aperture), float(focus_distance)  # thin lens (0: pinhole)
    p.pixel_stride = int(pixel_stride)  # s > 1: pixels (s i, s j) only (sampling modes 1-3)
    return p


def accum_shape(params: FrameParams) -> tuple[int, int]:
    """(height, width) of the accumulation a frame renders into: the frame's, or ceil(h / s) x
    ceil(w / s) at a pixel stride s."""
    s = max(1, int(params.pixel_stride))
    return (params.height + s - 1) // s, (params.width + s - 1) // s


class Scene:
    """A renderable scene on the device (vt_scene): mesh, material slots, the lights, spectral
    tables and the FP64 accumulation.

    With a quad `light` the scene is lit as the reference's procedural scenes (sample_direct_light's
    quad branch). With light=None it is an imported scene (sceneIndex 6): every face whose slot is
    emissive is an emitter, chosen by power or, with light_tree=True (the reference's default), by
    walking the light tree."""

    def __init__(self, ctx: Context, mesh: Mesh, materials, light=None, spectral: dict | None = None,
                 light_tree: bool = True):
        lib = _lib.load()
        self.ctx, self.mesh = ctx, mesh
        self._mats = make_materials(materials)
        self.imported = light is None
        self._light = None if light is None else make_light(light)
        tables = None
        if spectral is not None:
            tables, self._spectral_arrays = spectral_struct(spectral)
        p = C.c_void_p()
        tp = C.byref(tables) if tables is not None else None
        if self.imported:
            st = lib.vt_scene_create_imported(ctx.handle, mesh._p, self._mats, len(materials), tp,
                                              1 if light_tree else 0, C.byref(p))
            _check(ctx.handle, st, "vt_scene_create_imported")
        else:
            st = lib.vt_scene_create(ctx.handle, mesh._p, self._mats, len(materials), C.byref(self._light), tp,
                                     C.byref(p))
            _check(ctx.handle, st, "vt_scene_create")
        self._p = p
        self.width = self.height = 0
        if any(int(m["type"]) in (VT_MAT_GLOSSY, VT_MAT_DIELECTRIC, VT_MAT_OPENPBR) for m in materials):
            # OPENPBR, GLOSSY and DIELECTRIC slots: roughness, metalness, IOR and diffuse roughness per
            # slot (the reference's SurfaceSettings surface.x/y and detail.y; base colour is the albedo;
            # a GLOSSY slot below roughness 0.02 is a mirror, a DIELECTRIC slot ideal glass).
            openpbr_tables_set(ctx)
            params = (_lib.OpenPBRParams * len(materials))()
            for i, m in enumerate(materials):
                params[i].roughness = float(m.get("roughness", 0.5))
                params[i].metalness = float(m.get("metalness", 0.0))
                params[i].ior = float(m.get("ior", 1.5))
                params[i].diffuse_roughness = float(m.get("diffuse_roughness", 0.0))
                # Thin film (spectral transport only): weight, thickness in micrometres, IOR.
                params[i].thin_film_weight = float(m.get("thin_film_weight", 0.0))
                params[i].thin_film_thickness = float(m.get("thin_film_thickness", 0.0))
                params[i].thin_film_ior = float(m.get("thin_film_ior", 1.4))
                params[i].coat = float(m.get("coat", 0.0))
                params[i].fuzz = float(m.get("fuzz", 0.0))
                params[i].anisotropy = float(m.get("anisotropy", 0.0))
            _check(ctx.handle, lib.vt_scene_set_openpbr(ctx.handle, self._p, params, len(materials)), "vt_scene_set_openpbr")

    def set_environment(self, intensity: float = 0.0, sun_dir=(0.0, 1.0, 0.0), sun_intensity: float = 0.0,
                        sky_mode: int = 0) -> None:
        """The procedural sky and sun of an imported scene (vt_scene_set_environment; the reference's
        Uniforms.environment.x, sunParams and skyMode); intensity 0 removes it. Restarts the
        accumulation."""
        e = _lib.Environment()
        e.intensity = float(intensity)
        e.sun_dir[:] = [float(x) for x in sun_dir]
        e.sun_intensity = float(sun_intensity)
        e.sky_mode = int(sky_mode)
        _check(self.ctx.handle, _lib.load().vt_scene_set_environment(self.ctx.handle, self._p, C.byref(e)),
               "vt_scene_set_environment")

    def set_environment_map(self, image, intensity: float = 1.0, rotation: float = 0.0) -> None:
        """An equirectangular environment image instead of the procedural sky
        (vt_scene_set_environment_map): `image` is (height, width, 3 or 4) float linear sRGB, row 0
        toward +y; `rotation` turns it about +y (radians). None removes it. Restarts the accumulation."""
        lib = _lib.load()
        if image is None:
            _check(self.ctx.handle, lib.vt_scene_set_environment_map(self.ctx.handle, self._p, None, 0, 0, 0.0, 0.0),
                   "vt_scene_set_environment_map")
            return
        img = np.asarray(image, np.float32)
        if img.ndim != 3 or img.shape[2] not in (3, 4):
            raise ValueError("image must be (height, width, 3 or 4)")
        if img.shape[2] == 3:
            img = np.concatenate([img, np.ones(img.shape[:2] + (1,), np.float32)], axis=2)
        img = np.ascontiguousarray(img)
        _check(self.ctx.handle, lib.vt_scene_set_environment_map(self.ctx.handle, self._p, img.ctypes.data, img.shape[1],
                                                                 img.shape[0], float(intensity), float(rotation)),
               "vt_scene_set_environment_map")

    def emitter_words(self) -> np.ndarray:
        """The packed emitter list of an imported scene (uint32 words)."""
        lib = _lib.load()
        n = C.c_uint32()
        _check(self.ctx.handle, lib.vt_scene_emitter_words(self.ctx.handle, self._p, None, 0, C.byref(n)),
               "vt_scene_emitter_words")
        out = np.empty(n.value, np.uint32)
        _check(self.ctx.handle, lib.vt_scene_emitter_words(self.ctx.handle, self._p, out.ctypes.data, n.value,
                                                           C.byref(n)), "vt_scene_emitter_words")
        return out

    def di_weights(self) -> np.ndarray:
        """(height, width, 4) float32 ReSTIR DI reservoir weights of the last mode-0 frame:
        weight sum, M, W, wavelength number."""
        out = np.empty((self.height, self.width, 4), np.float32)
        _check(self.ctx.handle, _lib.load().vt_scene_di_weights(self.ctx.handle, self._p, out.ctypes.data, out.size),
               "vt_scene_di_weights")
        return out

    def gi_weights(self) -> np.ndarray:
        """(height, width, 4) float32 ReSTIR GI reservoir weights of the last mode-0 frame: weight sum,
        M, W, wavelength number (M 0 where no GI reservoir was built)."""
        out = np.empty((self.height, self.width, 4), np.float32)
        _check(self.ctx.handle, _lib.load().vt_scene_gi_weights(self.ctx.handle, self._p, out.ctypes.data, out.size),
               "vt_scene_gi_weights")
        return out

    def light_estimate(self, points, per_point: int, samples: int = 64) -> np.ndarray:
        """The reference's lt_estimate check on the device: (npoints * per_point, 8) float32 per
        thread (sum, squares, hits, zero pdfs, max pdf error, back-facing choices, 0, 0)."""
        pts = np.zeros((len(points), 4), np.float32)
        pts[:, :3] = np.asarray(points, np.float32)[:, :3]
        out = np.empty((len(points) * per_point, 8), np.float32)
        _check(self.ctx.handle, _lib.load().vt_light_estimate(self.ctx.handle, self._p, pts.ctypes.data, len(points),
                                                              int(per_point), int(samples), out.ctypes.data),
               "vt_light_estimate")
        return out

    def render(self, params: FrameParams, spp: int, stream=None) -> None:
        """Adds `spp` frames (one sample per pixel each) to the accumulation; stream-ordered."""
        self.height, self.width = accum_shape(params)
        _check(self.ctx.handle, _lib.load().vt_render(self.ctx.handle, self._p, C.byref(params), int(spp), stream),
               "vt_render")

    def render_wavefront(self, params: FrameParams, spp: int, stream=None) -> None:
        """The same frames through the wavefront integrator (vt_render_wavefront; sampling modes 1-3)."""
        self.height, self.width = accum_shape(params)
        _check(self.ctx.handle, _lib.load().vt_render_wavefront(self.ctx.handle, self._p, C.byref(params), int(spp),
                                                                stream), "vt_render_wavefront")

    def reset(self) -> None:
        _check(self.ctx.handle, _lib.load().vt_accum_reset(self.ctx.handle, self._p), "vt_accum_reset")

    def readback(self) -> tuple[np.ndarray, int]:
        """(height, width, 3) float64 mean radiance and the sample count."""
        n = 3 * self.width * self.height
        out = np.empty(n, np.float64)
        samples = C.c_uint32()
        _check(self.ctx.handle, _lib.load().vt_accum_readback(self.ctx.handle, self._p, out.ctypes.data, n,
                                                              C.byref(samples)), "vt_accum_readback")
        return out.reshape(self.height, self.width, 3), int(samples.value)

    def save_accumulation(self, path, params: FrameParams) -> int:
        """Save the accumulation (mean radiance in FP64 and its sample count, with the frame's size and
        pixel stride) to an .npz file, to resume a long render later (restore_accumulation); returns
        the sample count."""
        img, n = self.readback()
        np.savez(path, rgb=img, samples=n, width=params.width, height=params.height,
                 pixel_stride=max(1, int(params.pixel_stride)))
        return n

    def restore_accumulation(self, path) -> int:
        """Resume an accumulation saved by save_accumulation (vt_accum_restore); the next render
        continues it with first_sample = the returned sample count + 1."""
        d = np.load(path)
        rgb = np.ascontiguousarray(d["rgb"], np.float64)
        w, h, s, n = int(d["width"]), int(d["height"]), int(d["pixel_stride"]), int(d["samples"])
        _check(self.ctx.handle, _lib.load().vt_accum_restore(self.ctx.handle, self._p, w, h, s, rgb.ctypes.data,
                                                             rgb.size, n), "vt_accum_restore")
        self.height, self.width = rgb.shape[0], rgb.shape[1]
        return n

    def save_exr(self, path) -> int:
        """Write the accumulation's mean radiance as a FLOAT RGB OpenEXR (the reference's HDR export);
        returns the sample count."""
        from .exr import write_exr
        img, n = self.readback()
        write_exr(path, img)
        return n

    def close(self) -> None:
        if getattr(self, "_p", None) is not None and self.ctx._p is not None:
            _lib.load().vt_scene_destroy(self.ctx.handle, self._p)
        self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sampler_frame(ctx: Context, width: int, height: int, z: bool, model: int, sample_index: int, frame_index: int,
                  vertex: int, stream: int) -> np.ndarray:
    """(height, width, 6) float32: rand_f, rand_f2, rand_f3 of one sampling event per pixel, drawn on
    the device (the sampler's diagnostic entry point)."""
    out = np.empty((height, width, 6), np.float32)
    _check(ctx.handle, _lib.load().vt_sampler_frame(ctx.handle, width, height, 1 if z else 0, model, sample_index,
                                                    frame_index, vertex, stream, out.ctypes.data), "vt_sampler_frame")
    return out


def known_answers(ctx: Context) -> np.ndarray:
    """The reference's device known answers (regression_checks, tests/GPUChecks.swift:14-37) as the
    integrator's device functions compute them: power heuristic, emission weights, the grazing
    cosine sample, rand_f's range, the scattering budget and glass total internal reflection
    (layout in include/vt.h)."""
    out = np.empty(_lib.KNOWN_ANSWERS, np.float32)
    _check(ctx.handle, _lib.load().vt_known_answers(ctx.handle, out.ctypes.data, out.size), "vt_known_answers")
    return out


class Batch:
    """Scenes rendered by one persistent launch per pass (vt_batch): each pass adds spp[i] frames to
    scene i. The first six passes try launch shapes; later passes replay a captured CUDA graph."""

    def __init__(self, ctx: Context, scenes, params, spp):
        lib = _lib.load()
        self.ctx, self.scenes = ctx, list(scenes)
        n = len(self.scenes)
        self._ptrs = (C.c_void_p * n)(*[sc._p.value for sc in self.scenes])
        self._params = (FrameParams * n)(*params)
        self._spp = (C.c_uint32 * n)(*[int(x) for x in spp])
        p = C.c_void_p()
        _check(ctx.handle, lib.vt_batch_create(ctx.handle, self._ptrs, self._params, self._spp, n, C.byref(p)),
               "vt_batch_create")
        self._p = p
        for sc, prm in zip(self.scenes, params):
            sc.width, sc.height = prm.width, prm.height

    def render(self, stream=None) -> float:
        """One pass; returns its device time in ms."""
        _check(self.ctx.handle, _lib.load().vt_batch_render(self.ctx.handle, self._p, stream), "vt_batch_render")
        return self.stats()[0].last_ms

    def render_wavefront(self, stream=None) -> float:
        """One pass through the wavefront integrator (per-scene queues on four streams); the first
        passes try queue size x block size x compaction frequency. Returns its device time in ms."""
        _check(self.ctx.handle, _lib.load().vt_batch_render_wavefront(self.ctx.handle, self._p, stream),
               "vt_batch_render_wavefront")
        return self.stats()[0].last_ms

    def stats(self):
        """(vt_batch_stats, per-scene completion ms of the last pass)."""
        st = _lib.BatchStats()
        ms = np.zeros(len(self.scenes), np.float64)
        _check(self.ctx.handle, _lib.load().vt_batch_stats(self.ctx.handle, self._p, C.byref(st), ms.ctypes.data,
                                                           len(self.scenes)), "vt_batch_stats")
        return st, ms

    def close(self) -> None:
        if getattr(self, "_p", None) is not None and self.ctx._p is not None:
            _lib.load().vt_batch_destroy(self.ctx.handle, self._p)
        self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass



# ---- RGB -> spectrum uplift (spectral.cu) -----------------------------------------------------
def spectral_grid_build(ctx: Context, spectral: dict) -> None:
    """Solve the context's uplift moment grid for the tables' colour model (once per context)."""
    s, keep = spectral_struct(spectral)
    _check(ctx.handle, _lib.load().vt_spectral_grid_build(ctx.handle, C.byref(s)), "vt_spectral_grid_build")
    del keep


def spectral_grid_info(ctx: Context) -> dict:
    info = _lib.SpectralGridInfo()
    _check(ctx.handle, _lib.load().vt_spectral_grid_get_info(ctx.handle, C.byref(info)), "vt_spectral_grid_get_info")
    return {"built": bool(info.built), "refined_cells": int(info.refined_cells), "flagged_cells": int(info.flagged_cells),
            "max_residual": float(info.max_residual)}


def spectral_grid(ctx: Context) -> np.ndarray:
    """The grid as (86^3 + 64 * refined cells, 4) float32: c0, c1, c2, refined slot + 1."""
    n = 86 ** 3 + 64 * spectral_grid_info(ctx)["refined_cells"]
    out = np.empty((n, 4), np.float32)
    _check(ctx.handle, _lib.load().vt_spectral_grid_read(ctx.handle, out.ctypes.data, out.size), "vt_spectral_grid_read")
    return out


def spectral_lagrange(ctx: Context, rgb) -> np.ndarray:
    """Device spectral_lagrange of linear colours (n, 3) -> (n, 4)."""
    rgb = np.ascontiguousarray(np.atleast_2d(rgb), np.float32)
    out = np.empty((rgb.shape[0], 4), np.float32)
    _check(ctx.handle, _lib.load().vt_spectral_lagrange(ctx.handle, rgb.ctypes.data, rgb.shape[0], out.ctypes.data),
           "vt_spectral_lagrange")
    return out


def spectral_round_trip(ctx: Context) -> tuple[float, int]:
    """(largest 8-bit error over every code, codes off by more than half a step)."""
    worst, over = C.c_float(), C.c_uint32()
    _check(ctx.handle, _lib.load().vt_spectral_round_trip(ctx.handle, C.byref(worst), C.byref(over)),
           "vt_spectral_round_trip")
    return float(worst.value), int(over.value)


# ---- OpenPBR (openpbr.cu) ---------------------------------------------------------------------
def openpbr_tables_set(ctx: Context) -> None:
    """Hand the context the OpenPBR energy tables (once; data/openpbr_energy.bin)."""
    if getattr(ctx, "_pbr_tables_set", False):
        return
    from . import openpbr_tables
    t = openpbr_tables.load()
    e, a, ltc = t["opaque_energy"], t["opaque_average"], t["ltc"]
    s = _lib.OpenPBRTables(e.ctypes.data, a.ctypes.data, ltc.ctypes.data)
    _check(ctx.handle, _lib.load().vt_openpbr_tables_set(ctx.handle, C.byref(s)), "vt_openpbr_tables_set")
    ctx._pbr_tables_set = True


def openpbr_energy_table(ctx: Context) -> tuple[np.ndarray, np.ndarray]:
    """The dense GGX energy complement solved on the device: (129, 129) and (129,)."""
    table = np.empty((129, 129), np.float32)
    avg = np.empty(129, np.float32)
    _check(ctx.handle, _lib.load().vt_openpbr_energy_table(ctx.handle, table.ctypes.data, avg.ctypes.data),
           "vt_openpbr_energy_table")
    return table, avg


def openpbr_evaluate(ctx: Context, cases) -> np.ndarray:
    """BSDF queries on the device: `cases` is an (n, 20) float32 array of the _lib.OpenPBRCase fields
    up to `rand` (no thin film, the upstream RGB wavelengths, no coat or fuzz), (n, 26) with the thin
    film's weight, thickness (micrometres) and IOR and the three wavelengths (nm), (n, 28) with the
    coat and fuzz weights as well, or (n, 32) with the anisotropy and the unit tangent; returns (n, 12)
    float32 results (f_cos, pdf, dir, weight, sample_pdf, ok)."""
    arr = np.asarray(cases, np.float32)
    if arr.ndim == 2 and arr.shape[1] in (20, 26, 27, 28):
        arr = np.concatenate([arr, np.zeros((arr.shape[0], 32 - arr.shape[1]), np.float32)], axis=1)
    arr = np.ascontiguousarray(arr, np.float32).reshape(-1, 32)
    out = np.empty((arr.shape[0], 12), np.float32)
    _check(ctx.handle, _lib.load().vt_openpbr_evaluate(ctx.handle, arr.ctypes.data, arr.shape[0], out.ctypes.data),
           "vt_openpbr_evaluate")
    return out


def environment_tables(image):
    """The environment image's sampling tables as vt_scene_set_environment_map builds them (host code
    of the library): (rows (height, 2), cols (2, height, width)); table 0 compensated, 1 original."""
    img = np.asarray(image, np.float32)
    if img.shape[2] == 3:
        img = np.concatenate([img, np.ones(img.shape[:2] + (1,), np.float32)], axis=2)
    img = np.ascontiguousarray(img)
    h, w = img.shape[:2]
    rows = np.empty((h, 2), np.float32)
    cols = np.empty((2, h, w), np.float32)
    st = _lib.load().vt_environment_tables(img.ctypes.data, w, h, rows.ctypes.data, cols.ctypes.data)
    if st != _lib.VT_OK:
        raise ValueError("vt_environment_tables failed")
    return rows, cols

