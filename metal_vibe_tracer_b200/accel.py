"""Mesh acceleration structures and ray queries on the B200 (the host side of include/vt.h).

This is the Python face of the reference's acceleration-structure role: a mesh publish
(``MaterialLibrary.setMesh`` -> ``publishTwoLevel``, Sources/Acceleration.swift:652-782), its
``WideBVH.build`` (Sources/Acceleration.swift:296; Result = order, nodes, depth) and the
``mesh_closest`` / ``mesh_occluded`` queries (main.swift:1843-1984). Build and traversal run in
libvt_b200.so; failures raise :class:`MaterialLibraryError`, the reference's
``MaterialLibrary.error(String)``.

Rays may be host numpy arrays (RAY_DTYPE or (n, 8) float32: the call copies in and out through
the library's pipelined host path) or CUDA torch tensors of shape (n, 8) float32 (device path,
stream-ordered on torch's current stream).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (FACE_DTYPE, HIT_DTYPE, INSTANCE_DTYPE, INSTANCE_RECORD_DTYPE, RAY_DTYPE, VERTEX_DTYPE,
                   WIDE_NODE_DTYPE, BuildOptions, MeshInfo, TlasInfo)


class MaterialLibraryError(RuntimeError):
    """A failed publish or query, with the library's message (MaterialLibrary.error)."""


def _check(ctx_ptr, status: int, what: str) -> None:
    if status != _lib.VT_OK:
        lib = _lib.load()
        msg = lib.vt_last_error(ctx_ptr)
        msg = msg.decode() if msg else ""
        raise MaterialLibraryError(f"{what}: {_lib.STATUS_NAMES.get(status, status)}: {msg}")


class Context:
    """One CUDA device and its stream (vt_ctx). Single-threaded, like the reference renderer."""

    def __init__(self, device: int = 0):
        lib = _lib.load()
        p = C.c_void_p()
        st = lib.vt_ctx_create(int(device), C.byref(p))
        if st != _lib.VT_OK:
            msg = lib.vt_last_error(None)
            raise MaterialLibraryError(f"vt_ctx_create: {_lib.STATUS_NAMES.get(st, st)}: "
                                       f"{msg.decode() if msg else ''}")
        self._p = p
        self.device = device

    @property
    def handle(self) -> C.c_void_p:
        if self._p is None:
            raise MaterialLibraryError("context is closed")
        return self._p

    def sync(self) -> None:
        _check(self._p, _lib.load().vt_sync(self.handle), "vt_sync")

    def close(self) -> None:
        if getattr(self, "_p", None) is not None:
            _lib.load().vt_ctx_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclass
class WideBVHResult:
    """WideBVH.Result (Sources/Acceleration.swift:107-111): leaf order, 4-wide nodes, depth."""
    order: np.ndarray
    nodes: np.ndarray
    depth: int


def as_faces(faces) -> np.ndarray:
    a = np.asarray(faces)
    if a.dtype == FACE_DTYPE:
        return np.ascontiguousarray(a)
    a = np.ascontiguousarray(a, dtype=np.uint32)
    if a.ndim != 2 or a.shape[1] not in (3, 4):
        raise MaterialLibraryError("faces must be (n, 3) or (n, 4) uint32 or FACE_DTYPE")
    if a.shape[1] == 3:
        a = np.concatenate([a, np.zeros((a.shape[0], 1), np.uint32)], axis=1)
    return np.ascontiguousarray(a).view(FACE_DTYPE).reshape(-1)


def as_vertices(verts) -> np.ndarray:
    a = np.asarray(verts)
    if a.dtype == VERTEX_DTYPE:
        return np.ascontiguousarray(a)
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] not in (3, 8):
        raise MaterialLibraryError("vertices must be (n, 3) or (n, 8) float32 or VERTEX_DTYPE")
    if a.shape[1] == 3:
        a = np.concatenate([a, np.zeros((a.shape[0], 5), np.float32)], axis=1)
    return np.ascontiguousarray(a).view(VERTEX_DTYPE).reshape(-1)


def as_rays(rays) -> np.ndarray:
    a = np.asarray(rays)
    if a.dtype == RAY_DTYPE:
        return np.ascontiguousarray(a)
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] != 8:
        raise MaterialLibraryError("rays must be (n, 8) float32 (o, tmin, d, tmax) or RAY_DTYPE")
    return a.view(RAY_DTYPE).reshape(-1)


def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


class Mesh:
    """A published mesh: its device acceleration structure (vt_mesh)."""

    def __init__(self, ctx: Context, faces, vertices, *, leaf_size: int = 2, treelet_size: int = 7,
                 refine_rounds: int = 2, max_depth: int = 31):
        lib = _lib.load()
        self.ctx = ctx
        opts = BuildOptions(leaf_size, treelet_size, refine_rounds, max_depth)
        p = C.c_void_p()
        if _is_torch_cuda(faces):
            import torch
            if faces.dtype not in (torch.int32, torch.uint32) or faces.shape[-1] != 4:
                raise MaterialLibraryError("device faces must be (n, 4) int32")
            if not (_is_torch_cuda(vertices) and vertices.dtype == torch.float32 and vertices.shape[-1] == 8):
                raise MaterialLibraryError("device vertices must be (m, 8) float32 CUDA")
            faces = faces.contiguous()
            vertices = vertices.contiguous()
            torch.cuda.current_stream().synchronize()
            st = lib.vt_mesh_build_device(ctx.handle, faces.data_ptr(), faces.shape[0], vertices.data_ptr(),
                                          vertices.shape[0], C.byref(opts), C.byref(p))
        else:
            f = as_faces(faces)
            v = as_vertices(vertices)
            st = lib.vt_mesh_build(ctx.handle, f.ctypes.data, f.shape[0], v.ctypes.data, v.shape[0],
                                   C.byref(opts), C.byref(p))
        _check(ctx.handle, st, "vt_mesh_build")
        self._p = p

    @classmethod
    def _adopt(cls, ctx: Context, handle: C.c_void_p) -> "Mesh":
        """Wraps a vt_mesh the library built (vt_tlas_flatten)."""
        m = cls.__new__(cls)
        m.ctx = ctx
        m._p = handle
        return m

    # ---- inspection -------------------------------------------------------------------------
    def info(self) -> MeshInfo:
        out = MeshInfo()
        _check(self.ctx.handle, _lib.load().vt_mesh_get_info(self.ctx.handle, self._p, C.byref(out)),
               "vt_mesh_get_info")
        return out

    def order(self) -> np.ndarray:
        n = self.info().faces
        out = np.empty(n, np.int32)
        _check(self.ctx.handle, _lib.load().vt_mesh_get_order(self.ctx.handle, self._p, out.ctypes.data, n),
               "vt_mesh_get_order")
        return out

    def nodes(self) -> np.ndarray:
        n = self.info().wide_nodes
        out = np.empty(n, WIDE_NODE_DTYPE)
        _check(self.ctx.handle, _lib.load().vt_mesh_get_nodes(self.ctx.handle, self._p, out.ctypes.data, n),
               "vt_mesh_get_nodes")
        return out

    def wide_bvh(self) -> WideBVHResult:
        return WideBVHResult(self.order(), self.nodes(), int(self.info().depth))

    def morton(self) -> tuple[np.ndarray, np.ndarray]:
        n = self.info().faces
        codes = np.empty(n, np.uint32)
        sorted_ = np.empty(n, np.int32)
        _check(self.ctx.handle, _lib.load().vt_mesh_get_morton(self.ctx.handle, self._p, codes.ctypes.data,
                                                               sorted_.ctypes.data, n), "vt_mesh_get_morton")
        return codes, sorted_

    def binary(self) -> tuple[np.ndarray, np.ndarray]:
        n = max(0, self.info().faces - 1)
        ch = np.empty((n, 2), np.int32)
        boxes = np.empty((n, 6), np.float32)
        _check(self.ctx.handle, _lib.load().vt_mesh_get_binary(self.ctx.handle, self._p, ch.ctypes.data,
                                                               boxes.ctypes.data, n), "vt_mesh_get_binary")
        return ch, boxes

    # ---- queries ----------------------------------------------------------------------------
    def closest(self, rays, out=None):
        """Closest hits. numpy rays -> numpy HIT_DTYPE; CUDA tensor (n, 8) -> CUDA tensor (n, 4)."""
        lib = _lib.load()
        if _is_torch_cuda(rays):
            import torch
            r = rays.contiguous()
            n = r.shape[0]
            if out is None:
                out = torch.empty((n, 4), dtype=torch.float32, device=r.device)
            stream = torch.cuda.current_stream(r.device).cuda_stream
            _check(self.ctx.handle, lib.vt_trace_closest(self.ctx.handle, self._p, r.data_ptr(), n,
                                                         out.data_ptr(), stream), "vt_trace_closest")
            return out
        r = as_rays(rays)
        hits = np.empty(r.shape[0], HIT_DTYPE) if out is None else out
        _check(self.ctx.handle, lib.vt_trace_closest_host(self.ctx.handle, self._p, r.ctypes.data, r.shape[0],
                                                          hits.ctypes.data), "vt_trace_closest_host")
        return hits

    def occluded(self, rays, out=None):
        """Any hit in [tmin, tmax). numpy -> uint8 numpy; CUDA tensor -> uint8 CUDA tensor."""
        lib = _lib.load()
        if _is_torch_cuda(rays):
            import torch
            r = rays.contiguous()
            n = r.shape[0]
            if out is None:
                out = torch.empty((n,), dtype=torch.uint8, device=r.device)
            stream = torch.cuda.current_stream(r.device).cuda_stream
            _check(self.ctx.handle, lib.vt_trace_any(self.ctx.handle, self._p, r.data_ptr(), n,
                                                     out.data_ptr(), stream), "vt_trace_any")
            return out
        r = as_rays(rays)
        occ = np.empty(r.shape[0], np.uint8) if out is None else out
        _check(self.ctx.handle, lib.vt_trace_any_host(self.ctx.handle, self._p, r.ctypes.data, r.shape[0],
                                                      occ.ctypes.data), "vt_trace_any_host")
        return occ

    def count(self, rays, closest: bool = True) -> tuple[int, int]:
        """(wide nodes fetched, triangles tested) summed over CUDA rays (instrumented kernel)."""
        import torch
        if not _is_torch_cuda(rays):
            rays = torch.from_numpy(as_rays(rays).view(np.float32).reshape(-1, 8)).cuda()
        r = rays.contiguous()
        torch.cuda.current_stream().synchronize()
        a, b = C.c_uint64(), C.c_uint64()
        _check(self.ctx.handle, _lib.load().vt_trace_count(self.ctx.handle, self._p, r.data_ptr(), r.shape[0],
                                                           1 if closest else 0, C.byref(a), C.byref(b)),
               "vt_trace_count")
        return int(a.value), int(b.value)

    def close(self) -> None:
        if getattr(self, "_p", None) is not None and self.ctx._p is not None:
            _lib.load().vt_mesh_destroy(self.ctx.handle, self._p)
        self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def instances_array(transforms, meshes, slot_bases=None) -> np.ndarray:
    """INSTANCE_DTYPE records from (n, 3, 4) object-to-world transforms and per-instance mesh indices."""
    t = np.asarray(transforms, np.float32).reshape(-1, 12)
    out = np.zeros(t.shape[0], INSTANCE_DTYPE)
    out["world"] = t
    out["mesh"] = np.asarray(meshes, np.uint32)
    if slot_bases is not None:
        out["slot_base"] = np.asarray(slot_bases, np.uint32)
    return out


class Tlas:
    """The two-level hierarchy over instances of meshes (vt_tlas): MeshSceneLayout.sceneBlob's TLAS
    (Sources/Acceleration.swift:519-573) traversed like mesh_closest / mesh_occluded
    (main.swift:1840-1984). The meshes must stay open while the TLAS is in use."""

    def __init__(self, ctx: Context, meshes, instances):
        lib = _lib.load()
        self.ctx = ctx
        self.meshes = list(meshes)
        inst = np.ascontiguousarray(instances, INSTANCE_DTYPE)
        handles = (C.c_void_p * len(self.meshes))(*[m._p.value for m in self.meshes])
        p = C.c_void_p()
        _check(ctx.handle, lib.vt_tlas_build(ctx.handle, handles, len(self.meshes), inst.ctypes.data, inst.shape[0],
                                             C.byref(p)), "vt_tlas_build")
        self._p = p

    def info(self) -> TlasInfo:
        out = TlasInfo()
        _check(self.ctx.handle, _lib.load().vt_tlas_get_info(self.ctx.handle, self._p, C.byref(out)), "vt_tlas_get_info")
        return out

    def nodes(self) -> np.ndarray:
        n = self.info().nodes
        out = np.empty(n, WIDE_NODE_DTYPE)
        _check(self.ctx.handle, _lib.load().vt_tlas_get_nodes(self.ctx.handle, self._p, out.ctypes.data, n),
               "vt_tlas_get_nodes")
        return out

    def records(self) -> np.ndarray:
        n = self.info().instances
        out = np.empty(n, INSTANCE_RECORD_DTYPE)
        _check(self.ctx.handle, _lib.load().vt_tlas_get_instances(self.ctx.handle, self._p, out.ctypes.data, n),
               "vt_tlas_get_instances")
        return out

    def _device_rays(self, rays):
        import torch
        if _is_torch_cuda(rays):
            return rays.contiguous(), False
        r = as_rays(rays).view(np.float32).reshape(-1, 8)
        return torch.from_numpy(np.ascontiguousarray(r)).cuda(self.ctx.device), True

    def closest(self, rays):
        """(hits, instances): numpy rays -> numpy HIT_DTYPE and uint32; CUDA tensor (n, 8) -> CUDA
        tensors (n, 4) float32 (t, b1, b2, face bits) and (n,) int32 (instance, -1 on a miss)."""
        import torch
        r, host = self._device_rays(rays)
        n = r.shape[0]
        hits = torch.empty((n, 4), dtype=torch.float32, device=r.device)
        inst = torch.empty((n,), dtype=torch.int32, device=r.device)
        stream = torch.cuda.current_stream(r.device).cuda_stream
        _check(self.ctx.handle, _lib.load().vt_tlas_trace_closest(self.ctx.handle, self._p, r.data_ptr(), n, hits.data_ptr(),
                                                                  inst.data_ptr(), stream), "vt_tlas_trace_closest")
        if host:
            return hits.cpu().numpy().view(HIT_DTYPE).reshape(-1), inst.cpu().numpy().view(np.uint32)
        return hits, inst

    def occluded(self, rays):
        """Any hit in [tmin, tmax): uint8 per ray (numpy for numpy rays, else a CUDA tensor)."""
        import torch
        r, host = self._device_rays(rays)
        n = r.shape[0]
        occ = torch.empty((n,), dtype=torch.uint8, device=r.device)
        stream = torch.cuda.current_stream(r.device).cuda_stream
        _check(self.ctx.handle, _lib.load().vt_tlas_trace_any(self.ctx.handle, self._p, r.data_ptr(), n, occ.data_ptr(),
                                                              stream), "vt_tlas_trace_any")
        return occ.cpu().numpy() if host else occ

    def flatten(self, *, leaf_size: int = 2, treelet_size: int = 7, refine_rounds: int = 2, max_depth: int = 31) -> Mesh:
        """One world-space Mesh of all instances' triangles (rendered face = rendered_base + face)."""
        opts = BuildOptions(leaf_size, treelet_size, refine_rounds, max_depth)
        p = C.c_void_p()
        _check(self.ctx.handle, _lib.load().vt_tlas_flatten(self.ctx.handle, self._p, C.byref(opts), C.byref(p)),
               "vt_tlas_flatten")
        return Mesh._adopt(self.ctx, p)

    def close(self) -> None:
        if getattr(self, "_p", None) is not None and self.ctx._p is not None:
            _lib.load().vt_tlas_destroy(self.ctx.handle, self._p)
        self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
