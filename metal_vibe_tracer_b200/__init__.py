"""B200-native rendering hot path of Metal Vibe Tracer: LBVH build, watertight traversal and the
spectral MIS path tracer.

The kernels live in libvt_b200.so (C ABI: include/vt.h); this package is the host side that
mirrors the reference's acceleration-structure interface. Nothing here computes a result on the
CPU: a missing library raises.
"""
from ._lib import (FACE_DTYPE, HIT_DTYPE, RAY_DTYPE, VERTEX_DTYPE, WIDE_NODE_DTYPE, LIB_PATH,
                   exported_symbols, load)
from .accel import Context, MaterialLibraryError, Mesh, Tlas, WideBVHResult, instances_array
from .render import FrameParams, Scene, make_params

__all__ = [
    "Context", "Mesh", "Tlas", "instances_array", "MaterialLibraryError", "WideBVHResult", "Scene", "FrameParams", "make_params", "FACE_DTYPE", "VERTEX_DTYPE",
    "RAY_DTYPE", "HIT_DTYPE", "WIDE_NODE_DTYPE", "LIB_PATH", "exported_symbols", "load",
]
