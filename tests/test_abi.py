"""The C-ABI library loads and exports every symbol include/vt.h declares (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "vt.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vt_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = vt.load()
    names = declared_symbols()
    assert len(names) >= 18
    for name in names:
        assert hasattr(lib, name), name
    # The ctypes signature table covers exactly the header's declarations.
    assert sorted(_lib.SIGNATURES) == names


def test_abi_version_and_struct_sizes():
    lib = vt.load()
    assert lib.vt_abi_version() == 1
    assert C.sizeof(_lib.BuildOptions) == 16
    assert C.sizeof(_lib.MeshInfo) == 48
    assert _lib.WIDE_NODE_DTYPE.itemsize == 128


def test_no_context_without_device_or_bad_args():
    lib = vt.load()
    # A null out pointer is rejected before any device work.
    assert lib.vt_ctx_create(0, None) == 1
    assert lib.vt_mesh_get_info(None, None, None) == 1
    assert lib.vt_trace_closest(None, None, None, 0, None, None) == 1


def test_host_side_input_conversion():
    from metal_vibe_tracer_b200.accel import as_faces, as_rays, as_vertices
    f = as_faces(np.array([[0, 1, 2]], np.uint32))
    assert f.dtype == vt.FACE_DTYPE and f["tag"][0] == 0
    v = as_vertices(np.zeros((3, 3), np.float32))
    assert v.dtype == vt.VERTEX_DTYPE and v.shape == (3,)
    r = as_rays(np.zeros((5, 8), np.float32))
    assert r.dtype == vt.RAY_DTYPE and r.shape == (5,)
