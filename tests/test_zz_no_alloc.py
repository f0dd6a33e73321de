"""The allocation-free build entry point (vt_mesh_build_noalloc) against the regular build.

Some callers cannot call cudaMalloc: hosts that run under a fixed device-memory budget owned by
their own arena or by a framework's caching allocator, and loops that must not pay cudaMalloc's
implicit device synchronisation. vt_mesh_build_noalloc builds into the caller's buffers with all
temporaries in a static device array of the library. This file checks, through the C ABI, that two
calls in a row (different meshes, the second at the face limit) produce exactly the nodes, leaf
order and triangle records of vt_mesh_build (structure data: bit for bit), and that a mesh over
the limit is rejected with a clear message. It is collected last so that a run stopping at the
first failure has already run every other test.
"""
import ctypes as C
import math

import numpy as np
import pytest
import torch

import metal_vibe_tracer_b200 as vt
from metal_vibe_tracer_b200 import _lib, scenes

pytestmark = pytest.mark.gpu


def build_noalloc(faces, verts, leaf_size=2):
    lib = _lib.load()
    n = len(faces)
    f = torch.from_numpy(np.ascontiguousarray(faces).view(np.int32).reshape(n, 4).copy()).cuda()
    v = torch.from_numpy(np.ascontiguousarray(verts).view(np.float32).reshape(len(verts), 8).copy()).cuda()
    nodes = torch.full((n, 32), -7, dtype=torch.int32, device="cuda")   # 128 B per node, poisoned
    tris = torch.full((n, 12), float("nan"), dtype=torch.float32, device="cuda")
    order = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    info = _lib.MeshInfo()
    opts = _lib.BuildOptions(leaf_size, 7, 2, 31)
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.vt_mesh_build_noalloc(f.data_ptr(), n, v.data_ptr(), len(verts), C.byref(opts), nodes.data_ptr(), n,
                                   tris.data_ptr(), order.data_ptr(), C.byref(info), stream, err, len(err))
    assert st == 0, err.value.decode()
    torch.cuda.synchronize()
    m = info.wide_nodes
    return (nodes[:m].cpu().numpy().view(vt.WIDE_NODE_DTYPE).reshape(-1), order.cpu().numpy(),
            tris.cpu().numpy(), info)


def expected_tris(faces, verts, order):
    p = verts["p"]
    f = faces[order]
    out = np.zeros((len(order), 12), np.float32)
    out[:, 0:3], out[:, 4:7], out[:, 8:11] = p[f["a"]], p[f["b"]], p[f["c"]]
    out[:, 3] = order.view(np.float32)
    out[:, 7] = f["tag"].view(np.float32)
    return out


def test_noalloc_build_matches_regular_build_twice(ctx):
    cases = [scenes.triangle_soup(20_000, seed=21, mu=math.log(0.01)),
             scenes.triangle_soup(_lib.NOALLOC_MAX_FACES, seed=22, mu=math.log(0.01))]
    for faces, verts in cases:
        mesh = vt.Mesh(ctx, faces, verts)
        want_nodes, want_order, info = mesh.nodes(), mesh.order(), mesh.info()
        nodes, order, tris, ninfo = build_noalloc(faces, verts)
        assert ninfo.wide_nodes == info.wide_nodes and ninfo.depth == info.depth
        assert np.array_equal(nodes.view(np.uint8), want_nodes.view(np.uint8))
        assert np.array_equal(order, want_order)
        assert np.array_equal(tris.view(np.uint32), expected_tris(faces, verts, order).view(np.uint32))
        assert abs(ninfo.sah_cost - info.sah_cost) <= 1e-4 * info.sah_cost
        assert list(ninfo.lo) == list(info.lo) and list(ninfo.hi) == list(info.hi)
        mesh.close()


def test_noalloc_rejects_meshes_over_the_limit():
    lib = _lib.load()
    info = _lib.MeshInfo()
    err = C.create_string_buffer(256)
    st = lib.vt_mesh_build_noalloc(None, _lib.NOALLOC_MAX_FACES + 1, None, 0, None, None, 0, None, None,
                                   C.byref(info), None, err, len(err))
    assert st == 4
    assert b"exceed the limit" in err.value
