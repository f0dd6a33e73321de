"""Test-side restatement of the two-level build's host arithmetic (checker only).

`instance_setup` repeats, in numpy float64, what vt_tlas_build computes per instance (the reference's
MeshLayout.addInstance and sceneBlob, Sources/Acceleration.swift:474-573): the inverse transform, the
infinity norms, reach and condition, and the world box (corners transformed in double, rounded
outward, enlarged by 2^-20 of the instance's reach). `oracle_tlas` builds the oracle's LBVH (leaf size
1) over the same box triangles and rewrites its leaves to name instances, so the GPU's TLAS nodes and
records can be compared with it bit for bit, and the oracle's two-level traversal can run on it.
"""
import numpy as np

from metal_vibe_tracer_b200._lib import FACE_DTYPE, INSTANCE_RECORD_DTYPE, VERTEX_DTYPE


def _norm_inf(m):
    return np.max(np.abs(m[..., 0]) + np.abs(m[..., 1]) + np.abs(m[..., 2]), axis=-1)


def instance_setup(transforms, mesh_of, slots, mesh_faces, mesh_lo, mesh_hi):
    """records (INSTANCE_RECORD_DTYPE), grow, reach, box triangles (faces, vertices)."""
    T = np.asarray(transforms, np.float32).reshape(-1, 3, 4)
    n = T.shape[0]
    m = T[:, :, :3].astype(np.float64)
    tr = T[:, :, 3].astype(np.float64)
    det = (m[:, 0, 0] * (m[:, 1, 1] * m[:, 2, 2] - m[:, 1, 2] * m[:, 2, 1])
           - m[:, 0, 1] * (m[:, 1, 0] * m[:, 2, 2] - m[:, 1, 2] * m[:, 2, 0])
           + m[:, 0, 2] * (m[:, 1, 0] * m[:, 2, 1] - m[:, 1, 1] * m[:, 2, 0]))
    inv = np.empty_like(m)
    inv[:, 0, 0] = (m[:, 1, 1] * m[:, 2, 2] - m[:, 1, 2] * m[:, 2, 1]) / det
    inv[:, 0, 1] = (m[:, 0, 2] * m[:, 2, 1] - m[:, 0, 1] * m[:, 2, 2]) / det
    inv[:, 0, 2] = (m[:, 0, 1] * m[:, 1, 2] - m[:, 0, 2] * m[:, 1, 1]) / det
    inv[:, 1, 0] = (m[:, 1, 2] * m[:, 2, 0] - m[:, 1, 0] * m[:, 2, 2]) / det
    inv[:, 1, 1] = (m[:, 0, 0] * m[:, 2, 2] - m[:, 0, 2] * m[:, 2, 0]) / det
    inv[:, 1, 2] = (m[:, 0, 2] * m[:, 1, 0] - m[:, 0, 0] * m[:, 1, 2]) / det
    inv[:, 2, 0] = (m[:, 1, 0] * m[:, 2, 1] - m[:, 1, 1] * m[:, 2, 0]) / det
    inv[:, 2, 1] = (m[:, 0, 1] * m[:, 2, 0] - m[:, 0, 0] * m[:, 2, 1]) / det
    inv[:, 2, 2] = (m[:, 0, 0] * m[:, 1, 1] - m[:, 0, 1] * m[:, 1, 0]) / det
    lo = np.asarray(mesh_lo, np.float32)[mesh_of]
    hi = np.asarray(mesh_hi, np.float32)[mesh_of]
    root = np.maximum(np.abs(lo), np.abs(hi)).max(axis=1)  # float32
    norm = _norm_inf(m)
    tmax = np.abs(tr).max(axis=1)
    reach_i = tmax + norm * root.astype(np.float64)
    rec = np.zeros(n, INSTANCE_RECORD_DTYPE)
    rec["world"] = T.reshape(n, 12)
    local = np.zeros((n, 3, 4), np.float32)
    local[:, :, :3] = inv.astype(np.float32)
    local[:, :, 3] = (-(inv[:, :, 0] * tr[:, 0:1] + inv[:, :, 1] * tr[:, 1:2] + inv[:, :, 2] * tr[:, 2:3])).astype(np.float32)
    rec["local"] = local.reshape(n, 12)
    rec["mesh"] = mesh_of
    rec["slot_base"] = slots
    counts = np.asarray(mesh_faces, np.uint64)[mesh_of]
    rec["rendered_base"] = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    rec["mirrored"] = (det < 0).astype(np.uint32)
    rec["bound"][:, 0] = tmax.astype(np.float32)
    rec["bound"][:, 1] = norm.astype(np.float32)
    rec["bound"][:, 2] = root
    grow = np.float32(2.0 ** -18 * (1.0 + (norm * _norm_inf(inv)).max()))
    reach = np.float32(reach_i.max())
    blo = np.full((n, 3), np.finfo(np.float32).max, np.float32)
    bhi = np.full((n, 3), -np.finfo(np.float32).max, np.float32)
    for k in range(8):
        p = np.stack([np.where(k & 1, hi[:, 0], lo[:, 0]), np.where(k & 2, hi[:, 1], lo[:, 1]),
                      np.where(k & 4, hi[:, 2], lo[:, 2])], 1).astype(np.float64)
        v = m[:, :, 0] * p[:, 0:1] + m[:, :, 1] * p[:, 1:2] + m[:, :, 2] * p[:, 2:3] + tr
        vf = v.astype(np.float32)
        blo = np.minimum(blo, np.nextafter(vf, np.float32(-np.inf)))
        bhi = np.maximum(bhi, np.nextafter(vf, np.float32(np.inf)))
    margin = (2.0 ** -20 * reach_i).astype(np.float32)[:, None]
    blo = (blo - margin).astype(np.float32)
    bhi = (bhi + margin).astype(np.float32)
    verts = np.zeros(3 * n, VERTEX_DTYPE)
    verts["p"][0::3] = blo
    verts["p"][1::3] = bhi
    verts["p"][2::3] = np.stack([blo[:, 0], bhi[:, 1], blo[:, 2]], 1)
    faces = np.zeros(n, FACE_DTYPE)
    faces["a"], faces["b"], faces["c"] = 3 * np.arange(n), 3 * np.arange(n) + 1, 3 * np.arange(n) + 2
    return rec, float(grow), float(reach), faces, verts


def oracle_tlas(oracle, box_faces, box_verts):
    """The oracle's LBVH (leaf size 1) over the box triangles, leaves renamed to instances."""
    top = oracle.Bvh.lbvh(box_faces, box_verts, leaf_size=1)
    nodes = top.nodes().copy()
    order = top.order()
    leaf = nodes["child"] < 0
    nodes["child"][leaf] = -(order[-nodes["child"][leaf] - 1] + 1)
    return nodes


def flatten_world(meshes, transforms, mesh_of, slots):
    """World-space soup of every instance's triangles in float64 (rendered order; b, c swapped for a
    mirrored instance), as float32 faces/vertices for brute-force checks."""
    T = np.asarray(transforms, np.float64).reshape(-1, 3, 4)
    fs, vs, base = [], [], 0
    for k, mi in enumerate(mesh_of):
        f, v = meshes[mi]
        p = v["p"].astype(np.float64) @ T[k, :, :3].T + T[k, :, 3]
        det = np.linalg.det(T[k, :, :3])
        a, b, c = f["a"], f["b"], f["c"]
        if det < 0:
            b, c = c, b
        tri = np.stack([p[a], p[b], p[c]], 1).reshape(-1, 3)
        vv = np.zeros(len(tri), VERTEX_DTYPE)
        vv["p"] = tri.astype(np.float32)
        ff = np.zeros(len(f), FACE_DTYPE)
        idx = base * 3 + 3 * np.arange(len(f))
        ff["a"], ff["b"], ff["c"] = idx, idx + 1, idx + 2
        ff["tag"] = f["tag"] + slots[k]
        fs.append(ff)
        vs.append(vv)
        base += len(f)
    return np.concatenate(fs), np.concatenate(vs)


def probe_rays(lo, hi, n, seed=0):
    """Rays from points in the (slightly enlarged) bounds toward random directions, and camera-like
    rays from above the grid toward points inside it: (n, 8) float32."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    c, e = (lo + hi) / 2, (hi - lo) / 2 * 1.05
    h = n // 2
    o1 = c + e * rng.uniform(-1, 1, (h, 3))
    d1 = rng.standard_normal((h, 3))
    eye = c + np.array([0.0, 1.5 * e[1] + 2.0, -1.2 * max(e[0], e[2])])
    tgt = c + e * rng.uniform(-1, 1, (n - h, 3)) * np.array([1.0, 0.2, 1.0])
    d2 = tgt - eye
    o = np.concatenate([o1, np.tile(eye, (n - h, 1))])
    d = np.concatenate([d1, d2])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 4:7], r[:, 7] = o, d, np.inf
    return r
