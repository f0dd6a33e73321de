"""Seeded synthetic workloads: the traversal microbenchmark and the integrator's Cornell box.

Triangle soup: ``n`` triangles whose centroids are uniform in the unit cube, with edge lengths
lognormal(mu = ln 0.002, sigma = 0.5) and uniformly random orientations; each triangle is
equilateral with that edge length, rotated by a uniform random rotation about its centroid. FP32
vertices, unwelded (three vertices per face).

Ray sets (32-byte records: origin, tmin, direction, tmax):
  * coherent: one primary ray per pixel of a W x H pinhole camera at (0.5, 0.5, -1.2) looking at
    the cube centre (vertical field of view 45 degrees), tmin 0, tmax inf;
  * incoherent: origins uniform in the cube, directions uniform on the sphere, tmin 0, tmax inf.
Any-hit sets use the same rays with a finite tmax per ray (shadow-ray style): uniform in
[1.0, 2.2] for the camera rays (the cube spans t in about [1.2, 2.4]) and in [0.05, 1.0] for the
incoherent ones.
"""
from __future__ import annotations

import math

import numpy as np

from ._lib import FACE_DTYPE, VERTEX_DTYPE


def triangle_soup(n: int, seed: int = 0, mu: float = math.log(0.002), sigma: float = 0.5):
    """(faces FACE_DTYPE[n], vertices VERTEX_DTYPE[3n]) of the soup described above."""
    rng = np.random.default_rng(seed)
    centre = rng.random((n, 3))
    edge = rng.lognormal(mean=mu, sigma=sigma, size=n)
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    # Rotation matrix rows of unit quaternion (w, x, y, z).
    R = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], axis=1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], axis=1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], axis=1),
    ], axis=1)  # (n, 3, 3)
    radius = edge / math.sqrt(3.0)
    verts = np.empty((n, 3, 3))
    for k in range(3):
        a = 2.0 * math.pi * k / 3.0
        local = np.array([math.cos(a), math.sin(a), 0.0])
        verts[:, k, :] = centre + radius[:, None] * (R @ local)
    v = np.zeros(3 * n, VERTEX_DTYPE)
    v["p"] = verts.reshape(-1, 3).astype(np.float32)
    f = np.zeros(n, FACE_DTYPE)
    idx = np.arange(n, dtype=np.uint32)
    f["a"], f["b"], f["c"] = 3 * idx, 3 * idx + 1, 3 * idx + 2
    return f, v


def _camera_dirs(xs, ys, width, height, fov_deg, lib):
    eye = (0.5, 0.5, -1.2)
    # Looking down +z at the cube centre; right = +x, up = +y.
    th = math.tan(math.radians(fov_deg) * 0.5)
    aspect = width / height
    u = (2.0 * (xs + 0.5) / width - 1.0) * th * aspect
    v = (1.0 - 2.0 * (ys + 0.5) / height) * th
    d = lib.stack([u, v, lib.ones_like(u)], -1) if lib is not np else np.stack([u, v, np.ones_like(u)], -1)
    norm = (d * d).sum(-1, keepdims=True) ** 0.5
    return eye, d / norm


def coherent_rays_np(width: int, height: int, rows: slice | None = None, fov_deg: float = 45.0):
    """Camera rays (n, 8) float32 for the pixel rows in `rows` (all rows by default)."""
    ys_all = np.arange(height, dtype=np.float64)
    if rows is not None:
        ys_all = ys_all[rows]
    ys, xs = np.meshgrid(ys_all, np.arange(width, dtype=np.float64), indexing="ij")
    eye, d = _camera_dirs(xs.reshape(-1), ys.reshape(-1), width, height, fov_deg, np)
    out = np.empty((d.shape[0], 8), np.float32)
    out[:, 0:3] = eye
    out[:, 3] = 0.0
    out[:, 4:7] = d
    out[:, 7] = np.inf
    return out


def incoherent_rays_np(n: int, seed: int = 1):
    rng = np.random.default_rng(seed)
    o = rng.random((n, 3))
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = np.empty((n, 8), np.float32)
    out[:, 0:3] = o
    out[:, 3] = 0.0
    out[:, 4:7] = d
    out[:, 7] = np.inf
    return out


def shadow_tmax_np(rays: np.ndarray, coherent: bool, seed: int = 2) -> np.ndarray:
    """Copy of `rays` with the any-hit tmax distribution of the set."""
    rng = np.random.default_rng(seed)
    out = rays.copy()
    lo, hi = (1.0, 2.2) if coherent else (0.05, 1.0)
    out[:, 7] = (lo + (hi - lo) * rng.random(rays.shape[0])).astype(np.float32)
    return out


def coherent_rays_torch(width: int, height: int, device, fov_deg: float = 45.0):
    import torch
    ys, xs = torch.meshgrid(torch.arange(height, device=device, dtype=torch.float64),
                            torch.arange(width, device=device, dtype=torch.float64), indexing="ij")
    eye, d = _camera_dirs(xs.reshape(-1), ys.reshape(-1), width, height, fov_deg, torch)
    out = torch.empty((d.shape[0], 8), dtype=torch.float32, device=device)
    out[:, 0] = eye[0]
    out[:, 1] = eye[1]
    out[:, 2] = eye[2]
    out[:, 3] = 0.0
    out[:, 4:7] = d.float()
    out[:, 7] = float("inf")
    return out


def camera_rays_torch(camera: dict, width: int, height: int, device):
    """Pinhole rays (n, 8) float32 through the pixel centres of a look-at camera dict (pos, target,
    up, fov in degrees), tmax infinite."""
    import torch
    eye = torch.tensor(camera["pos"], dtype=torch.float64, device=device)
    fwd = torch.tensor(camera["target"], dtype=torch.float64, device=device) - eye
    fwd = fwd / fwd.norm()
    right = torch.linalg.cross(fwd, torch.tensor(camera["up"], dtype=torch.float64, device=device))
    right = right / right.norm()
    up = torch.linalg.cross(right, fwd)
    th = math.tan(math.radians(camera["fov"]) * 0.5)
    ys, xs = torch.meshgrid(torch.arange(height, device=device, dtype=torch.float64),
                            torch.arange(width, device=device, dtype=torch.float64), indexing="ij")
    u = ((2.0 * (xs.reshape(-1) + 0.5) / width - 1.0) * th * width / height)[:, None]
    v = ((1.0 - 2.0 * (ys.reshape(-1) + 0.5) / height) * th)[:, None]
    d = fwd[None, :] + u * right[None, :] + v * up[None, :]
    d = d / d.norm(dim=1, keepdim=True)
    out = torch.empty((d.shape[0], 8), dtype=torch.float32, device=device)
    out[:, 0:3] = eye.float()
    out[:, 3] = 0.0
    out[:, 4:7] = d.float()
    out[:, 7] = float("inf")
    return out


def incoherent_rays_torch(n: int, device, seed: int = 1):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    o = torch.rand((n, 3), generator=g, device=device, dtype=torch.float32)
    d = torch.randn((n, 3), generator=g, device=device, dtype=torch.float32)
    d = d / d.norm(dim=1, keepdim=True)
    out = torch.empty((n, 8), dtype=torch.float32, device=device)
    out[:, 0:3] = o
    out[:, 3] = 0.0
    out[:, 4:7] = d
    out[:, 7] = float("inf")
    return out


def shadow_tmax_torch(rays, coherent: bool, seed: int = 2):
    import torch
    g = torch.Generator(device=rays.device)
    g.manual_seed(seed)
    out = rays.clone()
    lo, hi = (1.0, 2.2) if coherent else (0.05, 1.0)
    out[:, 7] = lo + (hi - lo) * torch.rand((rays.shape[0],), generator=g, device=rays.device)
    return out


# ---- procedural Cornell box (the integrator's workload) ------------------------------------------
def _pcg_hash(v: int) -> int:
    state = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & 0xFFFFFFFF
    return ((word >> 22) ^ word) & 0xFFFFFFFF


def cornell_box(light_radiance: float = 17.0, seed: int = 0):
    """Procedural Cornell box of the reference's scene 1 (main.swift:1421-1438) as triangles.

    Five walls of the cube [-1, 1]^3, open at -z toward the camera (10 triangles), two axis-aligned
    boxes at scene 1's centres and half extents (tall (-0.33, -0.4, 0.35) +- (0.3, 0.6, 0.3), short
    (0.33, -0.7, -0.25) +- (0.3, 0.3, 0.3); 24 triangles), and a 0.25 x 0.25 emitter quad under the
    ceiling at y = 0.999, facing down (2 triangles). Surfaces are grey Lambert: surface s (floor,
    ceiling, back, left, right, tall box, short box) has albedo 0.2 + 0.6 u with u the first PCG
    draw of state (seed * 7 + s) (main.swift:91-101). The emitter has grey radiance
    `light_radiance` (CIE D65 spectrum in spectral transport, luminance = radiance).
    Returns faces, vertices, materials (list of dicts), the quad light (dict) and the camera
    (scene 1's default view, main.swift:10749-10755: yaw 0.45, pitch 0.25, distance 3.4, target
    (0, -0.1, 0), fov 42 degrees).
    """
    quads = [  # corner, u, v (scene 1's walls)
        ((-1, -1, -1), (2, 0, 0), (0, 0, 2)),     # floor
        ((-1, 1, -1), (2, 0, 0), (0, 0, 2)),      # ceiling
        ((1, 1, 1), (-2, 0, 0), (0, -2, 0)),      # back
        ((-1, 1, 1), (0, 0, -2), (0, -2, 0)),     # left
        ((1, 1, -1), (0, 0, 2), (0, -2, 0)),      # right
    ]
    tris, tags = [], []

    def quad(c, u, v, tag):
        c, u, v = np.array(c, float), np.array(u, float), np.array(v, float)
        tris.extend([(c, c + u, c + u + v), (c, c + u + v, c + v)])
        tags.extend([tag, tag])

    for s, (c, u, v) in enumerate(quads):
        quad(c, u, v, s)

    def box(center, half, tag):
        lo, hi = np.array(center) - np.array(half), np.array(center) + np.array(half)
        x0, y0, z0 = lo
        x1, y1, z1 = hi
        quad((x0, y0, z0), (x1 - x0, 0, 0), (0, y1 - y0, 0), tag)   # -z
        quad((x0, y0, z1), (0, y1 - y0, 0), (x1 - x0, 0, 0), tag)   # +z
        quad((x0, y0, z0), (0, y1 - y0, 0), (0, 0, z1 - z0), tag)   # -x
        quad((x1, y0, z0), (0, 0, z1 - z0), (0, y1 - y0, 0), tag)   # +x
        quad((x0, y0, z0), (0, 0, z1 - z0), (x1 - x0, 0, 0), tag)   # -y
        quad((x0, y1, z0), (x1 - x0, 0, 0), (0, 0, z1 - z0), tag)   # +y

    box((-0.33, -0.4, 0.35), (0.3, 0.6, 0.3), 5)
    box((0.33, -0.7, -0.25), (0.3, 0.3, 0.3), 6)
    lc, lsu, lsv = (-0.125, 0.999, -0.125), (0.25, 0, 0), (0, 0, 0.25)
    quad(lc, lsu, lsv, 7)
    n = len(tris)
    verts = np.zeros(3 * n, VERTEX_DTYPE)
    verts["p"] = np.array(tris, np.float64).reshape(-1, 3).astype(np.float32)
    faces = np.zeros(n, FACE_DTYPE)
    i = np.arange(n, dtype=np.uint32)
    faces["a"], faces["b"], faces["c"] = 3 * i, 3 * i + 1, 3 * i + 2
    faces["tag"] = np.array(tags, np.uint32)
    materials = []
    for s in range(7):
        state = _pcg_hash((seed * 7 + s) & 0xFFFFFFFF)
        a = np.float32(0.2) + np.float32(0.6) * (np.float32(state >> 8) * np.float32(1.0 / 16777216.0))
        materials.append({"type": 0, "albedo": (float(a),) * 3, "emission": (0.0, 0.0, 0.0)})
    materials.append({"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (light_radiance,) * 3})
    light = {"corner": lc, "su": lsu, "sv": lsv, "normal": (0, -1, 0), "emission": (light_radiance,) * 3}
    yaw, pitch, dist, target = 0.45, 0.25, 3.4, np.array([0.0, -0.1, 0.0])
    eye = target + dist * np.array([math.cos(pitch) * math.sin(yaw), math.sin(pitch), -math.cos(pitch) * math.cos(yaw)])
    camera = {"pos": tuple(float(x) for x in eye.astype(np.float32)), "target": tuple(float(x) for x in target), "up": (0.0, 1.0, 0.0),
              "fov": 42.0}
    return faces, verts, materials, light, camera


def cornell_coloured(seed: int = 0):
    """The Cornell box with the classic coloured walls and the reference's scene-1 light colour
    (procedural_light_emission, main.swift:711-715: (18, 15, 10)): floor, ceiling and back white
    (0.73), left red (0.63, 0.065, 0.05), right green (0.14, 0.45, 0.091), tall box yellow
    (0.8, 0.6, 0.1), short box blue (0.1, 0.2, 0.7). Saturated colours exercise the spectral uplift
    (refined grid cells) and a coloured emitter the emission basis. Same geometry and camera as
    cornell_box."""
    faces, verts, materials, light, camera = cornell_box(seed=seed)
    palette = [(0.73, 0.73, 0.73), (0.73, 0.73, 0.73), (0.73, 0.73, 0.73), (0.63, 0.065, 0.05), (0.14, 0.45, 0.091),
               (0.8, 0.6, 0.1), (0.1, 0.2, 0.7)]
    for s, c in enumerate(palette):
        materials[s] = {"type": 0, "albedo": c, "emission": (0.0, 0.0, 0.0)}
    e = (18.0, 15.0, 10.0)
    materials[7] = {"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": e}
    light = dict(light, emission=e)
    return faces, verts, materials, light, camera


def cornell_openpbr(seed: int = 0):
    """The coloured Cornell box with OPENPBR slots (material type 4): glossy dielectric walls
    (roughness 0.35, IOR 1.5), a rough gold-coloured metal tall box (roughness 0.3, metalness 1) and a
    half-metallic short box (roughness 0.6, metalness 0.5); floor and ceiling stay Lambert."""
    faces, verts, materials, light, camera = cornell_coloured(seed=seed)
    def pbr(c, rough, metal, ior=1.5):
        return {"type": 4, "albedo": c, "emission": (0.0, 0.0, 0.0), "roughness": rough, "metalness": metal, "ior": ior}
    materials[2] = pbr((0.73, 0.73, 0.73), 0.35, 0.0)
    materials[3] = pbr((0.63, 0.065, 0.05), 0.35, 0.0)
    materials[4] = pbr((0.14, 0.45, 0.091), 0.35, 0.0, 1.4)
    materials[5] = pbr((0.95, 0.75, 0.3), 0.3, 1.0)
    materials[6] = pbr((0.1, 0.2, 0.7), 0.6, 0.5, 1.6)
    return faces, verts, materials, light, camera


def cornell_delta(seed: int = 0, film: bool = False):
    """The coloured Cornell box with ideal glass and mirrors (the reference's DIELECTRIC and GLOSSY
    types): a mirror tall box (GLOSSY, roughness 0, F0 (0.95, 0.9, 0.8); with `film` a 0.45 um film
    of IOR 1.5 on it), a glass short box (DIELECTRIC, IOR 1.5, tint (0.98, 0.95, 0.9)) and a rough
    GLOSSY red wall (roughness 0.3, the OpenPBR metal); the rest stays Lambert. Glass needs a closed
    volume: the boxes are wound outward (their `front` side is the outside), and the glass box stands
    0.02 above the floor, so that no ray leaving it meets the floor and its bottom at the same
    distance."""
    faces, verts, materials, light, camera = cornell_coloured(seed=seed)
    p = verts["p"].astype(np.float64)
    for tag in (5, 6):
        sel = np.nonzero(faces["tag"] == tag)[0]
        centre = p[np.concatenate([faces["a"][sel], faces["b"][sel], faces["c"][sel]])].mean(0)
        for k in sel:
            a, b, c = p[faces["a"][k]], p[faces["b"][k]], p[faces["c"][k]]
            if np.dot(np.cross(b - a, c - a), (a + b + c) / 3.0 - centre) < 0.0:
                faces["b"][k], faces["c"][k] = faces["c"][k], faces["b"][k]
    glass = np.unique(np.concatenate([faces["a"][faces["tag"] == 6], faces["b"][faces["tag"] == 6],
                                      faces["c"][faces["tag"] == 6]]))
    verts["p"][glass, 1] += np.float32(0.02)
    materials[3] = {"type": 1, "albedo": (0.63, 0.065, 0.05), "emission": (0.0, 0.0, 0.0), "roughness": 0.3, "ior": 1.5}
    materials[5] = {"type": 1, "albedo": (0.95, 0.9, 0.8), "emission": (0.0, 0.0, 0.0), "roughness": 0.0, "ior": 1.5}
    if film:
        materials[5].update(thin_film_weight=1.0, thin_film_thickness=0.45, thin_film_ior=1.5)
    materials[6] = {"type": 2, "albedo": (0.98, 0.95, 0.9), "emission": (0.0, 0.0, 0.0), "roughness": 0.0, "ior": 1.5}
    return faces, verts, materials, light, camera


def _mesh_from_triangles(tris, tags):
    n = len(tris)
    verts = np.zeros(3 * n, VERTEX_DTYPE)
    verts["p"] = np.array(tris, np.float64).reshape(-1, 3).astype(np.float32)
    faces = np.zeros(n, FACE_DTYPE)
    i = np.arange(n, dtype=np.uint32)
    faces["a"], faces["b"], faces["c"] = 3 * i, 3 * i + 1, 3 * i + 2
    faces["tag"] = np.array(tags, np.uint32)
    return faces, verts


def ceiling_lights(rows: int = 24, up_row: int = 12):
    """The light-tree check's emitters (tests/Fix_light-tree.swift:38-51): a rows x rows grid of
    0.3-sided right triangles at y = 3 facing down (x = -24 + 2i, z = -24 + 2j; slot 1 where
    (i + j) % 3 == 0, else slot 0) and a row of `up_row` facing up (x = -23 + 4i, z = 0.9, slot 0).
    Slot 0 emits (5, 5, 5), slot 1 (1, 4, 2). Returns faces, vertices, materials."""
    s = 0.3
    tris, tags = [], []

    def emitter(x, z, slot, down):
        a, b, c = (x, 3.0, z), (x + s, 3.0, z), (x, 3.0, z + s)
        tris.append((a, b, c) if down else (a, c, b))
        tags.append(slot)

    for i in range(rows):
        for j in range(rows):
            emitter(-24 + 2 * i, -24 + 2 * j, 1 if (i + j) % 3 == 0 else 0, True)
    for i in range(up_row):
        emitter(-23 + 4 * i, 0.9, 0, False)
    faces, verts = _mesh_from_triangles(tris, tags)
    materials = [{"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (5.0, 5.0, 5.0)},
                 {"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (1.0, 4.0, 2.0)}]
    return faces, verts, materials


def lamp(count: int = 6):
    """One lamp: `count` coincident downward triangles at (1, 3, 1) (tests/Fix_light-tree.swift:170)."""
    s = 0.3
    tris = [((1.0, 3.0, 1.0), (1.0 + s, 3.0, 1.0), (1.0, 3.0, 1.0 + s))] * count
    faces, verts = _mesh_from_triangles(tris, [0] * count)
    return faces, verts, [{"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (5.0, 5.0, 5.0)}]


def cornell_emitters(grid: int = 4, seed: int = 0, lamps: bool = True):
    """The Cornell box lit by emitter triangles (an imported scene): the ceiling light split into a
    grid x grid array of quads (radiance 17) plus, with `lamps`, two small lamps on the back wall
    facing the camera (radiance 6 and 40, each 0.1 x 0.1). All emitters are grey. Returns faces,
    vertices, materials and the camera."""
    faces, verts, materials, light, camera = cornell_box(seed=seed)
    p = verts["p"].reshape(-1, 3, 3).astype(np.float64)
    keep = faces["tag"] != 7
    tris = [tuple(map(tuple, t)) for t in p[keep]]
    tags = list(faces["tag"][keep])

    def quad(c, u, v, tag):
        c, u, v = np.array(c, float), np.array(u, float), np.array(v, float)
        tris.extend([(tuple(c), tuple(c + u), tuple(c + u + v)), (tuple(c), tuple(c + u + v), tuple(c + v))])
        tags.extend([tag, tag])

    step = 0.25 / grid
    for i in range(grid):
        for j in range(grid):
            quad((-0.125 + i * step, 0.999, -0.125 + j * step), (step, 0, 0), (0, 0, step), 7)
    if lamps:
        quad((0.5, 0.2, 0.999), (0, 0.1, 0), (0.1, 0, 0), 8)     # facing -z
        quad((-0.7, -0.3, 0.999), (0, 0.1, 0), (0.1, 0, 0), 9)
    faces, verts = _mesh_from_triangles(tris, tags)
    materials = materials[:7] + [
        {"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (17.0,) * 3},
        {"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (6.0,) * 3},
        {"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (40.0,) * 3}]
    return faces, verts, materials, camera


def icosphere(subdivisions: int = 3, center=(0.0, 0.0, 0.0), radius: float = 1.0, displace: float = 0.0,
              seed: int = 0):
    """A unit icosahedron subdivided `subdivisions` times (each triangle into 4, midpoints pushed to
    the sphere), scaled and moved. With `displace` > 0 each vertex moves along its normal by
    displace * (2 n - 1), n a smooth value noise of the direction (a PCG hash of a 16^3 lattice,
    trilinear). Returns (positions (V, 3), normals (V, 3), triangles (F, 3)); the normals are
    the normalised averages of the incident face normals (smooth shading)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    pts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    for _ in range(subdivisions):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                m = pts[a] + pts[b]
                pts.append(m / np.linalg.norm(m))
                mid[key] = len(pts) - 1
            return mid[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    p = np.array(pts)
    if displace > 0.0:
        lattice = np.array([_pcg_hash((seed * 4099 + i) & 0xFFFFFFFF) for i in range(17 ** 3)], np.float64) / 2.0 ** 32
        g = (p * 0.5 + 0.5) * 16.0
        i0 = np.clip(np.floor(g).astype(int), 0, 15)
        fr = g - i0
        noise = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = (fr[:, 0] if dx else 1 - fr[:, 0]) * (fr[:, 1] if dy else 1 - fr[:, 1]) * (fr[:, 2] if dz else 1 - fr[:, 2])
                    noise += w * lattice[((i0[:, 0] + dx) * 17 + (i0[:, 1] + dy)) * 17 + (i0[:, 2] + dz)]
        p = p * (1.0 + displace * (2.0 * noise - 1.0))[:, None]
    tri = np.array(f, np.int64)
    fn = np.cross(p[tri[:, 1]] - p[tri[:, 0]], p[tri[:, 2]] - p[tri[:, 0]])
    vn = np.zeros_like(p)
    for k in range(3):
        np.add.at(vn, tri[:, k], fn)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    return p * radius + np.asarray(center, float), vn, tri


def cornell_sphere(subdivisions: int = 3, seed: int = 0):
    """The Cornell box (quad light) with a smooth-shaded icosphere (radius 0.3 at (-0.45, -0.7, -0.35),
    the short box's albedo, vertex normals for shading) in front of the boxes. Returns faces,
    vertices, materials, the quad light and the camera."""
    faces, verts, materials, light, camera = cornell_box(seed=seed)
    p, n, tri = icosphere(subdivisions, (-0.45, -0.7, -0.35), 0.3)
    base = len(verts)
    sv = np.zeros(len(p), VERTEX_DTYPE)
    sv["p"] = p.astype(np.float32)
    sv["n"] = n.astype(np.float32)
    sf = np.zeros(len(tri), FACE_DTYPE)
    sf["a"], sf["b"], sf["c"] = tri[:, 0] + base, tri[:, 1] + base, tri[:, 2] + base
    sf["tag"] = 6
    return np.concatenate([faces, sf]), np.concatenate([verts, sv]), materials, light, camera


_UNIT_SPHERES: dict = {}


def _unit_icosphere(subdivisions: int):
    """Cached undisplaced unit icosphere: (positions (V, 3), triangles (F, 3))."""
    if subdivisions not in _UNIT_SPHERES:
        p, _, t = icosphere(subdivisions)
        _UNIT_SPHERES[subdivisions] = (p, t)
    return _UNIT_SPHERES[subdivisions]


def _lattice_noise(dirs, seeds):
    """icosphere's displacement noise for many spheres at once: dirs (V, 3) unit directions, seeds (S,)
    -> (S, V) trilinear value noise of a 17^3 lattice of PCG hashes of (seed * 4099 + node)."""
    idx = np.arange(17 ** 3, dtype=np.uint64)
    h = ((np.asarray(seeds, np.uint64)[:, None] * np.uint64(4099) + idx[None, :]) & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    state = h * np.uint32(747796405) + np.uint32(2891336453)
    word = ((state >> ((state >> np.uint32(28)) + np.uint32(4))) ^ state) * np.uint32(277803737)
    lattice = ((word >> np.uint32(22)) ^ word).astype(np.float64) / 2.0 ** 32
    g = (dirs * 0.5 + 0.5) * 16.0
    i0 = np.clip(np.floor(g).astype(int), 0, 15)
    fr = g - i0
    noise = np.zeros((len(seeds), len(dirs)))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (fr[:, 0] if dx else 1 - fr[:, 0]) * (fr[:, 1] if dy else 1 - fr[:, 1]) * (fr[:, 2] if dz else 1 - fr[:, 2])
                noise += w[None, :] * lattice[:, ((i0[:, 0] + dx) * 17 + (i0[:, 1] + dy)) * 17 + (i0[:, 2] + dz)]
    return noise


def environment_image(width: int = 64, height: int = 32, sun=(0.3, 0.28), sun_radiance: float = 40.0):
    """A synthetic lat-long environment image (height, width, 4) float32, row 0 toward +y: a sky
    gradient from a blue zenith to a bright horizon, a darker ground below it, and a small bright
    "sun" patch of `sun_radiance` around the (u, v) position `sun` (2 x 2 texels), so that the
    compensated sampling table (texels above the mean) differs from the original one."""
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    y = np.cos(np.pi * v)[:, None]                      # +1 at the zenith, -1 at the nadir
    zenith, horizon, ground = np.array([0.15, 0.35, 0.9]), np.array([1.0, 0.85, 0.7]), np.array([0.25, 0.2, 0.15])
    up = np.clip(y, 0.0, 1.0)[..., None]
    sky = horizon * (1 - up ** 0.5) + zenith * up ** 0.5
    img = np.where(y[..., None] >= 0, sky, ground * (1.0 + y[..., None]) + horizon * 0.2 * (-y[..., None] + 1) * 0.2)
    img = img * (1.0 + 0.1 * np.sin(2 * np.pi * u)[None, :, None])
    out = np.ones((height, width, 4), np.float32)
    out[..., :3] = img
    cx, cy = int(sun[0] * width), int(sun[1] * height)
    out[cy:cy + 2, cx:cx + 2, :3] = sun_radiance
    return out


def sky_scene(emitter: bool = True, subdivisions: int = 2):
    """An open scene for the procedural sky and sun (imported-scene lighting): a 10 x 10 ground
    quad, a smooth-shaded icosphere of radius 1 resting on it, a 1 x 1 x 1 box and, with `emitter`,
    a small emissive triangle above them. Returns (faces, vertices, materials, camera)."""
    tris, tags = [], []
    g = 5.0
    tris += [((-g, 0, -g), (g, 0, g), (g, 0, -g)), ((-g, 0, -g), (-g, 0, g), (g, 0, g))]
    tags += [0, 0]
    lo, hi = np.array([1.2, 0.0, -0.3]), np.array([2.2, 1.0, 0.7])
    c = [np.array([hi[0] if i & 1 else lo[0], hi[1] if i & 2 else lo[1], hi[2] if i & 4 else lo[2]]) for i in range(8)]
    for a, b, cc, d in ((0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)):
        tris += [(c[a], c[b], c[cc]), (c[a], c[cc], c[d])]
        tags += [2, 2]
    if emitter:
        tris.append(((-1.5, 2.5, 0.5), (-1.0, 2.5, -0.5), (-0.5, 2.5, 0.5)))  # faces down
        tags.append(3)
    faces, verts = _mesh_from_triangles(tris, tags)
    pos, nrm, ftri = icosphere(subdivisions, center=(-0.3, 1.0, 0.4), radius=1.0)
    base = len(verts)
    sv = np.zeros(len(pos), VERTEX_DTYPE)
    sv["p"] = pos.astype(np.float32)
    sv["n"] = nrm.astype(np.float32)
    sf = np.zeros(len(ftri), FACE_DTYPE)
    sf["a"], sf["b"], sf["c"] = (ftri[:, 0] + base).astype(np.uint32), (ftri[:, 1] + base).astype(np.uint32), \
        (ftri[:, 2] + base).astype(np.uint32)
    sf["tag"] = 1
    faces = np.concatenate([faces, sf])
    verts = np.concatenate([verts, sv])
    materials = [{"type": 0, "albedo": (0.5, 0.5, 0.5), "emission": (0.0, 0.0, 0.0)},
                 {"type": 0, "albedo": (0.7, 0.35, 0.2), "emission": (0.0, 0.0, 0.0)},
                 {"type": 0, "albedo": (0.25, 0.45, 0.7), "emission": (0.0, 0.0, 0.0)},
                 {"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (6.0, 5.0, 4.0)}]
    camera = {"pos": (0.0, 1.6, -5.5), "target": (0.0, 0.8, 0.0), "up": (0.0, 1.0, 0.0), "fov": 50.0}
    return faces, verts, materials, camera


def sphere_grid(triangles: int, seed: int = 0, emissive_every: int = 16, displace: float = 0.05, nmat: int = 8,
                coloured: bool = False):
    """The grid scene's generator (configs C3/C4): a k x k grid of displaced icospheres on a ground quad,
    with k and the subdivision level chosen so that the mesh has about `triangles` triangles (the
    largest subdivision <= 5 whose 20 * 4^s triangles fit four spheres, then k = round(sqrt(T / per))).
    Spheres have radius 0.4 on a unit lattice; each vertex moves along its direction by
    displace * (2 n - 1), n a trilinear value noise of the direction over a 17^3 lattice of PCG hashes
    seeded per sphere; normals are the normalised sums of incident face normals (smooth shading).
    Albedos are grey Lambert 0.2 + 0.6 u from `nmat` slots (with `coloured`, base colours uniform in
    [0, 1]^3 instead); every `emissive_every`-th sphere is an emitter (radiance 4, 8 or 12, grey, in
    slots nmat .. nmat + 2), so the scene is an imported scene lit by its emissive triangles.
    Returns faces, vertices, materials and a camera looking down on the grid."""
    per = 20
    sub = 0
    while sub < 5 and per * 4 * 4 <= max(triangles, 1) / 4:
        per *= 4
        sub += 1
    k = max(1, int(round((triangles / per) ** 0.5)))
    rng = np.random.default_rng(seed)
    unit, tri = _unit_icosphere(sub)
    S, V, F = k * k, len(unit), len(tri)
    sid = np.arange(S)
    centers = np.stack([sid // k - (k - 1) / 2.0, np.full(S, 0.4), sid % k - (k - 1) / 2.0], 1)
    scale = 1.0 + displace * (2.0 * _lattice_noise(unit, seed * 7919 + sid) - 1.0)        # (S, V)
    local = unit[None, :, :] * scale[:, :, None]                                           # (S, V, 3)
    fn = np.cross(local[:, tri[:, 1]] - local[:, tri[:, 0]], local[:, tri[:, 2]] - local[:, tri[:, 0]])
    vn = np.zeros_like(local)
    for c in range(3):
        for ax in range(3):
            vn[:, :, ax] += np.stack([np.bincount(tri[:, c], weights=fn[s, :, ax], minlength=V) for s in range(S)])
    vn /= np.linalg.norm(vn, axis=2, keepdims=True)
    pos = local * 0.4 + centers[:, None, :]
    emissive = (emissive_every > 0) & (sid % max(emissive_every, 1) == emissive_every // 2)
    sphere_tag = np.where(emissive, nmat + sid % 3, sid % nmat).astype(np.uint32)
    half = k / 2.0 + 1.0
    ground = np.array([(-half, 0.0, -half), (half, 0.0, -half), (half, 0.0, half), (-half, 0.0, half)])
    p = np.concatenate([pos.reshape(-1, 3), ground])
    n = np.concatenate([vn.reshape(-1, 3), np.tile([0.0, 1.0, 0.0], (4, 1))])
    t = np.concatenate([(tri[None, :, :] + (sid * V)[:, None, None]).reshape(-1, 3),
                        np.array([[0, 2, 1], [0, 3, 2]]) + S * V])
    tg = np.concatenate([np.repeat(sphere_tag, F), np.zeros(2, np.uint32)])
    verts = np.zeros(len(p), VERTEX_DTYPE)
    verts["p"] = p.astype(np.float32)
    verts["n"] = n.astype(np.float32)
    faces = np.zeros(len(t), FACE_DTYPE)
    faces["a"], faces["b"], faces["c"] = t[:, 0], t[:, 1], t[:, 2]
    faces["tag"] = tg
    if coloured:
        mats = [{"type": 0, "albedo": tuple(float(x) for x in c), "emission": (0.0, 0.0, 0.0)} for c in rng.random((nmat, 3))]
    else:
        mats = [{"type": 0, "albedo": (float(a),) * 3, "emission": (0.0, 0.0, 0.0)} for a in 0.2 + 0.6 * rng.random(nmat)]
    mats += [{"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (float(e),) * 3} for e in (4.0, 8.0, 12.0)]
    d = max(2.0, 0.9 * k)
    camera = {"pos": (0.0, 0.8 * d, -1.2 * d), "target": (0.0, 0.0, 0.0), "up": (0.0, 1.0, 0.0), "fov": 45.0}
    return faces, verts, mats, camera


def production_scene(seed: int = 0, triangles: int = 10_000_000, emitters: int = 100_000, nmat: int = 287):
    """The production-scale grid scene: ~`triangles` triangles of displaced subdivision-5 icospheres
    (20,480 triangles each), ~`emitters` emissive triangles (whole emissive spheres), `nmat` OPENPBR
    slots (base colour uniform in [0, 1]^3, roughness uniform in [0, 1], metalness 1 with
    probability 0.3 else 0, IOR uniform in [1.3, 1.8]; with probability 0.1 a thin film of weight 1,
    thickness uniform in [200, 800] nm and IOR 1.4) and a camera over the grid. Returns faces,
    vertices, materials, camera."""
    spheres = max(1, round(triangles / 20480))
    every = max(1, round(spheres / max(1, round(emitters / 20480))))
    faces, verts, mats, camera = sphere_grid(triangles, seed=seed, emissive_every=every, nmat=nmat, coloured=True)
    rng = np.random.default_rng(seed + 1)
    for i in range(nmat):
        mats[i] = dict(mats[i], type=4, roughness=float(rng.random()), metalness=1.0 if rng.random() < 0.3 else 0.0,
                       ior=float(1.3 + 0.5 * rng.random()))
    _thin_films(mats[:nmat], seed)
    return faces, verts, mats, camera


def _thin_films(mats, seed: int, fraction: float = 0.1):
    """Gives `fraction` of the OPENPBR slots (seeded, own stream) a thin film: weight 1, thickness
    uniform in [0.2, 0.8] micrometres, IOR 1.4 (OpenPBR's default film IOR)."""
    rng = np.random.default_rng(seed + 2)
    for i in range(len(mats)):
        if rng.random() < fraction:
            mats[i].update(thin_film_weight=1.0, thin_film_thickness=float(0.2 + 0.6 * rng.random()), thin_film_ior=1.4)


def displaced_sphere_asset(subdivisions: int, seed: int, displace: float = 0.05):
    """One displaced icosphere in object space (radius 1 before displacement): the grid scenes'
    displacement (sphere_grid) with the noise seeded by `seed`. Returns faces (tag 0) and vertices."""
    unit, tri = _unit_icosphere(subdivisions)
    V = len(unit)
    scale = 1.0 + displace * (2.0 * _lattice_noise(unit, np.array([seed]))[0] - 1.0)
    local = unit * scale[:, None]
    fn = np.cross(local[tri[:, 1]] - local[tri[:, 0]], local[tri[:, 2]] - local[tri[:, 0]])
    vn = np.zeros_like(local)
    for c in range(3):
        for ax in range(3):
            vn[:, ax] += np.bincount(tri[:, c], weights=fn[:, ax], minlength=V)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    verts = np.zeros(V, VERTEX_DTYPE)
    verts["p"] = local.astype(np.float32)
    verts["n"] = vn.astype(np.float32)
    faces = np.zeros(len(tri), FACE_DTYPE)
    faces["a"], faces["b"], faces["c"] = tri[:, 0], tri[:, 1], tri[:, 2]
    return faces, verts


def instanced_grid(grid: int = 32, assets: int = 16, subdivisions: int = 5, seed: int = 0, displace: float = 0.05,
                   nmat: int = 287, emissive_every: int = 10, mirrored_fraction: float = 0.1):
    """The instanced grid scene: a grid x grid lattice of instances of `assets` displaced icospheres
    (subdivision `subdivisions`, per-vertex noise displacement `displace`), each instance turned by a
    random angle about y, scaled by 0.4 u (u uniform in [0.8, 1.2]) and, for `mirrored_fraction` of
    them, mirrored in x; plus a ground quad (its own mesh, one instance). Instance k's faces take slot
    k % nmat (OPENPBR, as production_scene's), every `emissive_every`-th instance an emissive slot
    (radiance 4, 8 or 12). Returns (meshes [(faces, verts)], transforms (n, 3, 4), mesh index per
    instance, slot base per instance, materials, camera)."""
    rng = np.random.default_rng(seed)
    meshes = [displaced_sphere_asset(subdivisions, seed * 7919 + a, displace) for a in range(assets)]
    half = grid / 2.0 + 1.0
    ground = np.zeros(4, VERTEX_DTYPE)
    ground["p"] = np.array([(-half, 0.0, -half), (half, 0.0, -half), (half, 0.0, half), (-half, 0.0, half)], np.float32)
    ground["n"] = (0.0, 1.0, 0.0)
    gf = np.zeros(2, FACE_DTYPE)
    gf["a"], gf["b"], gf["c"] = (0, 0), (2, 3), (1, 2)
    meshes.append((gf, ground))
    n = grid * grid
    k = np.arange(n)
    cx, cz = k // grid - (grid - 1) / 2.0, k % grid - (grid - 1) / 2.0
    theta = rng.uniform(0.0, 2.0 * np.pi, n)
    sc = 0.4 * rng.uniform(0.8, 1.2, n)
    mirror = np.where(rng.random(n) < mirrored_fraction, -1.0, 1.0)
    c, s_ = np.cos(theta), np.sin(theta)
    T = np.zeros((n + 1, 3, 4))
    T[:n, 0, 0], T[:n, 0, 2] = c * sc * mirror, s_ * sc
    T[:n, 1, 1] = sc
    T[:n, 2, 0], T[:n, 2, 2] = -s_ * sc * mirror, c * sc
    T[:n, 0, 3], T[:n, 1, 3], T[:n, 2, 3] = cx, 0.45, cz
    T[n, 0, 0] = T[n, 1, 1] = T[n, 2, 2] = 1.0
    mesh_of = np.concatenate([rng.integers(0, assets, n), [assets]]).astype(np.uint32)
    emissive = (k % max(emissive_every, 1)) == emissive_every // 2
    slots = np.concatenate([np.where(emissive, nmat + k % 3, k % nmat), [0]]).astype(np.uint32)
    mats = [{"type": 4, "albedo": tuple(float(x) for x in rng.random(3)), "emission": (0.0, 0.0, 0.0),
             "roughness": float(rng.random()), "metalness": 1.0 if rng.random() < 0.3 else 0.0,
             "ior": float(1.3 + 0.5 * rng.random())} for _ in range(nmat)]
    _thin_films(mats, seed)
    mats += [{"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": (float(e),) * 3} for e in (4.0, 8.0, 12.0)]
    d = max(2.0, 0.9 * grid)
    camera = {"pos": (0.0, 0.8 * d, -1.2 * d), "target": (0.0, 0.0, 0.0), "up": (0.0, 1.0, 0.0), "fov": 45.0}
    return meshes, T.astype(np.float32), mesh_of, slots, mats, camera


def batch_workload(count: int = 64, seed: int = 0, lo: int = 10_000, hi: int = 2_000_000):
    """Config C4's scene list: per scene (triangles log-uniform in [lo, hi], resolution from
    {256, 512, 1024} squared, spp uniform in 4..64), seeded."""
    rng = np.random.default_rng(seed)
    tri = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(int)
    res = rng.choice([256, 512, 1024], count)
    spp = rng.integers(4, 65, count)
    return [(int(a), int(b), int(c)) for a, b, c in zip(tri, res, spp)]
