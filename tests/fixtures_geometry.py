"""Test geometry restated from the reference's traversal parity protocol (tests/Fix_accel.swift).

* ``lcg``: the test's 32-bit LCG, seed 20260928 (tests/Fix_accel.swift:200-204).
* ``patch``: the curved N x N height-field patch in [-1, 1]^2 whose quads alternate their diagonal
  (tests/Fix_accel.swift:16-34), welded (shared vertices), so rays at its interior vertices and
  edges probe watertightness.
* ``patch_targets``: interior vertices and the 0.25 / 0.5 / 0.75 points of interior edges, with the
  eyes above the patch that aim at them (tests/Fix_accel.swift:244-262).
* ``lcg_soup`` / ``lcg_rays``: the scattered soup and random rays of the parity section
  (tests/Fix_accel.swift:216-243), identity instance.
"""
from __future__ import annotations

import math

import numpy as np

from metal_vibe_tracer_b200._lib import FACE_DTYPE, VERTEX_DTYPE


class Lcg:
    def __init__(self, seed: int = 20260928):
        self.seed = seed & 0xFFFFFFFF

    def random(self) -> np.float32:
        self.seed = (self.seed * 1664525 + 1013904223) & 0xFFFFFFFF
        return np.float32(self.seed >> 8) / np.float32(1 << 24)

    def vec3(self) -> np.ndarray:
        return np.array([self.random(), self.random(), self.random()], np.float32)

    def unit(self) -> np.ndarray:
        while True:
            v = self.vec3() * np.float32(2) - np.float32(1)
            l2 = float(np.dot(v, v))
            if l2 > 1e-4 and l2 <= 1:
                return (v / np.float32(math.sqrt(l2))).astype(np.float32)


def patch(cells: int):
    """(faces, vertices, grid) of the alternating-diagonal curved patch."""
    grid = np.zeros((cells + 1, cells + 1, 3), np.float32)
    for i in range(cells + 1):
        for j in range(cells + 1):
            x = np.float32(i) / np.float32(cells) * np.float32(2) - np.float32(1)
            z = np.float32(j) / np.float32(cells) * np.float32(2) - np.float32(1)
            y = np.float32(0.15) * np.float32(math.sin(1.7 * float(x) + 0.3)) * np.float32(
                math.cos(1.3 * float(z))) + np.float32(0.05) * x
            grid[i, j] = (x, y, z)
    idx = lambda i, j: i * (cells + 1) + j
    tris = []
    for i in range(cells):
        for j in range(cells):
            a, b, c, d = idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)
            if (i + j) % 2 == 0:
                tris += [(a, b, c), (a, c, d)]
            else:
                tris += [(a, b, d), (b, c, d)]
    faces = np.zeros(len(tris), FACE_DTYPE)
    t = np.array(tris, np.uint32)
    faces["a"], faces["b"], faces["c"] = t[:, 0], t[:, 1], t[:, 2]
    verts = np.zeros((cells + 1) ** 2, VERTEX_DTYPE)
    verts["p"] = grid.reshape(-1, 3)
    return faces, verts, grid


def patch_targets(grid: np.ndarray, every: int = 1) -> np.ndarray:
    """Rays (n, 8) from eyes above the patch at its interior vertices and edge points."""
    cells = grid.shape[0] - 1
    targets = [grid[i, j] for i in range(1, cells) for j in range(1, cells)]
    for i in range(1, cells - 1):
        for j in range(1, cells - 1):
            for f in (0.25, 0.5, 0.75):
                f = np.float32(f)
                targets.append(grid[i, j] + (grid[i + 1, j] - grid[i, j]) * f)
                targets.append(grid[i, j] + (grid[i, j + 1] - grid[i, j]) * f)
    rays = []
    for q, p in enumerate(targets[::every]):
        eye = np.array([0.3 * math.sin(q), 2.5, 0.3 * math.cos(q)], np.float32)
        d = (p - eye).astype(np.float32)
        length = np.float32(math.sqrt(float(np.dot(d, d))))
        d = d / length
        rays.append([*eye, 0.0, *d, length * np.float32(1.001)])
    return np.array(rays, np.float32)


def lcg_soup(count: int = 4000, rng: Lcg | None = None):
    rng = rng or Lcg()
    tris = []
    for _ in range(count):
        c = rng.vec3() * np.float32(2) - np.float32(1)
        e = lambda: rng.vec3() * np.float32(0.2) - np.float32(0.1)
        a, b, d = c + e(), c + e(), c + e()
        if np.linalg.norm(np.cross(b - a, d - a)) > 1e-4:
            tris.append((a, b, d))
    n = len(tris)
    verts = np.zeros(3 * n, VERTEX_DTYPE)
    verts["p"] = np.array(tris, np.float32).reshape(-1, 3)
    faces = np.zeros(n, FACE_DTYPE)
    i = np.arange(n, dtype=np.uint32)
    faces["a"], faces["b"], faces["c"] = 3 * i, 3 * i + 1, 3 * i + 2
    return faces, verts


def lcg_rays(count: int, rng: Lcg) -> np.ndarray:
    out = np.zeros((count, 8), np.float32)
    for k in range(count):
        o = np.array([rng.random() * np.float32(10) - np.float32(5), rng.random() * np.float32(4) - np.float32(1.5),
                      rng.random() * np.float32(8) - np.float32(2.5)], np.float32)
        tmax = np.float32(0.2) + np.float32(6) * rng.random()
        out[k, 0:3] = o
        out[k, 3] = 0.0
        out[k, 4:7] = rng.unit()
        out[k, 7] = tmax
    return out
