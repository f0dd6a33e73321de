"""Oracle: a pure-Python restatement of the reference's light BVH and emitter list.

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may use it, as
the checker; the product builds the tree in libvt_b200.so's native host code.

Follows Sources/LightTree.swift:
* LightTree.Bounds / union (:19-49) and coneUnion / angleBetween (:52-69): pbrt-v4's LightBounds and
  DirectionCone unions, in double precision;
* LightTree.cost (:73-85): the surface area orientation heuristic with the thin-split penalty Kr;
* LightTree.build (:112-160), split (:165-184), bucket (:185-188), partition (:190-198): 12 buckets
  per axis, leaves of up to maxLeaf emitters kept whole when a split saves less than leafRatio, the
  two-pointer partition (Swift's MutableCollection.partition(by:)), the middle for an empty side;
* LightTree.node (:203-214) and octahedral (:216-223): 8 words per node, bounds quantised outward in
  the grid, cosines rounded down;
and the emitter list of main.swift:9313-9345 (power sampling) and lightTreeList (main.swift:9374-9401).

Nodes are numbered in preorder (a node, then its first subtree, then its second), as the reference's
LIFO work list numbers them; this restatement recurses instead. The quaternion rotation of coneUnion is
written out as t = 2 (q.xyz x v), v' = v + q.w t + q.xyz x t.
"""
from __future__ import annotations

import math
import struct

import numpy as np

BUCKETS = 12
MAX_LEAF, LEAF_RATIO = 8, 0.75
MAX_NODES = (1 << 27) - 1
NO_PARENT = MAX_NODES
MAX_DEPTH = 64
INF = math.inf


def _dot(a, b):
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def _scale(a, s):
    return (a[0] * s, a[1] * s, a[2] * s)


def _length(a):
    return math.sqrt(_dot(a, a))


def _normalize(a):
    n = _length(a)
    return (a[0] / n, a[1] / n, a[2] / n)


def _clamp1(c):
    return min(1.0, max(-1.0, c))


def _min3(a, b):
    return tuple(min(x, y) for x, y in zip(a, b))


def _max3(a, b):
    return tuple(max(x, y) for x, y in zip(a, b))


class Bounds:
    __slots__ = ("lo", "hi", "phi", "w", "cos_o", "cos_e")

    def __init__(self):
        self.lo, self.hi = (INF, INF, INF), (-INF, -INF, -INF)
        self.phi, self.w, self.cos_o, self.cos_e = 0.0, (0.0, 0.0, 1.0), 1.0, 1.0

    def copy(self):
        b = Bounds()
        b.lo, b.hi, b.phi, b.w, b.cos_o, b.cos_e = self.lo, self.hi, self.phi, self.w, self.cos_o, self.cos_e
        return b

    def centroid(self):
        return tuple(0.5 * (x + y) for x, y in zip(self.lo, self.hi))


def emitter_bounds(a, b, c, power, cos_emission) -> Bounds:
    """LightTree.Bounds.init(_ e: Emitter)."""
    a, b, c = (tuple(float(x) for x in v) for v in (a, b, c))
    r = Bounds()
    r.lo, r.hi = _min3(a, _min3(b, c)), _max3(a, _max3(b, c))
    n = _cross(_sub(b, a), _sub(c, a))
    length = _length(n)
    r.phi = max(0.0, power) if length > 0 and math.isfinite(power) else 0.0
    r.w = (n[0] / length, n[1] / length, n[2] / length) if length > 0 else (0.0, 0.0, 1.0)
    r.cos_o = 1.0
    r.cos_e = min(1.0, max(0.0, cos_emission))
    return r


def angle_between(a, b):
    if _dot(a, b) < 0:
        return math.pi - 2 * math.asin(min(1.0, _length(_add(a, b)) / 2))
    return 2 * math.asin(min(1.0, _length(_sub(b, a)) / 2))


def _rotate(v, k, angle):
    s, w = math.sin(angle / 2), math.cos(angle / 2)
    q = _scale(k, s)
    t = _scale(_cross(q, v), 2.0)
    return _add(_add(v, _scale(t, w)), _cross(q, t))


def cone_union(wa, ca, wb, cb):
    theta_a, theta_b = math.acos(_clamp1(ca)), math.acos(_clamp1(cb))
    theta_d = angle_between(wa, wb)
    if min(theta_d + theta_b, math.pi) <= theta_a:
        return wa, ca
    if min(theta_d + theta_a, math.pi) <= theta_b:
        return wb, cb
    theta_o = (theta_a + theta_d + theta_b) / 2
    if theta_o >= math.pi:
        return wa, -1.0
    axis = _cross(wa, wb)
    if _dot(axis, axis) == 0:
        return wa, -1.0
    w = _rotate(wa, _normalize(axis), theta_o - theta_a)
    return _normalize(w), math.cos(theta_o)


def union(a: Bounds, o: Bounds) -> Bounds:
    if a.phi == 0:
        return o
    if o.phi == 0:
        return a
    r = Bounds()
    r.lo, r.hi = _min3(a.lo, o.lo), _max3(a.hi, o.hi)
    r.phi = a.phi + o.phi
    r.w, r.cos_o = cone_union(a.w, a.cos_o, o.w, o.cos_o)
    r.cos_e = min(a.cos_e, o.cos_e)
    return r


def cost(b: Bounds, diagonal, axis) -> float:
    if not b.phi > 0:
        return 0.0
    theta_o, theta_e = math.acos(_clamp1(b.cos_o)), math.acos(_clamp1(b.cos_e))
    theta_w = min(theta_o + theta_e, math.pi)
    sin_o = math.sqrt(max(0.0, 1 - b.cos_o * b.cos_o))
    m_omega = 2 * math.pi * (1 - b.cos_o) + math.pi / 2 * (
        2 * theta_w * sin_o - math.cos(theta_o - 2 * theta_w) - 2 * theta_o * sin_o + b.cos_o)
    kr = 1.0 if axis is None else max(max(diagonal[0], diagonal[1]), diagonal[2]) / max(diagonal[axis], 1e-300)
    d = _sub(b.hi, b.lo)
    area = 2 * (d[0] * d[1] + d[0] * d[2] + d[1] * d[2])
    return b.phi * m_omega * kr * area


def _bucket(b: Bounds, axis, cent):
    lo = cent[0][axis]
    extent = cent[1][axis] - lo
    return min(BUCKETS - 1, int(float(BUCKETS) * (b.centroid()[axis] - lo) / extent))


def _split(items, bounds, node: Bounds, cent):
    diagonal = _sub(node.hi, node.lo)
    best = None
    for axis in range(3):
        if not cent[1][axis] > cent[0][axis]:
            continue
        buckets = [Bounds() for _ in range(BUCKETS)]
        for e in items:
            k = _bucket(bounds[e], axis, cent)
            buckets[k] = union(buckets[k], bounds[e])
        below, above = [None] * BUCKETS, [None] * BUCKETS
        for k in range(BUCKETS):
            below[k] = buckets[0] if k == 0 else union(below[k - 1], buckets[k])
        for k in range(BUCKETS - 1, -1, -1):
            above[k] = buckets[k] if k == BUCKETS - 1 else union(above[k + 1], buckets[k])
        for k in range(BUCKETS - 1):
            if not (below[k].phi > 0 or above[k + 1].phi > 0):
                continue
            c = cost(below[k], diagonal, axis) + cost(above[k + 1], diagonal, axis)
            if c < (INF if best is None else best[0]):
                best = (c, axis, k)
    return best


def _partition(order, begin, end, bounds, cent, split):
    middle = begin + (end - begin) // 2
    if split is None:
        return middle
    _, axis, bucket = split

    def second(e):
        return _bucket(bounds[e], axis, cent) > bucket

    lo, hi = begin, end
    while True:
        while True:
            if lo >= hi:
                return middle if lo in (begin, end) else lo
            if second(order[lo]):
                break
            lo += 1
        while True:
            hi -= 1
            if lo >= hi:
                return middle if lo in (begin, end) else lo
            if not second(order[hi]):
                break
        order[lo], order[hi] = order[hi], order[lo]
        lo += 1


def _f32bits(x) -> int:
    return struct.unpack("<I", struct.pack("<f", float(np.float32(x))))[0]


def _round_half_away(x):
    f = math.floor(x)
    return f + (1 if x - f >= 0.5 else 0)


def octahedral(v) -> int:
    s = abs(v[0]) + abs(v[1]) + abs(v[2])
    px, py = v[0] / s, v[1] / s
    if v[2] < 0:
        px, py = (1 - abs(py)) * (1 if px >= 0 else -1), (1 - abs(px)) * (1 if py >= 0 else -1)

    def e(x):
        return int(min(65535, max(0, _round_half_away((x * 0.5 + 0.5) * 65535))))
    return e(px) | e(py) << 16


def _node_words(b: Bounds, grid, child, parent, leaf_count):
    g_lo = [float(x) for x in grid[0]]
    extent = [float(h) - l for h, l in zip(grid[1], g_lo)]

    def q(v, axis, up):
        if not extent[axis] > 0 or not math.isfinite(v):
            return 65535 if up else 0
        x = (v - g_lo[axis]) / extent[axis] * 65535
        return int(min(65535.0, max(0.0, math.ceil(x) if up else math.floor(x))))

    def qcos(c):
        return int(min(65535.0, max(0.0, math.floor((c + 1) / 2 * 65535))))
    lo = [q(b.lo[k], k, False) for k in range(3)]
    hi = [q(b.hi[k], k, True) for k in range(3)]
    return [octahedral(b.w), _f32bits(b.phi), qcos(b.cos_o) | qcos(b.cos_e) << 16, lo[0] | lo[1] << 16,
            lo[2] | hi[0] << 16, hi[1] | hi[2] << 16, child, parent | leaf_count << 27]


def build(emitters, max_leaf=MAX_LEAF, leaf_ratio=LEAF_RATIO):
    """LightTree.build: (words (n, 8) uint32, order int32, leaf_node uint32, depth, grid_lo, grid_hi).

    `emitters` is a structured array with fields a, b, c (float32 x 3), power, cos_emission."""
    count = len(emitters)
    bounds = [emitter_bounds(e["a"], e["b"], e["c"], float(e["power"]), float(e["cos_emission"])) for e in emitters]
    g_lo, g_hi = (INF, INF, INF), (-INF, -INF, -INF)
    for b in bounds:
        g_lo, g_hi = _min3(g_lo, b.lo), _max3(g_hi, b.hi)
    if count:
        grid = (np.nextafter(np.array(g_lo, np.float32), np.float32(-np.inf)),
                np.nextafter(np.array(g_hi, np.float32), np.float32(np.inf)))
    else:
        grid = (np.zeros(3, np.float32), np.zeros(3, np.float32))
    order = list(range(count))
    nodes: list[list[int]] = []
    leaf_node = [0] * count
    depth = 0

    def visit(begin, end, parent, level):
        nonlocal depth
        index = len(nodes)
        nodes.append([])
        depth = max(depth, level)
        total = Bounds()
        c_lo, c_hi = (INF, INF, INF), (-INF, -INF, -INF)
        for i in range(begin, end):
            b = bounds[order[i]]
            total = union(total, b)
            c = b.centroid()
            c_lo, c_hi = _min3(c_lo, c), _max3(c_hi, c)
        if total.phi == 0:
            total = total.copy()
            for i in range(begin, end):
                total.lo, total.hi = _min3(total.lo, bounds[order[i]].lo), _max3(total.hi, bounds[order[i]].hi)
        n = end - begin
        cent = (c_lo, c_hi)
        split = _split(order[begin:end], bounds, total, cent) if n > 1 else None
        leaf = n == 1 or (n <= max_leaf and (total.phi == 0 or
                                             (INF if split is None else split[0]) >=
                                             leaf_ratio * cost(total, _sub(total.hi, total.lo), None)))
        if leaf:
            for i in range(begin, end):
                leaf_node[i] = index
            nodes[index] = _node_words(total, grid, begin, parent, n)
            return index
        mid = _partition(order, begin, end, bounds, cent, split)
        nodes[index] = _node_words(total, grid, 0, parent, 0)
        visit(begin, mid, index, level + 1)
        nodes[index][6] = visit(mid, end, index, level + 1)
        return index

    if count:
        visit(0, count, NO_PARENT, 0)
    return (np.array(nodes, np.uint32).reshape(-1, 8), np.array(order, np.int32), np.array(leaf_node, np.uint32),
            depth, grid[0], grid[1])


def emitter_list(ids, emitters, light_tree=True) -> np.ndarray:
    """The packed emitter list (main.swift:9313-9345, 9374-9401) for emitters sorted by id."""
    count = len(emitters)
    cumulative, total = [], 0.0
    for e in emitters:
        total += float(e["power"])
        cumulative.append(total)
    if not (total > 0 and math.isfinite(total)):
        return np.array([0, 0], np.uint32)
    ids = [int(i) for i in ids]
    if light_tree and count > 1:
        words, order, leaf_node, depth, g_lo, g_hi = build(emitters)
        if len(words) > 1 and depth <= MAX_DEPTH and len(words) < MAX_NODES:
            position = [0] * count
            for leaf, src in enumerate(order):
                position[src] = leaf
            out = [count] + ids + position + [_f32bits(total)]
            node_offset = len(out) + 9
            while node_offset % 4:
                node_offset += 1
            leaf_offset = node_offset + words.size
            out += [len(words), node_offset, leaf_offset]
            out += [_f32bits(x) for x in g_lo] + [_f32bits(x) for x in g_hi]
            out += [0] * (node_offset - len(out))
            out += words.reshape(-1).tolist()
            for leaf, src in enumerate(order):
                out += [ids[src], _f32bits(float(emitters[src]["power"])), int(leaf_node[leaf])]
            return np.array(out, np.uint32)
    cdf = [_f32bits(1.0) if i == count - 1 else _f32bits(cumulative[i] / total) for i in range(count)]
    return np.array([count] + ids + cdf + [_f32bits(total), 0], np.uint32)


def selection_weight(e) -> np.float32:
    """max(1e-8, luminance) of an emission rgb, in float (main.swift:9303-9306)."""
    e = np.asarray(e, np.float32)
    lum = np.float32(np.float32(np.float32(0.2126) * e[0]) + np.float32(np.float32(0.7152) * e[1])) + \
        np.float32(np.float32(0.0722) * e[2])
    return np.float32(max(np.float32(1e-8), np.float32(lum)))


def scene_emitters(faces, verts, materials):
    """(ids, emitters) of a mesh's emissive faces, ids = face indices: power = area (double, from float
    edges) x the slot's float selection weight (main.swift:9318-9323)."""
    from metal_vibe_tracer_b200.lights import make_emitters
    weights = {}
    for slot, m in enumerate(materials):
        e = np.asarray(m["emission"], np.float32)
        if int(m["type"]) == 3 and float(np.dot(e.astype(np.float64), e.astype(np.float64))) > 0:
            weights[slot] = selection_weight(e)
    f = np.asarray(faces)
    p = np.asarray(verts["p"], np.float32)
    ids = [i for i in range(len(f)) if int(f[i]["tag"]) in weights]
    a, b, c = p[f["a"][ids]], p[f["b"][ids]], p[f["c"][ids]]
    power = []
    for i, k in enumerate(ids):
        e1 = (b[i] - a[i]).astype(np.float64)
        e2 = (c[i] - a[i]).astype(np.float64)
        n = _cross(tuple(e1), tuple(e2))
        power.append(0.5 * math.sqrt((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2]) * float(weights[int(f[k]["tag"])]))
    return np.array(ids, np.uint32), make_emitters(a, b, c, power)
