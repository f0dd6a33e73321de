"""Wavefront OBJ / MTL input: triangles, vertex normals and UVs, and material slots for the
renderer's scenes (vt_mesh_build + vt_scene_create_imported).

The reference imports OBJ files through `OBJMaterials` (Sources/OBJMaterials.swift): each `mtllib`
material becomes an OpenPBR MaterialX graph. This reader keeps the constant part of that mapping
(Sources/OBJMaterials.swift:4-27) for the material types this renderer has:

* Kd                -> base colour (albedo), clamped to [0, 1];
* Ns                -> specular roughness sqrt(alpha), alpha = sqrt(2 / (Ns + 2)) (Walter et al. 2007);
* Ni                -> specular IOR when > 1 (clamped to [1.01, 2.5]), else 1.5;
* Ks, illum         -> illum 0 and 1, or Ks = 0: no specular lobe (a Lambert slot); illum 3, 5, 8 with
                       max(Ks) above the dielectric's F0(Ni): metalness max(Ks); otherwise an OPENPBR
                       dielectric slot (its specular weight is 1: max(Ks) / F0(Ni) is not supported and is
                       reported when it differs);
* Ke                -> an emissive slot of radiance Ke (emission luminance 1).

Not supported, and reported once each: texture maps (map_*, bump, norm), dissolve / transparency and
the glass illumination models (rendered opaque), and unknown statements. Faces with more than three
vertices are fanned from their first vertex; negative indices count from the end, as OBJ defines.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

from .accel import FACE_DTYPE, VERTEX_DTYPE

DEFAULT = {"type": 0, "albedo": (0.8, 0.8, 0.8), "emission": (0.0, 0.0, 0.0)}


def _floats(tokens, n, line_no, what):
    try:
        vals = [float(x) for x in tokens[:n]]
    except ValueError:
        raise ValueError(f"line {line_no}: bad {what}: {' '.join(tokens)}") from None
    if len(vals) < n:
        raise ValueError(f"line {line_no}: {what} needs {n} numbers")
    return vals


def read_mtl(text: str, report: list) -> dict:
    """MTL statements per material name: kd, ks, ke, ns, ni, d, illum."""
    mats, cur = {}, None
    noted = set()

    def note(s):
        if s not in noted:
            noted.add(s)
            report.append(s)

    for no, raw in enumerate(text.splitlines(), 1):
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        key, *rest = line.split()
        k = key.lower()
        if k == "newmtl":
            cur = " ".join(rest)
            mats[cur] = {"kd": (0.8, 0.8, 0.8), "ks": (0.0, 0.0, 0.0), "ke": (0.0, 0.0, 0.0), "ns": 0.0, "ni": None,
                         "d": 1.0, "illum": 2}
            continue
        if cur is None:
            continue
        m = mats[cur]
        if k in ("kd", "ks", "ke"):
            v = _floats(rest, 1, no, key)
            m[k] = tuple(_floats(rest, 3, no, key)) if len(rest) >= 3 else (v[0],) * 3
        elif k == "ns":
            m["ns"] = _floats(rest, 1, no, key)[0]
        elif k == "ni":
            m["ni"] = _floats(rest, 1, no, key)[0]
        elif k == "d":
            m["d"] = _floats(rest, 1, no, key)[0]
        elif k == "tr":
            m["d"] = 1.0 - _floats(rest, 1, no, key)[0]
        elif k == "illum":
            m["illum"] = int(min(max(_floats(rest, 1, no, key)[0], -1), 99))
        elif k in ("ka", "tf", "sharpness"):
            pass
        elif k.startswith("map_") or k in ("bump", "norm", "disp", "decal"):
            note(f"MTL {key}: texture maps are not supported and were ignored.")
        else:
            note(f"MTL statement {key} is not supported and was ignored.")
    return mats


def _f0(ior: float) -> float:
    return ((ior - 1.0) / (ior + 1.0)) ** 2


def material_slot(name: str, m: dict, report: list) -> dict:
    """The slot dict for one MTL material (the mapping in the module docstring)."""
    if max(m["ke"]) > 0.0:
        return {"type": 3, "albedo": (0.0, 0.0, 0.0), "emission": tuple(float(x) for x in m["ke"]), "name": name}
    kd = tuple(min(1.0, max(0.0, float(x))) for x in m["kd"])
    ior = min(2.5, max(1.01, m["ni"])) if (m["ni"] or 0.0) > 1.0 else 1.5
    if m["illum"] in (4, 6, 7, 9) or m["d"] < 1.0:
        report.append(f"{name}: transparency (illum {m['illum']}, d {m['d']}) is not supported; rendered opaque.")
    ks = max(m["ks"])
    if m["illum"] < 2 or ks <= 0.0:
        return {"type": 0, "albedo": kd, "emission": (0.0, 0.0, 0.0), "name": name}
    alpha = math.sqrt(2.0 / (max(0.0, m["ns"]) + 2.0))
    slot = {"type": 4, "albedo": kd, "emission": (0.0, 0.0, 0.0), "roughness": math.sqrt(alpha), "metalness": 0.0,
            "ior": ior, "name": name}
    if m["illum"] in (3, 5, 8) and ks > _f0(ior):
        slot["metalness"] = min(1.0, ks)
    elif abs(ks / _f0(ior) - 1.0) > 1e-3:
        report.append(f"{name}: specular weight max(Ks) / F0(Ni) = {min(1.0, ks / _f0(ior)):.3g} is not supported; 1 is used.")
    return slot


def load_obj(path, mtl_text: dict | None = None):
    """Read an OBJ file (and the `mtllib` files beside it, or `mtl_text` {name: text}).

    Returns faces (FACE_DTYPE, tag = material slot), vertices (VERTEX_DTYPE: position, normal or
    zero, uv), the slot list (dicts for vt.Scene) and the report of what was ignored."""
    path = Path(path)
    text = path.read_text()
    report: list = []
    pos, nrm, uvs = [], [], []
    keys, index = [], {}
    tris, tags = [], []
    libs: dict = {}
    slot_of, slots = {}, []
    cur_slot = None

    def slot(name):
        if name not in slot_of:
            slot_of[name] = len(slots)
            slots.append(name)
        return slot_of[name]

    def ref(tok, no):
        parts = tok.split("/")
        out = []
        for j, n in enumerate((len(pos), len(uvs), len(nrm))):
            if j >= len(parts) or parts[j] == "":
                out.append(-1)
                continue
            i = int(parts[j])
            i = i - 1 if i > 0 else n + i
            if not 0 <= i < n:
                raise ValueError(f"line {no}: index {parts[j]} out of range")
            out.append(i)
        return tuple(out)

    for no, raw in enumerate(text.splitlines(), 1):
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        key, *rest = line.split()
        if key == "v":
            pos.append(_floats(rest, 3, no, "vertex"))
        elif key == "vn":
            nrm.append(_floats(rest, 3, no, "normal"))
        elif key == "vt":
            uvs.append((_floats(rest, 1, no, "uv") + [0.0])[:2] if len(rest) < 2 else _floats(rest, 2, no, "uv"))
        elif key == "f":
            if len(rest) < 3:
                raise ValueError(f"line {no}: a face needs three vertices")
            if cur_slot is None:
                cur_slot = slot("")
            ids = []
            for tok in rest:
                k = ref(tok, no)
                if k not in index:
                    index[k] = len(keys)
                    keys.append(k)
                ids.append(index[k])
            for j in range(1, len(ids) - 1):
                tris.append((ids[0], ids[j], ids[j + 1]))
                tags.append(cur_slot)
        elif key == "usemtl":
            cur_slot = slot(" ".join(rest))
        elif key == "mtllib":
            for lib in rest:
                if mtl_text is not None and lib in mtl_text:
                    libs.update(read_mtl(mtl_text[lib], report))
                elif (path.parent / lib).exists():
                    libs.update(read_mtl((path.parent / lib).read_text(), report))
                else:
                    report.append(f"mtllib {lib} was not found; its materials use the default.")
        elif key in ("o", "g", "s", "l", "p"):
            pass
        else:
            report.append(f"OBJ statement {key} is not supported and was ignored.")
    verts = np.zeros(len(keys), VERTEX_DTYPE)
    if keys:
        k = np.asarray(keys)
        verts["p"] = np.asarray(pos, np.float32)[k[:, 0]]
        has_n = k[:, 2] >= 0
        if nrm:
            n = np.asarray(nrm, np.float32)[np.maximum(k[:, 2], 0)]
            n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
            verts["n"] = np.where(has_n[:, None], n, 0.0)
        if uvs:
            uv = np.asarray(uvs, np.float32)[np.maximum(k[:, 1], 0)]
            verts["uv"] = np.where((k[:, 1] >= 0)[:, None], uv, 0.0)
    faces = np.zeros(len(tris), FACE_DTYPE)
    if tris:
        t = np.asarray(tris, np.uint32)
        faces["a"], faces["b"], faces["c"] = t[:, 0], t[:, 1], t[:, 2]
        faces["tag"] = np.asarray(tags, np.uint32)
    materials = []
    for name in slots:
        if name in libs:
            materials.append(material_slot(name, libs[name], report))
        else:
            if name:
                report.append(f"material {name} is not defined; the default is used.")
            materials.append(dict(DEFAULT, name=name))
    return faces, verts, materials, report
