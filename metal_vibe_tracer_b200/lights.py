"""Emitter lights on the host: the light BVH and the packed emitter list (host side of include/vt.h).

The roles of the reference's `LightTree.build` (Sources/LightTree.swift:112-160) and of
MaterialLibrary's emitter list (power sampling, main.swift:9313-9345, and `lightTreeList`,
main.swift:9374-9401). Both run in libvt_b200.so's native host code; nothing is computed here, and
no GPU is needed.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .accel import MaterialLibraryError

EMITTER_DTYPE = _lib.EMITTER_DTYPE
MAX_LEAF, LEAF_RATIO = 8, 0.75      # LightTree.maxLeaf, LightTree.leafRatio
NO_PARENT = (1 << 27) - 1           # LightTree.noParent


def _check(st: int, what: str) -> None:
    if st != _lib.VT_OK:
        msg = _lib.load().vt_last_error(None)
        raise MaterialLibraryError(f"{what}: {_lib.STATUS_NAMES.get(st, st)}: {msg.decode() if msg else ''}")


def make_emitters(a, b, c, power, cos_emission=None) -> np.ndarray:
    """Emitter records (vt_emitter) from corner arrays (n, 3), powers (n,) and emission cosines."""
    a = np.asarray(a, np.float32).reshape(-1, 3)
    e = np.zeros(len(a), EMITTER_DTYPE)
    e["a"], e["b"], e["c"] = a, np.asarray(b, np.float32).reshape(-1, 3), np.asarray(c, np.float32).reshape(-1, 3)
    e["power"] = np.asarray(power, np.float64)
    e["cos_emission"] = 0.0 if cos_emission is None else np.asarray(cos_emission, np.float64)
    return e


@dataclass
class LightTree:
    """LightTree.Built: 8 words per node (depth-first), leaf order, leaf nodes, depth and grid."""
    words: np.ndarray       # (node_count, 8) uint32
    order: np.ndarray       # int32, leaf position -> input emitter
    leaf_node: np.ndarray   # uint32, leaf position -> node
    depth: int
    grid_lo: np.ndarray
    grid_hi: np.ndarray

    @property
    def node_count(self) -> int:
        return len(self.words)

    @classmethod
    def build(cls, emitters: np.ndarray, max_leaf: int = MAX_LEAF, leaf_ratio: float = LEAF_RATIO) -> "LightTree":
        lib = _lib.load()
        em = np.ascontiguousarray(emitters, EMITTER_DTYPE)
        p = C.c_void_p()
        _check(lib.vt_light_tree_build(None, em.ctypes.data if len(em) else None, len(em), int(max_leaf),
                                       float(leaf_ratio), C.byref(p)), "vt_light_tree_build")
        try:
            info = _lib.LightTreeInfo()
            _check(lib.vt_light_tree_get_info(None, p, C.byref(info)), "vt_light_tree_get_info")
            words = np.empty(8 * info.node_count, np.uint32)
            _check(lib.vt_light_tree_get_words(None, p, words.ctypes.data, len(words)), "vt_light_tree_get_words")
            order = np.empty(info.count, np.int32)
            leaf = np.empty(info.count, np.uint32)
            _check(lib.vt_light_tree_get_order(None, p, order.ctypes.data, leaf.ctypes.data, info.count),
                   "vt_light_tree_get_order")
        finally:
            lib.vt_light_tree_destroy(None, p)
        return cls(words.reshape(-1, 8), order, leaf, int(info.depth), np.array(info.grid_lo[:], np.float32),
                   np.array(info.grid_hi[:], np.float32))


def emitter_list(ids, emitters: np.ndarray, light_tree: bool = True) -> np.ndarray:
    """The packed emitter list for emitters with strictly increasing ids (uint32 words)."""
    lib = _lib.load()
    ids = np.ascontiguousarray(ids, np.uint32)
    em = np.ascontiguousarray(emitters, EMITTER_DTYPE)
    n = C.c_uint32()
    args = (ids.ctypes.data if len(ids) else None, em.ctypes.data if len(em) else None, len(em), 1 if light_tree else 0)
    _check(lib.vt_emitter_list_pack(None, *args, None, 0, C.byref(n)), "vt_emitter_list_pack")
    out = np.empty(n.value, np.uint32)
    _check(lib.vt_emitter_list_pack(None, *args, out.ctypes.data, n.value, C.byref(n)), "vt_emitter_list_pack")
    return out
