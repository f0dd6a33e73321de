"""The neural radiance cache (vt_nrc_*, nrc.cu, nrc_tc.cu): a hash-grid encoded MLP trained online on
the suffix radiance of training paths, queried by rendered paths where the spread-angle heuristic
stops them (or at a fixed vertex).

The reference has no radiance cache; the design follows Mueller et al. 2021 ("Real-time Neural
Radiance Caching for Path Tracing") with the multiresolution hash encoding of Mueller et al. 2022.
Queries are (n, 13) float32 rows in vt_nrc_input's order: position xyz, roughness, outgoing
direction (theta / pi, phi / 2 pi + 1/2), shading normal (same), diffuse rgb, specular, the path's
wavelength number u (spectral caches; 0 for rgb). Predictions and training targets are (n, 4): per
hero wavelength its radiance over the illuminant there (spectral caches), or rgb and 0.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .accel import Context, _check

NRC_TRAIN, NRC_RENDER = 1, 2
MLP_PARAMS = 21504
INPUT_FLOATS = 13
OUTPUTS = 4


def default_config() -> dict:
    cfg = _lib.NRCConfig()
    _lib.load().vt_nrc_config_default(C.byref(cfg))
    return {name: getattr(cfg, name) for name, _ in cfg._fields_}


def sphere(d) -> np.ndarray:
    """(theta / pi, phi / 2 pi + 1/2) of unit vectors (n, 3), the cache's direction parametrisation."""
    d = np.asarray(d, np.float64)
    return np.stack([np.arccos(np.clip(d[:, 2], -1.0, 1.0)) / np.pi, np.arctan2(d[:, 1], d[:, 0]) / (2 * np.pi) + 0.5], 1)


class RadianceCache:
    """A vt_nrc over the box [lo, hi]; `config` overrides vt_nrc_config_default's fields."""

    def __init__(self, ctx: Context, lo, hi, **config):
        lib = _lib.load()
        self.ctx = ctx
        cfg = _lib.NRCConfig()
        lib.vt_nrc_config_default(C.byref(cfg))
        for k, v in config.items():
            if not hasattr(cfg, k):
                raise KeyError(f"unknown cache setting {k}")
            setattr(cfg, k, v)
        self.config = {name: getattr(cfg, name) for name, _ in cfg._fields_}
        lo = (C.c_float * 3)(*[float(x) for x in lo])
        hi = (C.c_float * 3)(*[float(x) for x in hi])
        p = C.c_void_p()
        _check(ctx.handle, lib.vt_nrc_create(ctx.handle, C.byref(cfg), lo, hi, C.byref(p)), "vt_nrc_create")
        self._p = p
        self.grid_params = int(self.info()["grid_params"])

    def info(self) -> dict:
        st = _lib.NRCInfo()
        _check(self.ctx.handle, _lib.load().vt_nrc_get_info(self.ctx.handle, self._p, C.byref(st)), "vt_nrc_get_info")
        return {name: getattr(st, name) for name, _ in st._fields_ if name != "pad"}

    def params(self, grid: bool = True) -> tuple[np.ndarray, np.ndarray | None]:
        mlp = np.empty(MLP_PARAMS, np.float32)
        g = np.empty(self.grid_params, np.float32) if grid else None
        _check(self.ctx.handle, _lib.load().vt_nrc_get_params(self.ctx.handle, self._p, mlp.ctypes.data,
                                                              None if g is None else g.ctypes.data), "vt_nrc_get_params")
        return mlp, g

    def set_params(self, mlp, grid=None) -> None:
        mlp = np.ascontiguousarray(mlp, np.float32)
        if mlp.size != MLP_PARAMS:
            raise ValueError(f"mlp needs {MLP_PARAMS} floats")
        g = None
        if grid is not None:
            g = np.ascontiguousarray(grid, np.float32)
            if g.size != self.grid_params:
                raise ValueError(f"grid needs {self.grid_params} floats")
        _check(self.ctx.handle, _lib.load().vt_nrc_set_params(self.ctx.handle, self._p, mlp.ctypes.data,
                                                              None if g is None else g.ctypes.data), "vt_nrc_set_params")

    @staticmethod
    def _rows(inputs) -> np.ndarray:
        x = np.asarray(inputs, np.float32)
        if x.ndim != 2 or x.shape[1] != INPUT_FLOATS:
            raise ValueError("inputs must be (n, 13) float32")
        rows = np.zeros((len(x), 16), np.float32)  # vt_nrc_input: 64 bytes, 3 floats of padding
        rows[:, :INPUT_FLOATS] = x
        return rows

    def infer(self, inputs) -> np.ndarray:
        x = self._rows(inputs)
        out = np.empty((len(x), OUTPUTS), np.float32)
        _check(self.ctx.handle, _lib.load().vt_nrc_infer(self.ctx.handle, self._p, x.ctypes.data, len(x), out.ctypes.data),
               "vt_nrc_infer")
        return out

    def gradients(self, inputs, targets, grid: bool = True):
        """(mlp gradient sums, grid gradient sums or None, loss sum) over the records, no update."""
        x = self._rows(inputs)
        y = np.ascontiguousarray(targets, np.float32).reshape(len(x), OUTPUTS)
        gm = np.empty(MLP_PARAMS, np.float32)
        gg = np.empty(self.grid_params, np.float32) if grid else None
        loss = C.c_double()
        _check(self.ctx.handle, _lib.load().vt_nrc_gradients(self.ctx.handle, self._p, x.ctypes.data, y.ctypes.data,
                                                             len(x), gm.ctypes.data, None if gg is None else gg.ctypes.data,
                                                             C.byref(loss)), "vt_nrc_gradients")
        return gm, gg, float(loss.value)

    def train(self, inputs, targets) -> float:
        """One Adam step; the records' mean loss before it."""
        x = self._rows(inputs)
        y = np.ascontiguousarray(targets, np.float32).reshape(len(x), OUTPUTS)
        loss = C.c_float()
        _check(self.ctx.handle, _lib.load().vt_nrc_train(self.ctx.handle, self._p, x.ctypes.data, y.ctypes.data, len(x),
                                                         C.byref(loss)), "vt_nrc_train")
        return float(loss.value)

    def render(self, scene, params, spp: int, train: bool = True, render: bool = True, stream=None) -> None:
        """One frame through vt_render_nrc: the training paths and step, then spp cached samples."""
        flags = (NRC_TRAIN if train else 0) | (NRC_RENDER if render else 0)
        if render:
            scene.width, scene.height = params.width, params.height
        _check(self.ctx.handle, _lib.load().vt_render_nrc(self.ctx.handle, scene._p, self._p, C.byref(params), int(spp),
                                                          flags, stream), "vt_render_nrc")

    def close(self) -> None:
        if getattr(self, "_p", None) is not None and self.ctx._p is not None:
            _lib.load().vt_nrc_destroy(self.ctx.handle, self._p)
        self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
