"""CPU restatement of the radiance cache's network (test infrastructure: the checker of nrc.cu's
encoding, inference and gradients; never a product path).

The reference has no radiance cache, so nothing of the reference pins this module: parity is
unpinned against the reference. It restates, in numpy float64, the published algorithms the CUDA
kernels follow (Mueller et al. 2021, neural radiance caching: relative L2 loss with the prediction
held constant in the denominator; Mueller et al. 2022, multiresolution hash encoding: the spatial
hash x ^ 2654435761 y ^ 805459861 z and trilinear corner weights; Mueller et al. 2019, one-blob
encoding), with the same fp16 roundings of the device: encoded inputs, weights, every layer's
output, the loss gradient (times the loss scale, as the device's backward pass carries it) and every
layer's pre-activation gradient are rounded to fp16 (clamped to +-65504); sums are exact (float64)
where the device accumulates in fp32. `exact=True` drops the roundings, for finite-difference checks
of the gradients.

Records are (n, 13) rows in vt_nrc_input's order (position, roughness, direction, normal, diffuse,
specular, wavelength number u); the network has four outputs, and the loss normaliser weighs them
by rgb luminance (rgb caches) or equally (spectral caches: the four hero wavelengths' terms).
"""
from __future__ import annotations

import math

import numpy as np

HIDDEN = 5
OUT_ROWS = 16
OUTPUTS = 4
MLP_PARAMS = HIDDEN * 64 * 64 + OUT_ROWS * 64
GRAD_CLIP = 512.0
LOSS_SCALE = 64.0
PRIMES = (1, 2654435761, 805459861)


class Grid:
    """The hash grid's geometry as vt_nrc_create computes it (float32 box arithmetic, float64
    level growth)."""

    def __init__(self, levels: int, log2_table: int, base: int, finest: int, lo, hi):
        self.levels, self.log_t = levels, log2_table
        lo = np.asarray(lo, np.float32)
        hi = np.asarray(hi, np.float32)
        ext = np.float32(max(float(hi[k] - lo[k]) for k in range(3)))
        ext = np.float32(ext * np.float32(1.02)) if ext > 0 else np.float32(1.0)
        self.lo = (np.float32(0.5) * (lo + hi) - np.float32(0.5) * ext).astype(np.float32)
        self.inv = np.full(3, np.float32(1.0) / ext, np.float32)
        growth = math.exp((math.log(finest) - math.log(base)) / (levels - 1)) if levels > 1 else 1.0
        self.res = [int(math.floor(base * growth ** l + 1e-6)) for l in range(levels)]

    @property
    def entries(self) -> int:
        return 1 << self.log_t

    def position(self, pos: np.ndarray) -> np.ndarray:
        """Normalised positions in [0, 1]^3 (float32 as the device)."""
        return np.clip(np.nan_to_num((pos.astype(np.float32) - self.lo) * self.inv, nan=0.0), 0.0, 1.0).astype(np.float32)

    def corners(self, pos: np.ndarray, level: int):
        """(n, 8) entry indices within the level and (n, 8) trilinear weights (float32 as the device)."""
        q = self.position(pos)
        res = self.res[level]
        x = (q * np.float32(res)).astype(np.float32)
        c = np.minimum(x.astype(np.int64), res - 1)
        f = (x - c.astype(np.float32)).astype(np.float32)
        side = res + 1
        dense = side ** 3 <= self.entries
        idx = np.empty((len(pos), 8), np.int64)
        w = np.empty((len(pos), 8), np.float32)
        for k in range(8):
            d = np.array([k & 1, (k >> 1) & 1, k >> 2])
            g = c + d
            if dense:
                idx[:, k] = g[:, 0] + side * (g[:, 1] + side * g[:, 2])
            else:
                h = (g[:, 0].astype(np.uint64) * np.uint64(PRIMES[0])) ^ (g[:, 1].astype(np.uint64) * np.uint64(PRIMES[1])) \
                    ^ (g[:, 2].astype(np.uint64) * np.uint64(PRIMES[2]))
                idx[:, k] = (h & np.uint64(0xffffffff) & np.uint64(self.entries - 1)).astype(np.int64)
            wk = np.where(d[0], f[:, 0], np.float32(1) - f[:, 0]) * np.where(d[1], f[:, 1], np.float32(1) - f[:, 1])
            w[:, k] = (wk.astype(np.float32) * np.where(d[2], f[:, 2], np.float32(1) - f[:, 2])).astype(np.float32)
        return idx, w


def _h(x, exact: bool):
    if exact:
        return np.asarray(x, np.float64)
    return np.clip(np.asarray(x, np.float64), -65504.0, 65504.0).astype(np.float16).astype(np.float64)


def blob4(s) -> np.ndarray:
    s = np.clip(np.nan_to_num(np.asarray(s, np.float32), nan=0.0), 0.0, 1.0)
    c = (np.arange(4, dtype=np.float32) + np.float32(0.5)) * np.float32(0.25)
    d = (s[:, None] - c[None, :]) * np.float32(4.0)
    return np.exp(np.float32(-0.5) * d * d).astype(np.float64)


def encode(inputs: np.ndarray, table: np.ndarray, grid: Grid, exact: bool = False) -> np.ndarray:
    """(n, 64) encoded rows (fp16 values unless exact). table: (levels, entries, 2)."""
    x = np.asarray(inputs, np.float32)
    n = len(x)
    out = np.zeros((n, 64), np.float64)
    for l in range(grid.levels):
        idx, w = grid.corners(x[:, 0:3], l)
        v = table[l][idx].astype(np.float64)  # (n, 8, 2)
        out[:, 2 * l:2 * l + 2] = np.einsum("nc,ncf->nf", w.astype(np.float64), v)
    out[:, 32:36] = blob4(x[:, 4])
    out[:, 36:40] = blob4(x[:, 5])
    out[:, 40:44] = blob4(x[:, 6])
    out[:, 44:48] = blob4(x[:, 7])
    out[:, 48:52] = blob4(1.0 - np.exp(-np.maximum(x[:, 3], 0.0)))
    out[:, 52:56] = np.clip(np.nan_to_num(x[:, 8:12], nan=0.0), 0.0, 1.0)
    out[:, 56:60] = blob4(x[:, 12])
    out[:, 60:63] = np.sin(2.0 * np.pi * grid.position(x[:, 0:3]).astype(np.float64))
    out[:, 63] = 1.0
    return _h(out, exact)


def split(mlp: np.ndarray):
    m = np.asarray(mlp, np.float64)
    ws = [m[l * 4096:(l + 1) * 4096].reshape(64, 64) for l in range(HIDDEN)]
    wo = m[HIDDEN * 4096:].reshape(OUT_ROWS, 64)
    return ws, wo


def forward(x: np.ndarray, mlp: np.ndarray, exact: bool = False):
    """Layer outputs (fp16 values unless exact) and the (n, 4) prediction."""
    ws, wo = split(mlp)
    ws = [_h(w, exact) for w in ws]
    wo = _h(wo, exact)
    hs = []
    h = x
    for w in ws:
        h = _h(np.maximum(h @ w.T, 0.0), exact)
        hs.append(h)
    return hs, (h @ wo.T)[:, :OUTPUTS]


def predict(inputs, mlp, table, grid: Grid, exact: bool = False) -> np.ndarray:
    return forward(encode(inputs, table, grid, exact), mlp, exact)[1]


def lum_weights(spectral: bool) -> np.ndarray:
    return np.full(4, 0.25) if spectral else np.array([0.2126, 0.7152, 0.0722, 0.0])


def gradients(inputs, targets, mlp, table, grid: Grid, exact: bool = False, spectral: bool = False,
              loss_scale: float = LOSS_SCALE):
    """Gradient sums of the relative L2 loss over the records: (mlp grad (21,504), table grad
    (levels, entries, 2), loss sum). The fp16 roundings see the loss gradient times `loss_scale`, as
    on the device; the sums returned are the loss's own."""
    x = encode(inputs, table, grid, exact)
    ws, wo = split(mlp)
    wsh = [_h(w, exact) for w in ws]
    woh = _h(wo, exact)
    hs, p = forward(x, mlp, exact)
    y = np.asarray(targets, np.float64).reshape(-1, OUTPUTS)
    lum = p @ lum_weights(spectral)
    inv = 1.0 / (lum * lum + 0.01)
    e = p - y
    loss = float(np.sum(np.sum(e * e, 1) * inv))
    d = 2.0 * e * inv[:, None]
    scale = 1.0 if exact else loss_scale
    if not exact:
        d = np.clip(d, -GRAD_CLIP, GRAD_CLIP)
    dout = np.zeros((len(x), OUT_ROWS))
    dout[:, :OUTPUTS] = _h(d * scale, exact)
    g_mlp = np.zeros(MLP_PARAMS)
    g_mlp[HIDDEN * 4096:] = (dout.T @ hs[-1]).ravel()
    dh = dout @ woh
    for l in range(HIDDEN - 1, -1, -1):
        dz = _h(dh * (hs[l] > 0), exact)
        prev = hs[l - 1] if l > 0 else x
        g_mlp[l * 4096:(l + 1) * 4096] = (dz.T @ prev).ravel()
        dh = dz @ wsh[l]
    dfeat = dh[:, :32]
    g_table = np.zeros((grid.levels, grid.entries, 2))
    pos = np.asarray(inputs, np.float32)[:, 0:3]
    for l in range(grid.levels):
        idx, w = grid.corners(pos, l)
        for k in range(8):
            np.add.at(g_table[l], idx[:, k], w[:, k, None].astype(np.float64) * dfeat[:, 2 * l:2 * l + 2])
    return g_mlp / scale, g_table / scale, loss


def loss_sum(inputs, targets, mlp, table, grid: Grid, den=None, spectral: bool = False) -> float:
    """The exact loss (no roundings), for finite differences. `den` holds the per-record
    denominators lum(p)^2 + 0.01 fixed (the stop-gradient the gradient assumes); None computes
    them from this prediction."""
    p = predict(inputs, mlp, table, grid, exact=True)
    y = np.asarray(targets, np.float64).reshape(-1, OUTPUTS)
    if den is None:
        lum = p @ lum_weights(spectral)
        den = lum * lum + 0.01
    return float(np.sum(np.sum((p - y) ** 2, 1) / den))


def denominators(inputs, mlp, table, grid: Grid, spectral: bool = False) -> np.ndarray:
    p = predict(inputs, mlp, table, grid, exact=True)
    lum = p @ lum_weights(spectral)
    return lum * lum + 0.01


def relu_margins(inputs, mlp, table, grid: Grid) -> np.ndarray:
    """Per record the smallest |pre-activation| over the hidden layers. Where it is tiny, an fp16
    rounding of an input (fp32 interpolation on the device, float64 here) may flip a ReLU and with
    it the record's whole gradient; parity checks of gradients keep records with a margin."""
    ws, _ = split(mlp)
    h = encode(inputs, table, grid)
    m = np.full(len(h), np.inf)
    for w in ws:
        z = h @ _h(w, False).T
        m = np.minimum(m, np.abs(z).min(1))
        h = _h(np.maximum(z, 0.0), False)
    return m
