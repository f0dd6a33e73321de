"""OpenEXR output of the FP64 accumulation: single-part scanline files with 32-bit FLOAT R, G, B
channels, ZIP compression (16 scanlines per chunk) and Rec. 709 chromaticities, as the reference's
HDR export writes them (OpenEXRFloat, Sources/StudioRendering.swift:536-640; the layout is the
OpenEXR file format's). Radiance is clamped at zero, as the reference does before encoding; float
(not half) keeps radiance above 65,504.

`read_exr` reads back what `write_exr` writes (and uncompressed files of the same layout), for
checks.
"""
from __future__ import annotations

import struct
import zlib
from pathlib import Path

import numpy as np

MAGIC = b"\x76\x2f\x31\x01"
LINES = 16  # ZIP_COMPRESSION's scanlines per chunk


def _attr(name: str, kind: str, value: bytes) -> bytes:
    return name.encode() + b"\0" + kind.encode() + b"\0" + struct.pack("<i", len(value)) + value


def _zip_chunk(raw: bytes) -> bytes:
    """OpenEXR ZIP predictor: even bytes then odd bytes, byte deltas + 128, then zlib; the raw block
    when that does not shrink it."""
    a = np.frombuffer(raw, np.uint8)
    shuffled = np.concatenate([a[0::2], a[1::2]])
    d = shuffled.astype(np.int16)
    d[1:] = (shuffled[1:].astype(np.int16) - shuffled[:-1].astype(np.int16) + 128 + 256) % 256
    packed = zlib.compress(d.astype(np.uint8).tobytes(), 6)
    return packed if len(packed) < len(raw) else raw


def _unzip_chunk(data: bytes, size: int) -> bytes:
    if len(data) == size:
        return data
    d = np.frombuffer(zlib.decompress(data), np.uint8).astype(np.int16)
    out = np.empty_like(d)
    out[0] = d[0]
    out[1:] = d[1:] - 128
    out = np.cumsum(out) % 256
    s = out.astype(np.uint8)
    half = (size + 1) // 2
    raw = np.empty(size, np.uint8)
    raw[0::2] = s[:half]
    raw[1::2] = s[half:]
    return raw.tobytes()


def write_exr(path, rgb) -> Path:
    """Write (height, width, 3) linear sRGB radiance (any float dtype) as a FLOAT RGB OpenEXR."""
    img = np.maximum(np.asarray(rgb, np.float64), 0.0).astype(np.float32)
    if img.ndim != 3 or img.shape[2] != 3 or img.shape[0] < 1 or img.shape[1] < 1:
        raise ValueError("rgb must be (height, width, 3)")
    h, w, _ = img.shape
    chans = b""
    for name in (b"B", b"G", b"R"):  # channel lists are sorted by name
        chans += name + b"\0" + struct.pack("<i", 2) + b"\0\0\0\0" + struct.pack("<ii", 1, 1)
    chans += b"\0"
    window = struct.pack("<iiii", 0, 0, w - 1, h - 1)
    header = MAGIC + struct.pack("<I", 2)
    header += _attr("channels", "chlist", chans)
    header += _attr("chromaticities", "chromaticities", struct.pack("<8f", 0.64, 0.33, 0.30, 0.60, 0.15, 0.06, 0.3127, 0.3290))
    header += _attr("compression", "compression", bytes([3]))
    header += _attr("dataWindow", "box2i", window)
    header += _attr("displayWindow", "box2i", window)
    header += _attr("lineOrder", "lineOrder", bytes([0]))
    header += _attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
    header += _attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
    header += _attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
    header += b"\0"
    chunks = []
    for first in range(0, h, LINES):
        block = img[first:first + LINES]
        # Per scanline the B, G and R planes.
        raw = np.ascontiguousarray(block[:, :, ::-1].transpose(0, 2, 1)).astype("<f4").tobytes()
        packed = _zip_chunk(raw)
        chunks.append(struct.pack("<ii", first, len(packed)) + packed)
    offset = len(header) + 8 * len(chunks)
    table = b""
    for c in chunks:
        table += struct.pack("<Q", offset)
        offset += len(c)
    path = Path(path)
    tmp = path.with_suffix(path.suffix + ".tmp")
    tmp.write_bytes(header + table + b"".join(chunks))
    tmp.replace(path)
    return path


def read_exr(path) -> np.ndarray:
    """(height, width, 3) float32 from a FLOAT B/G/R scanline file (ZIP or no compression)."""
    b = Path(path).read_bytes()
    if b[:4] != MAGIC:
        raise ValueError("not an OpenEXR file")
    pos, attrs = 8, {}
    while b[pos] != 0:
        e = b.index(b"\0", pos)
        name = b[pos:e].decode()
        e2 = b.index(b"\0", e + 1)
        size = struct.unpack_from("<i", b, e2 + 1)[0]
        attrs[name] = b[e2 + 5:e2 + 5 + size]
        pos = e2 + 5 + size
    pos += 1
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    comp = attrs["compression"][0]
    lines = {0: 1, 3: 16}.get(comp)
    if lines is None:
        raise ValueError(f"compression {comp} is not supported")
    nchunks = (h + lines - 1) // lines
    offsets = struct.unpack_from(f"<{nchunks}Q", b, pos)
    img = np.empty((h, w, 3), np.float32)
    for off in offsets:
        first, size = struct.unpack_from("<ii", b, off)
        n = min(lines, h - (first - y0))
        raw = _unzip_chunk(b[off + 8:off + 8 + size], n * w * 12)
        planes = np.frombuffer(raw, "<f4").reshape(n, 3, w)
        img[first - y0:first - y0 + n] = planes.transpose(0, 2, 1)[:, :, ::-1]
    return img
