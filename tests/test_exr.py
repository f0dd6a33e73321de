"""OpenEXR output (CPU): a round trip of FLOAT RGB through ZIP compression, the header attributes the
reference writes (Sources/StudioRendering.swift:536-610), and the clamp of negative radiance."""
import struct

import numpy as np

from metal_vibe_tracer_b200 import exr


def test_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    img = rng.random((37, 53, 3)) * 1e5  # above half-float range
    img[0, 0] = [-1.0, 2.0, 3.0]
    p = exr.write_exr(tmp_path / "a.exr", img)
    back = exr.read_exr(p)
    ref = np.maximum(img, 0).astype(np.float32)
    assert np.array_equal(back, ref)
    b = p.read_bytes()
    assert b[:4] == b"\x76\x2f\x31\x01" and b[4] == 2
    for name in (b"channels\0chlist", b"compression\0compression\0\x01\0\0\0\x03", b"chromaticities", b"lineOrder",
                 b"dataWindow\0box2i\0\x10\0\0\0" + struct.pack("<iiii", 0, 0, 52, 36)):
        assert name in b


def test_constant_image_compresses(tmp_path):
    img = np.full((64, 64, 3), 0.5)
    p = exr.write_exr(tmp_path / "c.exr", img)
    assert p.stat().st_size < 64 * 64 * 12 // 10
    assert np.array_equal(exr.read_exr(p), img.astype(np.float32))
