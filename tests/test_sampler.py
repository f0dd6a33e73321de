"""The Z++ sampler (main.swift:122-305, 497-515) against the reference's own checks.

Restates tests/Fix_zsampling.swift:112-300 on the CPU restatement (oracle), then checks the GPU's
draws against it bit for bit:
* O2m3 blocks of 4^m points are (0, 2m, 3)-nets with (0, 2m, 2) pairwise projections, and 2D
  Sobol' blocks of 2^m points (0, m, 2)-nets, unscrambled and Owen-scrambled;
* the quadrant shuffle is a bijection mapping aligned blocks of 4^m indices onto aligned blocks;
* each frame is a Z mask (aligned 2^k x 2^k pixel blocks hold stratified 1D and 2D draws) in the
  per-pixel, TZ and reshuffled models;
* a pixel's draws over 16 / 64 frames of an accumulation are nets of each constituent;
* marginals over many pixels and frames are uniform.
"""
from itertools import product

import numpy as np
import pytest


def splits(total, parts):
    if parts == 1:
        return [[total]]
    return [[a] + rest for a in range(total + 1) for rest in splits(total - a, parts - 1)]


def is_net(points, axes, m):
    """Every elementary box with `bits` leading bits per listed axis (summing to m) holds one point."""
    pts = np.asarray(points, np.uint64)
    for bits in splits(m, len(axes)):
        key = np.zeros(len(pts), np.uint64)
        for axis, b in zip(axes, bits):
            if b:
                key = (key << np.uint64(b)) | (pts[:, axis] >> np.uint64(32 - b))
        if len(np.unique(key)) != len(pts):
            return False
    return True


def fixed(v):
    return (np.asarray(v, np.float64) * 16777216.0).astype(np.uint64) << np.uint64(8)


@pytest.mark.parametrize("seed", [0, 7, 0x5EED])
def test_constituent_nets(oracle, seed):
    o2m3, sobol = oracle.z_sequences(seed, 4096)
    for m in range(2, 11, 2):
        for start in range(0, min(4096, 4 << m), 1 << m):
            block = o2m3[start:start + (1 << m)]
            for axes in ([0, 1, 2], [0, 1], [1, 2], [0, 2], [0], [1], [2]):
                assert is_net(block, axes, m), (seed, m, start, axes)
    for m in range(1, 11):
        for start in range(0, min(4096, 4 << m), 1 << m):
            assert is_net(sobol[start:start + (1 << m)], [0, 1], m), (seed, m, start)


@pytest.mark.parametrize("base,dimension", [(0, 1), (4096 * 777, 12345), (0xFFFFF000, 3)])
def test_quadrant_shuffle_maps_aligned_blocks(oracle, base, dimension):
    v = oracle.z_shuffles(base, dimension, 4096).astype(np.uint64)
    assert len(np.unique(v)) == 4096
    for m in range(1, 7):
        for start in range(0, 4096, 1 << (2 * m)):
            block = v[start:start + (1 << (2 * m))]
            assert len(np.unique(block >> np.uint64(2 * m))) == 1
            assert len(np.unique(block & np.uint64((1 << (2 * m)) - 1))) == 1 << (2 * m)


@pytest.mark.parametrize("model", [0, 1, 3])
def test_frames_are_z_masks(oracle, model):
    side = 32
    one = oracle.sampler_frame(side, side, True, model, 1234, 1, 3, 1)   # event (vertex 3, NEE)
    for k in (1, 2, 3):
        n = 1 << k
        for by, bx in product(range(0, side, n), range(0, side, n)):
            block = one[by:by + n, bx:bx + n].reshape(-1, 6)
            assert is_net(fixed(block[:, :1]), [0], 2 * k)
            assert is_net(fixed(block[:, 1:3]), [0, 1], 2 * k)


@pytest.mark.parametrize("model", [0, 1, 2, 3])
def test_pixel_draws_over_frames_are_nets(oracle, model):
    side = 32
    frames = [oracle.sampler_frame(side, side, True, model, 5000 + j, j + 1, 3, 1).reshape(-1, 6) for j in range(64)]
    for pixel in range(0, side * side, 37):
        a = fixed([[f[pixel, 0]] for f in frames[:16]])
        b = fixed([[f[pixel, 1], f[pixel, 2]] for f in frames[:16]])
        c = fixed([[f[pixel, 3], f[pixel, 4], f[pixel, 5]] for f in frames])
        assert is_net(a, [0], 4) and is_net(b, [0, 1], 4) and is_net(c, [0, 1, 2], 6)


def test_uniform_marginals(oracle):
    total, count = np.zeros(3), 0
    for f in range(16):
        three = oracle.sampler_frame(32, 32, True, 0, 90000 + 13 * f, 1, 3, 1).reshape(-1, 6)[:, 3:]
        total += three.sum(0)
        count += len(three)
    assert np.all(np.abs(total / count - 0.5) < 0.005)


def test_pcg_mode_is_the_pcg_stream(oracle):
    draws = oracle.sampler_frame(8, 4, False, 0, 17, 1, 0, 0)
    for y, x in product(range(4), range(8)):
        s = (y * 8 + x) ^ ((17 * 1999999973) & 0xFFFFFFFF)
        want = []
        for _ in range(6):
            v, s = oracle.rand_f(s)
            want.append(v)
        assert np.array_equal(draws[y, x], np.array(want, np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("z,model", [(False, 0), (True, 0), (True, 1), (True, 2), (True, 3)])
def test_gpu_draws_equal_oracle(ctx, oracle, z, model):
    from metal_vibe_tracer_b200.render import sampler_frame
    for sample, frame, vertex, stream in ((1234, 1, 3, 1), (5003, 4, 1, 0), (77, 20000, 2, 2)):
        gpu = sampler_frame(ctx, 64, 48, z, model, sample, frame, vertex, stream)
        ref = oracle.sampler_frame(64, 48, z, model, sample, frame, vertex, stream)
        assert np.array_equal(gpu.view(np.uint32), ref.view(np.uint32))
