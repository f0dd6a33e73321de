"""The light BVH and the packed emitter list (Sources/LightTree.swift; main.swift:9313-9401).

The library's native builder is compared word for word with the pure-Python restatement
(oracle/light_tree.py), and the tree is checked as tests/Fix_light-tree.swift:5-36 checks it: every
emitter in exactly one leaf, consistent parent/child links, power sums, children's quantised bounds
inside their parent's, the root's power, depth and node count, also with coincident, degenerate and
powerless emitters. The emitter-list cases follow :150-176 (one lamp builds no tree; separate lights
do). These run on the CPU: the builder is host code.
"""
import numpy as np
import pytest

from metal_vibe_tracer_b200 import MaterialLibraryError, lights, scenes
from oracle import light_tree as LT


def random_emitters(seed, n=500, copies=40):
    """tests/Fix_light-tree.swift:8-17 with a seeded generator: n random small triangles, every
    7th powerless, every 5th with emission cosine 0.7, then `copies` of emitter 1 and a degenerate
    one."""
    rng = np.random.default_rng(seed)
    o = np.stack([rng.uniform(-10, 10, n), rng.uniform(-2, 2, n), rng.uniform(-10, 10, n)], 1).astype(np.float32)
    b = (o + rng.uniform(-0.5, 0.5, (n, 3))).astype(np.float32)
    c = (o + rng.uniform(-0.5, 0.5, (n, 3))).astype(np.float32)
    power = np.where(np.arange(n) % 7 == 0, 0.0, rng.uniform(0.1, 10, n))
    cose = np.where(np.arange(n) % 5 == 0, 0.7, 0.0)
    e = lights.make_emitters(o, b, c, power, cose)
    if copies:
        e = np.concatenate([e, np.repeat(e[1:2], copies)])
        e = np.concatenate([e, lights.make_emitters(np.zeros((1, 3)), np.zeros((1, 3)), np.zeros((1, 3)), [3.0])])
    return e


def check_well_formed(tree, emitters):
    w = tree.words
    phi = w[:, 1].view(np.float32).astype(np.float64)
    count = w[:, 7] >> 27
    parent = w[:, 7] & 0x7FFFFFF
    box = np.stack([w[:, 3] & 0xFFFF, w[:, 3] >> 16, w[:, 4] & 0xFFFF, w[:, 4] >> 16, w[:, 5] & 0xFFFF, w[:, 5] >> 16], 1)
    covered = np.zeros(len(emitters), int)
    for i in range(len(w)):
        if count[i]:
            assert count[i] <= lights.MAX_LEAF
            for pos in range(int(w[i, 6]), int(w[i, 6]) + int(count[i])):
                covered[tree.order[pos]] += 1
                assert tree.leaf_node[pos] == i
            continue
        children = [i + 1, int(w[i, 6])]
        for ch in children:
            assert ch < len(w) and parent[ch] == i
        assert abs(phi[i] - phi[children[0]] - phi[children[1]]) <= 1e-5 * max(1.0, phi[i])
        for ch in children:
            if phi[ch] > 0:
                o, n = box[i], box[ch]
                assert all(n[k] >= o[k] for k in range(3)) and all(n[k] <= o[k] for k in range(3, 6))
    assert np.all(covered == 1)
    assert parent[0] == lights.NO_PARENT
    area = np.linalg.norm(np.cross(emitters["b"].astype(np.float64) - emitters["a"], emitters["c"].astype(np.float64) -
                                   emitters["a"]), axis=1)
    root = float(np.sum(np.where((emitters["power"] > 0) & (area > 0), emitters["power"], 0.0)))
    assert abs(phi[0] - root) <= 1e-5 * root
    leaves = int(np.count_nonzero(count))
    assert tree.depth <= 64 and len(w) == 2 * leaves - 1


def assert_same_tree(tree, ref):
    words, order, leaf, depth, glo, ghi = ref
    assert np.array_equal(tree.words, words)
    assert np.array_equal(tree.order, order)
    assert np.array_equal(tree.leaf_node, leaf)
    assert tree.depth == depth
    assert np.array_equal(tree.grid_lo.view(np.uint32), np.asarray(glo, np.float32).view(np.uint32))
    assert np.array_equal(tree.grid_hi.view(np.uint32), np.asarray(ghi, np.float32).view(np.uint32))


@pytest.mark.parametrize("seed", [0, 1, 20260928])
def test_tree_matches_restatement_and_is_well_formed(seed):
    e = random_emitters(seed)
    tree = lights.LightTree.build(e)
    assert_same_tree(tree, LT.build(e))
    check_well_formed(tree, e)


@pytest.mark.parametrize("n,max_leaf,ratio", [(1, 8, 0.75), (2, 8, 0.75), (37, 1, 0.75), (200, 4, 0.5), (300, 31, 1.0)])
def test_tree_parameters(n, max_leaf, ratio):
    e = random_emitters(n + 11, n=n, copies=0)
    tree = lights.LightTree.build(e, max_leaf, ratio)
    assert_same_tree(tree, LT.build(e, max_leaf, ratio))
    if n > 1:
        check_well_formed(tree, e)


def test_empty_and_invalid():
    tree = lights.LightTree.build(lights.make_emitters(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3)), []))
    assert tree.node_count == 0 and len(tree.order) == 0
    e = random_emitters(3, n=10, copies=0)
    with pytest.raises(MaterialLibraryError, match="max_leaf"):
        lights.LightTree.build(e, max_leaf=32)
    with pytest.raises(MaterialLibraryError, match="increasing"):
        lights.emitter_list([3, 2, 5, 6, 7, 8, 9, 10, 11, 12], e)
    assert np.array_equal(lights.emitter_list([], e[:0]), [0, 0])
    zero = e.copy()
    zero["power"] = 0.0
    assert np.array_equal(lights.emitter_list(np.arange(10), zero), [0, 0])


@pytest.mark.parametrize("tree", [True, False])
def test_ceiling_emitter_list(tree):
    faces, verts, mats = scenes.ceiling_lights()
    ids, em = LT.scene_emitters(faces, verts, mats)
    words = lights.emitter_list(ids, em, tree)
    assert np.array_equal(words, LT.emitter_list(ids, em, tree))
    n = int(words[0])
    assert n == len(faces) and np.all(np.diff(words[1:1 + n].astype(np.int64)) > 0)
    if tree:
        assert words[2 * n + 2] > 0 and len(np.unique(words[1 + n:1 + 2 * n])) == n
        assert words[2 * n + 3] % 4 == 0
    else:
        cdf = words[1 + n:1 + 2 * n].view(np.float32)
        assert words[2 * n + 2] == 0 and cdf[-1] == 1.0 and np.all(np.diff(cdf) >= 0)


def test_one_lamp_builds_no_tree_and_eight_lights_do():
    faces, verts, mats = scenes.lamp()
    words = lights.emitter_list(*LT.scene_emitters(faces, verts, mats), True)
    assert int(words[0]) == 6 and words[2 * 6 + 2] == 0
    faces, verts, mats = scenes.ceiling_lights()
    ids, em = LT.scene_emitters(faces, verts, mats)
    eight = lights.emitter_list(ids[:8], em[:8], True)
    assert eight[2 * 8 + 2] > 1
    assert np.array_equal(eight, LT.emitter_list(ids[:8], em[:8], True))
