"""Pin the CPU oracle against the reference's own LBVH goldens.

Goldens: ``tests/golden/lbvh_unit_test.json``, extracted from
Solver/CollisionDetector/lbvh.cpp (LBVH::unit_test 920-984, expected Karras output in
the fn_build_inner_nodes comments 566-597) by ``tests/golden/make_lbvh_goldens.py``.
"""
import json
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(__file__), "golden", "lbvh_unit_test.json")


def _gold():
    with open(GOLD) as f:
        return json.load(f)


def test_morton_goldens(oracle):
    g = _gold()
    for lid in range(8):
        pos = np.float32(lid) / np.float32(10.0)
        assert oracle.morton32((pos, pos, pos)) == g["morton32"][lid]
        assert oracle.morton64((pos, pos, pos), lid) == g["morton64"][lid]


def test_karras_goldens(oracle):
    g = _gold()
    keys = np.array(g["morton64"], dtype=np.uint64)
    n = len(keys)
    for nid in range(1, n - 1):
        assert list(oracle.determine_range(keys, nid)) == g["ranges"][nid]
    # node 0 covers the whole range [0, n-1]
    assert g["ranges"][0] == [0, n - 1]
    for nid in range(n - 1):
        i, j = g["ranges"][nid]
        assert oracle.find_split(keys, i, j) == g["splits"][nid]
    parent, children = oracle.karras(keys)
    assert children[: n - 1].tolist() == g["inner_children"]
    assert parent[1:].tolist() == g["parents"][1:]
    assert parent[0] == 0xFFFFFFFF


def test_refit_complete_tree_root(oracle):
    """test_lbvh_refit.cpp:276-340: leaves i at [i, i+1] on a line, root AABB = [0, N]."""
    n = 64
    x = np.zeros((n + 1, 3), np.float32)
    x[:, 0] = np.arange(n + 1, dtype=np.float32)
    edges = np.stack([np.arange(n), np.arange(1, n + 1)], 1).astype(np.uint32)
    tree = oracle.lbvh_build(oracle.TREE_EDGE, x, edges)
    assert tree.unhealthy == 0
    aabb = oracle.lbvh_refit(tree, x, x, np.zeros(n + 1, np.float32), edges)
    assert aabb[0, 0] == 0.0 and aabb[0, 4] == float(n)
    # every inner node is the exact union of its children
    ni = n - 1
    for nid in range(ni):
        l, r = tree.children[nid]
        assert np.array_equal(aabb[nid, :3], np.minimum(aabb[l, :3], aabb[r, :3]))
        assert np.array_equal(aabb[nid, 4:7], np.maximum(aabb[l, 4:7], aabb[r, 4:7]))


def test_line_intersection_basic(oracle):
    a, b, c = (0, 0, 0), (1, 0, 0), (0, 1, 0)
    hit, bary, t = oracle.line_intersection((0.25, 0.25, -1.0), (0.25, 0.25, 1.0), a, b, c)
    assert hit and abs(t - 0.5) < 1e-6
    assert np.allclose(bary, [0.5, 0.25, 0.25], atol=1e-6)
    hit, _, _ = oracle.line_intersection((2.0, 2.0, -1.0), (2.0, 2.0, 1.0), a, b, c)
    assert not hit
    # parallel segment is rejected
    hit, _, _ = oracle.line_intersection((0.2, 0.2, 0.0), (0.3, 0.3, 0.0), a, b, c)
    assert not hit
