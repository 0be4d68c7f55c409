"""The oracle's LBVH broad phase and EF narrow phase agree with brute force.

Pins the oracle's traversal (stack 32, strict overlap) against an all-pairs AABB check
and its EF test against all (edge, face) pairs, on scenes where no stack overflows.
"""
import numpy as np
import pytest

from untangling26_b200 import synthetic


def _edge_face_brute(mesh, d_hat, thickness, node_boxes_leaf):
    # all (eid, fid) with strict overlap of the query box and the leaf box
    x = mesh.x
    e = mesh.edges
    qmn = np.minimum(x[e[:, 0]], x[e[:, 1]]) - (thickness + d_hat)
    qmx = np.maximum(x[e[:, 0]], x[e[:, 1]]) + (thickness + d_hat)
    lmn, lmx = node_boxes_leaf
    pairs = []
    for i in range(len(e)):
        ok = np.all(lmn < qmx[i], 1) & np.all(lmx > qmn[i], 1)
        for f in np.nonzero(ok)[0]:
            pairs.append((i, f))
    return np.array(pairs, np.uint32).reshape(-1, 2)


def _leaf_boxes(tree, n):
    ni = n - 1
    boxes = tree.node_aabb[ni:ni + n]
    inv = np.empty(n, np.int64)
    inv[tree.sorted_get_original[:n]] = np.arange(n)
    b = boxes[inv]
    return b[:, :3], b[:, 4:7]


def _sorted(p):
    p = np.asarray(p).reshape(-1, 2)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


@pytest.mark.parametrize("seed", [0, 5])
def test_broad_phase_matches_brute_force(oracle, seed):
    m = synthetic.two_sheets(12, seed=seed)
    d_hat = np.full(m.num_verts, 1e-3, np.float32)
    th = np.zeros(m.num_verts, np.float32)
    tree = oracle.lbvh_build(oracle.TREE_FACE, m.x, m.faces)
    assert tree.unhealthy == 0
    oracle.lbvh_refit(tree, m.x, m.x, th, m.faces)
    pairs, total, overflow = oracle.lbvh_query(tree, oracle.QUERY_EDGES_UNCULLED, m.x, m.x, m.edges, d_hat, th)
    assert overflow == 0
    brute = _edge_face_brute(m, np.float32(1e-3), np.float32(0), _leaf_boxes(tree, m.num_faces))
    assert np.array_equal(_sorted(pairs), _sorted(brute))


def test_ef_narrow_matches_all_pairs(oracle):
    m = synthetic.two_sheets(12, seed=2)
    d_hat = np.full(m.num_verts, 1e-3, np.float32)
    ne, nf = m.num_edges, m.num_faces
    allp = np.stack(np.meshgrid(np.arange(ne), np.arange(nf), indexing="ij"), -1).reshape(-1, 2).astype(np.uint32)
    ef_all, idx_all = oracle.ef_narrow(allp, m.x, m.edges, m.faces, d_hat)
    th = np.zeros(m.num_verts, np.float32)
    tree = oracle.lbvh_build(oracle.TREE_FACE, m.x, m.faces)
    oracle.lbvh_refit(tree, m.x, m.x, th, m.faces)
    broad, _, _ = oracle.lbvh_query(tree, oracle.QUERY_EDGES_UNCULLED, m.x, m.x, m.edges, d_hat, th)
    ef, idx = oracle.ef_narrow(broad, m.x, m.edges, m.faces, d_hat)
    assert len(ef) > 0
    assert np.array_equal(idx, idx_all)
    assert ef.tobytes() == ef_all.tobytes()
    # each EF pair lies on a genuine crossing: edge endpoints on opposite sides of the face plane
    for rec in ef:
        e0, e1, f0, f1, f2 = rec["idx"]
        a, b, c = m.x[f0], m.x[f1], m.x[f2]
        n = np.cross(b - a, c - a)
        assert np.dot(m.x[e0] - a, n) * np.dot(m.x[e1] - a, n) < 0
