"""Topology tables follow the reference's conventions (host-side input preparation)."""
import numpy as np

from untangling26_b200.mesh import Mesh
from untangling26_b200 import synthetic


def _tiny():
    # two triangles sharing edge (1, 2), plus one dangling triangle
    x = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [2, 2, 0], [3, 2, 0], [2, 3, 0]], np.float32)
    f = np.array([[0, 1, 2], [1, 3, 2], [4, 5, 6]], np.uint32)
    return Mesh(x, f)


def test_edges_sorted_unique():
    m = _tiny()
    e = m.edges
    assert (e[:, 0] < e[:, 1]).all()
    keys = e[:, 0].astype(np.int64) * 100 + e[:, 1]
    assert (np.diff(keys) > 0).all()
    assert e.tolist() == [[0, 1], [0, 2], [1, 2], [1, 3], [2, 3], [4, 5], [4, 6], [5, 6]]


def test_face_adj_edges_follow_face_order():
    m = _tiny()
    for fid, face in enumerate(m.faces):
        for j in range(3):
            a, b = sorted((int(face[j]), int(face[(j + 1) % 3])))
            assert m.edges[m.face_adj_edges[fid, j]].tolist() == [a, b]


def test_edge_adjacency_order():
    m = _tiny()
    eid = 2  # edge (1, 2) shared by faces 0 and 1
    assert m.edge_adj_faces_ext.row(eid).tolist() == [0, 1]
    # for each incident face, the two other edges in face_adj_edges order
    exp = []
    for f in (0, 1):
        exp += [e for e in m.face_adj_edges[f].tolist() if e != eid]
    assert m.edge_adj_edges_ext.row(eid).tolist() == exp
    # vertex 1: other endpoints in edge-id order
    assert m.vert_adj_verts.row(1).tolist() == [0, 2, 3]


def test_areas():
    m = _tiny()
    assert np.allclose(m.rest_face_area, [0.5, 0.5, 0.5])
    assert np.isclose(m.rest_vert_area[1], 1.0 / 3.0)
    assert np.isclose(m.rest_edge_area[2], 1.0 / 3.0)


def test_synthetic_shapes():
    m = synthetic.two_sheets(16, seed=3)
    assert m.num_verts == 2 * 256 and m.num_faces == 2 * 2 * 15 * 15
    assert m.num_edges == 2 * (3 * 15 * 15 + 2 * 15)
    assert m.num_objects == 2 and m.prefix_num_verts.tolist() == [0, 256, 512]
    f = synthetic.folded_sheet(32, seed=1)
    assert f.num_faces == 2 * 31 * 31
