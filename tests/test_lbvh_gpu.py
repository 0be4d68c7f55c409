"""LBVH on the GPU (through the C ABI) against the CPU oracle, bit for bit.

Compared: global AABB, sorted Morton keys, sorted_get_original, parent, children,
object_idx (topology, bit-exact), node AABB xyz after refit (bit-exact: min/max are
exact), and the broad-phase pair sets of all three query modes.
"""
import numpy as np
import pytest
import torch

from untangling26_b200 import synthetic
from untangling26_b200.lbvh import LBVH, TREE_EDGE, TREE_FACE, TREE_VERT
from untangling26_b200.mesh import Mesh

pytestmark = pytest.mark.gpu


def _dev(a, dtype=None):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a).cuda()


def _sorted_pairs(p):
    p = np.asarray(p, dtype=np.uint32).reshape(-1, 2)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def _build_both(oracle, ctx, tree_type, mesh, x0=None, x1=None, thickness=None, fused=True):
    x0 = mesh.x if x0 is None else x0
    x1 = x0 if x1 is None else x1
    prims = {TREE_FACE: mesh.faces, TREE_EDGE: mesh.edges, TREE_VERT: None}[tree_type]
    n = {TREE_FACE: mesh.num_faces, TREE_EDGE: mesh.num_edges, TREE_VERT: mesh.num_verts}[tree_type]
    th = np.zeros(mesh.num_verts, np.float32) if thickness is None else thickness
    ot = oracle.lbvh_build(tree_type, x0, prims, num_verts=mesh.num_verts)
    oracle.lbvh_refit(ot, x0, x1, th, prims)
    t = LBVH(ctx, tree_type, n)
    dx0, dx1, dth = _dev(x0), _dev(x1), _dev(th)
    dprims = None if prims is None else _dev(prims)
    if tree_type == TREE_FACE:
        t.reduce_face_tree_aabb(dx0, dprims)
    elif tree_type == TREE_EDGE:
        t.reduce_edge_tree_aabb(dx0, dprims)
    else:
        t.reduce_vert_tree_aabb(dx0)
    t.construct_tree()
    if fused:
        t.update_and_refit(dth, dx0, dx1, dprims)
    else:
        if tree_type == TREE_FACE:
            t.update_face_tree_leave_aabb(dth, dx0, dx1, dprims)
        elif tree_type == TREE_EDGE:
            t.update_edge_tree_leave_aabb(dth, dx0, dx1, dprims)
        else:
            t.update_vert_tree_leave_aabb(dth, dx0, dx1)
        t.refit()
    return ot, t, (dx0, dx1, dth, dprims)


def _assert_tree_equal(ot, arr):
    n = ot.n
    assert np.array_equal(arr["global_aabb"], ot.gaabb)
    assert np.array_equal(arr["morton_sorted"], ot.keys_sorted[:n])
    assert np.array_equal(arr["sorted_get_original"], ot.sorted_get_original[:n])
    assert np.array_equal(arr["parent"], ot.parent)
    ni = n - 1
    assert np.array_equal(arr["children"][:ni], ot.children[:ni])
    assert np.array_equal(arr["children"][ni:], ot.children[ni:])
    assert np.array_equal(arr["object_idx"], ot.object_idx)
    ab = arr["node_aabb"]
    assert np.array_equal(ab[:, [0, 1, 2, 4, 5, 6]], ot.node_aabb[:, [0, 1, 2, 4, 5, 6]])


@pytest.mark.parametrize("tree_type", [TREE_FACE, TREE_EDGE, TREE_VERT])
@pytest.mark.parametrize("fused", [True, False])
def test_build_refit_two_sheets(oracle, u26ctx, tree_type, fused):
    m = synthetic.two_sheets(64, seed=0)
    th = np.full(m.num_verts, 1e-3, np.float32)
    x1 = m.x + np.float32(0.01) * np.sin(m.x * 7).astype(np.float32)
    ot, t, _ = _build_both(oracle, u26ctx, tree_type, m, m.x, x1, th, fused=fused)
    assert t.check_health()
    _assert_tree_equal(ot, t.arrays())


def test_build_refit_folded_full_size(oracle, u26ctx):
    m = synthetic.folded_sheet(256, seed=1)
    th = np.full(m.num_verts, 1e-4, np.float32)
    for tt in (TREE_FACE, TREE_EDGE):
        ot, t, _ = _build_both(oracle, u26ctx, tt, m, thickness=th)
        assert t.check_health()
        _assert_tree_equal(ot, t.arrays())


@pytest.mark.parametrize("n_leaves", [1, 2, 3, 255, 256, 257, 5000])
def test_edge_cases_sizes(oracle, u26ctx, n_leaves):
    rng = np.random.default_rng(n_leaves)
    x = rng.uniform(-1, 1, (n_leaves * 3, 3)).astype(np.float32)
    f = np.arange(n_leaves * 3, dtype=np.uint32).reshape(-1, 3)
    m = Mesh(x, f)
    ot, t, _ = _build_both(oracle, u26ctx, TREE_FACE, m)
    arr = t.arrays()
    _assert_tree_equal(ot, arr)


def test_identical_centroids(oracle, u26ctx):
    """All leaves in one Morton cell: ties resolved by leaf id, tree still valid."""
    x = np.zeros((300, 3), np.float32)
    x[:, 0] = np.linspace(0, 1e-9, 300)
    f = np.stack([np.arange(100) * 3, np.arange(100) * 3 + 1, np.arange(100) * 3 + 2], 1).astype(np.uint32)
    m = Mesh(x, f)
    ot, t, _ = _build_both(oracle, u26ctx, TREE_FACE, m)
    assert t.check_health()
    _assert_tree_equal(ot, t.arrays())


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_broad_phase_pair_sets(oracle, u26ctx, mode):
    m = synthetic.two_sheets(64, seed=1)
    d_hat = np.full(m.num_verts, 1e-3, np.float32)
    th = np.full(m.num_verts, 5e-4, np.float32)
    tt = TREE_VERT if False else (TREE_FACE if mode in (0, 2) else TREE_EDGE)
    ot, t, (dx0, dx1, dth, dprims) = _build_both(oracle, u26ctx, tt, m, thickness=th)
    ref, total, overflow = oracle.lbvh_query(ot, mode, m.x, m.x, m.edges, d_hat, th)
    cap = total + 16
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    pairs = torch.zeros((cap, 2), dtype=torch.int32, device="cuda")
    dedges = _dev(m.edges)
    ddh = _dev(d_hat)
    if mode == 0:
        t.broad_phase_query_from_verts(dx0, dx0, count, pairs, ddh, dth)
    elif mode == 1:
        t.broad_phase_query_from_edges(dx0, dx0, dedges, count, pairs, ddh, dth)
    else:
        t.broad_phase_query_from_edges_unculled(dx0, dx0, dedges, count, pairs, ddh, dth)
    k = int(count.item())
    assert k == total
    got = pairs[:k].cpu().numpy().view(np.uint32)
    assert np.array_equal(_sorted_pairs(got), _sorted_pairs(ref))
    assert u26ctx.device_errors() == 0


def test_capacity_truncation_reports_count(oracle, u26ctx):
    m = synthetic.two_sheets(32, seed=1)
    d_hat = np.full(m.num_verts, 1e-3, np.float32)
    th = np.zeros(m.num_verts, np.float32)
    ot, t, (dx0, dx1, dth, dprims) = _build_both(oracle, u26ctx, TREE_FACE, m, thickness=th)
    _, total, _ = oracle.lbvh_query(ot, 2, m.x, m.x, m.edges, d_hat, th)
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    pairs = torch.full((8, 2), -7, dtype=torch.int32, device="cuda")
    t.broad_phase_query_from_edges_unculled(dx0, dx0, _dev(m.edges), count, pairs, _dev(d_hat), dth)
    assert int(count.item()) == total > 8
    assert (pairs.cpu().numpy() != -7).all()


@pytest.mark.parametrize("n_leaves", [2, 3, 33, 511, 512, 513, 1023, 1024, 1025, 2049, 70000])
def test_repeated_refits(oracle, u26ctx, n_leaves):
    """Refit after refit at moving positions, fused and leaf-only, around the 1024-leaf treelet
    bound (one chunk, a top tree of one node, several chunks): the refit plan made at
    construction serves every later refit, and every refit's boxes equal the oracle's."""
    rng = np.random.default_rng(n_leaves)
    x = rng.uniform(-1, 1, (n_leaves * 3, 3)).astype(np.float32)
    f = np.arange(n_leaves * 3, dtype=np.uint32).reshape(-1, 3)
    m = Mesh(x, f)
    th = np.zeros(m.num_verts, np.float32)
    ot, t, (dx0, dx1, dth, dprims) = _build_both(oracle, u26ctx, TREE_FACE, m)
    for k in range(4):
        xk = (x + np.float32(0.05 * (k + 1)) * np.sin(x * (k + 2))).astype(np.float32)
        oracle.lbvh_refit(ot, xk, xk, th, m.faces)
        dxk = _dev(xk)
        if k % 2:
            t.update_face_tree_leave_aabb(dth, dxk, dxk, dprims)
            t.refit()
        else:
            t.update_and_refit(dth, dxk, dxk, dprims)
        assert t.check_health()
        _assert_tree_equal(ot, t.arrays())


@pytest.mark.parametrize("clusters", [1, 7])
def test_refit_deep_tree(oracle, u26ctx, clusters):
    """Triangles crowded into a few points share Morton codes, so the Karras tree splits on the
    leaf index below them: long chains, treelets of every size, single-leaf treelets hanging off
    top nodes. The refit (fused and leaf-only) still equals the oracle bit for bit."""
    rng = np.random.default_rng(clusters)
    n = 6000
    centers = rng.uniform(-1, 1, (clusters, 3)).astype(np.float32)
    which = rng.integers(0, clusters, n * 3)
    x = (centers[which] + rng.normal(0, 1e-7, (n * 3, 3))).astype(np.float32)
    m = Mesh(x, np.arange(n * 3, dtype=np.uint32).reshape(-1, 3))
    for fused in (True, False):
        ot, t, _ = _build_both(oracle, u26ctx, TREE_FACE, m, fused=fused)
        assert t.check_health()
        _assert_tree_equal(ot, t.arrays())
