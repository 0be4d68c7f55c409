"""Region-based pair filtering on the GPU (u26_filter_invalid_pairs,
u26_filter_broad_phase_pairs) against the CPU oracle, on the contour regions of a real pass
and proximity / CCD broad-phase pairs of the same mesh. Bit-exact: disabled templates,
invalid-vertex marks and the flagged broad-phase lists."""
import numpy as np
import pytest
import torch

from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import COLLISION_PAIR_DTYPE, prp_params, response_params

pytestmark = pytest.mark.gpu


def _proximity(oracle, m, d_hat, seed):
    """VF (vertex, face) and EE (edge, edge) broad-phase pairs within d_hat, as narrow-phase
    templates with seeded barycentric coordinates."""
    rng = np.random.default_rng(seed)
    dh = np.full(m.num_verts, d_hat, np.float32)
    th = np.zeros(m.num_verts, np.float32)
    ft = oracle.lbvh_build(oracle.TREE_FACE, m.x, m.faces)
    oracle.lbvh_refit(ft, m.x, m.x, th, m.faces)
    vf, _, _ = oracle.lbvh_query(ft, oracle.QUERY_VERTS, m.x, m.x, None, dh, th)
    vf = np.array([p for p in vf if p[0] not in m.faces[p[1]]], np.uint32).reshape(-1, 2)
    et = oracle.lbvh_build(oracle.TREE_EDGE, m.x, m.edges)
    oracle.lbvh_refit(et, m.x, m.x, th, m.edges)
    ee, _, _ = oracle.lbvh_query(et, oracle.QUERY_EDGES, m.x, m.x, m.edges, dh, th)
    ee = np.array([p for p in ee if not set(m.edges[p[0]]) & set(m.edges[p[1]])], np.uint32).reshape(-1, 2)
    n = len(vf) + len(ee)
    pairs = np.zeros(n, COLLISION_PAIR_DTYPE)
    pidx = np.concatenate([vf, ee]).astype(np.uint32)
    for i, (v, f) in enumerate(vf):
        fv = m.faces[f]
        pairs[i]["indices"] = (v, fv[0], fv[1] | 0x80000000, fv[2])
    for j, (a, b) in enumerate(ee):
        pairs[len(vf) + j]["indices"] = (m.edges[a][0], m.edges[a][1], m.edges[b][0], m.edges[b][1] | 0x80000000)
    b0 = rng.uniform(0, 1, n).astype(np.float32)
    b1 = (rng.uniform(0, 1, n) * (1 - b0)).astype(np.float32)
    pairs["vec2"][:, 0] = -1e3
    pairs["vec2"][:, 1] = 1e5
    pairs["vec2"][:, 2] = b0
    pairs["vec2"][:, 3] = b1
    pairs["vec1"][:, 2] = 1.0
    return pairs, pidx, vf, ee


@pytest.mark.parametrize("n,seed", [(32, 0), (48, 3)])
def test_filter_pairs_on_pass_regions(oracle, u26ctx, n, seed):
    m = synthetic.two_sheets(n, seed=seed)
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    res = sc.untangle_pass(prp_params(), response=response_params(3e-3, 1e8))
    r = res.response
    num_ef = len(res.pairs)
    assert num_ef > 0 and r.num_pairs > 0
    regions = tuple(t.cpu().numpy().view(np.uint32) for t in (r.vert_regions, r.edge_regions, r.face_regions))
    pairs, pidx, vf, ee = _proximity(oracle, m, 0.02, seed)
    assert len(vf) > 0 and len(ee) > 0
    offset = np.full(m.num_verts, 1e-3, np.float32)
    dev = torch.device("cuda", u26ctx.device)

    # filter_invalid_pairs
    d_pairs = torch.from_numpy(pairs.view(np.int32).reshape(-1, 16).copy()).to(dev)
    d_pidx = torch.from_numpy(pidx.view(np.int32).copy()).to(dev)
    d_off = torch.from_numpy(offset).to(dev)
    d_inv = torch.zeros(m.num_verts, dtype=torch.int32, device=dev)
    sc.filter_invalid_pairs(d_pairs, d_pidx, len(pairs), d_off, d_inv, response=r)
    want, inv_w = oracle.filter_invalid_pairs(pairs, pidx, num_ef, m.x, offset, np.zeros(m.num_verts, np.uint32), regions)
    inv = d_inv.cpu().numpy().view(np.uint32)
    assert np.array_equal(inv, inv_w)
    assert d_pairs.cpu().numpy().view(np.uint32).tobytes() == want.tobytes()
    disabled = int((want["vec2"][:, 1] == 0).sum())
    assert 0 < int(inv.sum()) and 0 < disabled < len(want)

    # filter_broad_phase_pairs with the invalid marks just made
    d_vf = torch.from_numpy(vf.view(np.int32).copy()).to(dev)
    d_ee = torch.from_numpy(ee.view(np.int32).copy()).to(dev)
    sc.filter_broad_phase_pairs(d_vf, len(vf), d_ee, len(ee), d_inv, r)
    w_vf, w_ee = oracle.filter_broad_phase(vf, ee, num_ef, inv_w, regions, m.faces, m.edges)
    assert np.array_equal(d_vf.cpu().numpy().view(np.uint32), w_vf)
    assert np.array_equal(d_ee.cpu().numpy().view(np.uint32), w_ee)
    assert (w_vf[:, 0] >> 30 != 0).any()
    sc.close()


def test_filter_without_regions_or_ef(oracle, u26ctx):
    """No EF pairs: nothing changes; no regions: only the invalid-vertex rule applies."""
    m = synthetic.two_sheets(32, seed=0)
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    pairs, pidx, vf, ee = _proximity(oracle, m, 0.02, 1)
    offset = np.full(m.num_verts, 1e-3, np.float32)
    dev = torch.device("cuda", u26ctx.device)
    d_pairs = torch.from_numpy(pairs.view(np.int32).reshape(-1, 16).copy()).to(dev)
    d_pidx = torch.from_numpy(pidx.view(np.int32).copy()).to(dev)
    d_off = torch.from_numpy(offset).to(dev)
    d_inv = torch.zeros(m.num_verts, dtype=torch.int32, device=dev)
    sc.filter_invalid_pairs(d_pairs, d_pidx, len(pairs), d_off, d_inv, response=None, num_ef=0)
    assert d_pairs.cpu().numpy().view(np.uint32).tobytes() == pairs.tobytes() and int(d_inv.sum()) == 0
    sc.filter_invalid_pairs(d_pairs, d_pidx, len(pairs), d_off, d_inv, response=None, num_ef=5)
    want, inv_w = oracle.filter_invalid_pairs(pairs, pidx, 5, m.x, offset, np.zeros(m.num_verts, np.uint32), None)
    assert d_pairs.cpu().numpy().view(np.uint32).tobytes() == want.tobytes()
    assert np.array_equal(d_inv.cpu().numpy().view(np.uint32), inv_w)
    sc.close()
