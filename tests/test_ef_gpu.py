"""EF detection on the GPU against the CPU oracle: identical EF pair records (48 B each).

Both the drop-in narrow phase over a broad-phase list and the fused detect kernel are
checked, in canonical (eid, fid) order.
"""
import numpy as np
import pytest

from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene

pytestmark = pytest.mark.gpu


def _oracle_ef(oracle, m, d_hat, th):
    ot = oracle.lbvh_build(oracle.TREE_FACE, m.x, m.faces)
    oracle.lbvh_refit(ot, m.x, m.x, th, m.faces)
    broad, total, _ = oracle.lbvh_query(ot, oracle.QUERY_EDGES_UNCULLED, m.x, m.x, m.edges, d_hat, th)
    ef, idx = oracle.ef_narrow(broad, m.x, m.edges, m.faces, d_hat, m.vert_property)
    return ef, idx, total


@pytest.mark.parametrize("scene", ["two_sheets64", "folded128", "folded256"])
@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("parity_tree", [True, False])
def test_ef_pairs_bit_exact(oracle, u26ctx, scene, fused, parity_tree):
    if scene == "two_sheets64":
        m = synthetic.two_sheets(64, seed=0)
    elif scene == "folded128":
        m = synthetic.folded_sheet(128, seed=3)
    else:
        m = synthetic.folded_sheet(256, seed=1)
    d_hat = np.full(m.num_verts, 1e-3, np.float32)
    th = np.zeros(m.num_verts, np.float32)
    ef_ref, idx_ref, total = _oracle_ef(oracle, m, d_hat, th)
    assert len(ef_ref) > 0
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0, max_broad_pairs=total + 64, max_ef_pairs=len(ef_ref) + 64,
                        parity_tree=parity_tree)
    sc.construct_lbvh()
    if fused:
        sc.detect_ef_fused()
    else:
        sc.broadphase_dcd_ef()
        sc.narrowphase_dcd_ef()
    ef, idx = sc.ef_pairs()
    assert np.array_equal(idx, idx_ref)
    assert ef.tobytes() == ef_ref.tobytes()
    assert u26ctx.device_errors() == 0


def test_ef_fixed_and_rigid_filters(oracle, u26ctx):
    m = synthetic.two_sheets(32, seed=4)
    vp = m.vert_property.copy()
    vp[: m.num_verts // 2] |= 1  # sheet A fixed
    vp[m.num_verts // 2:] |= 1   # sheet B fixed too: every pair rejected
    m.vert_property = vp
    d_hat = np.full(m.num_verts, 1e-3, np.float32)
    th = np.zeros(m.num_verts, np.float32)
    ef_ref, _, _ = _oracle_ef(oracle, m, d_hat, th)
    assert len(ef_ref) == 0
    sc = CollisionScene(u26ctx, m)
    sc.construct_lbvh()
    sc.detect_ef_fused()
    ef, _ = sc.ef_pairs()
    assert len(ef) == 0


def test_ef_empty_scene(u26ctx):
    m = synthetic.two_sheets(8, seed=0)
    m.x[m.num_verts // 2:, 2] += 5.0  # separate the sheets
    sc = CollisionScene(u26ctx, m)
    sc.construct_lbvh()
    sc.detect_ef_fused()
    ef, idx = sc.ef_pairs()
    assert len(ef) == 0 and len(idx) == 0
