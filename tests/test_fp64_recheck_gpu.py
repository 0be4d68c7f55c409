"""The filtered FP32 predicates' FP64 recheck on the GPU against the oracle.

Every VF / FV / EE leaf test of the batched ray casts and every EF test of the fused
detection whose FP32 decision lies inside its static forward-error band is re-evaluated in
FP64; the hit and pair sets keep the FP32 decisions (they stay the oracle's, bit for bit).
Checked here: the recheck and flip counts against the oracle's restatement of the same
band over the same leaf tests, and the FP64 evaluation of the selected supports (depths,
D_C, J and the D_C tie recheck) against the oracle's double instantiation of those metrics.
"""
import numpy as np
import pytest

from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import prp_params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mesh_fn,kw", [
    (lambda: synthetic.folded_sheet(64, seed=2), dict(max_contours=64)),
    (lambda: synthetic.two_sheets(48, seed=3), {}),
    (lambda: synthetic.folded_sheet(48, seed=2), dict(max_contours=64, direction_mode=1, opt_iterations=4)),
], ids=["folded64", "two_sheets48", "folded48_26dirs_4steps"])
def test_recheck_counts_and_fp64_metrics(oracle, u26ctx, mesh_fn, kw):
    from test_prp_gpu import _compare
    m = mesh_fn()
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    res = sc.untangle_pass(prp_params(fp64_recheck=1, **kw))
    ef_stats = sc.stats.cpu().numpy()
    sc.close()
    ef, idx = oracle.detect_ef(m)
    ref = oracle.PrpRun(m, ef, idx, oracle.prp_params(fp64_recheck=1, **kw))
    _compare(res, ref)  # the sets and results keep the FP32 decisions
    g, o = res.fp64, ref.fp64
    assert g["rechecks"] == o["rechecks"] and g["flips"] == o["flips"], (g, o)
    assert g["rechecks"] > 0
    for k in ("dc_tie_rechecks", "dc_tie_flips"):
        assert g[k] == o[k], (k, g, o)
    for k in ("delta_rel_err", "dc_rel_err", "j_rel_err"):
        assert g[k] == o[k], (k, g, o)  # the same double arithmetic on both sides
    # EF detection's recheck over the face-tree overlaps (the broad-phase pairs)
    dh = np.full(m.num_verts, 1e-3, np.float32)
    th = np.zeros(m.num_verts, np.float32)
    tree = oracle.lbvh_build(oracle.TREE_FACE, m.x, m.faces)
    oracle.lbvh_refit(tree, m.x, m.x, th, m.faces)
    broad, _, _ = oracle.lbvh_query(tree, oracle.QUERY_EDGES_UNCULLED, m.x, m.x, m.edges, dh, th)
    assert (int(ef_stats[2]), int(ef_stats[3])) == oracle.ef_recheck(broad, m.x, m.edges, m.faces, dh, m.vert_property)


def test_recheck_off_changes_nothing(u26ctx):
    """With the recheck off the pass returns the same results and reports no rechecks."""
    from test_prp_gpu import _compare
    m = synthetic.folded_sheet(48, seed=2)
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    on = sc.untangle_pass(prp_params(max_contours=64, fp64_recheck=1))
    off = sc.untangle_pass(prp_params(max_contours=64, fp64_recheck=0))
    sc.close()
    _compare(on, off)
    assert off.fp64["rechecks"] == 0 and off.fp64["j_rel_err"] == 0.0
    assert on.fp64["j_rel_err"] < 1e-3
