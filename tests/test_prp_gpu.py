"""PRP contour evaluation on the GPU (C ABI u26_prp_resolve) against the CPU oracle.

Bit-exact: augmented EF list (loop-vertex pairs), contour flood fill and mesh parity,
candidate directions, per-contour results (selected direction, k-ring levels, J, depth,
volume, area, displacement cost, coverage, flags) and the selected hit sets S(r).
"""
import numpy as np
import pytest

from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import prp_params

pytestmark = pytest.mark.gpu


def _run_both(oracle, ctx, mesh, **kw):
    sc = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    res = sc.untangle_pass(prp_params(**kw))
    ef_ref, idx_ref = oracle.detect_ef(mesh)
    ref = oracle.PrpRun(mesh, ef_ref, idx_ref, oracle.prp_params(**kw))
    sc.close()
    return res, ref


def _compare(res, ref):
    assert res.num_orig_pairs == ref.num_orig_pairs
    # the ray-primitive pair count (the bench metric's unit) is the same work on both sides
    assert res.pairs_tested == ref.pairs_tested
    assert res.requests == ref.requests
    assert res.pairs.tobytes() == ref.pairs.tobytes()
    assert np.array_equal(res.pair_indices, ref.pair_indices)
    assert np.array_equal(res.mesh_index, ref.mesh_index)
    assert np.array_equal(res.contour_index, ref.contour_index)
    assert res.pair_length.tobytes() == ref.pair_length.tobytes()
    assert len(res.contours) == len(ref.contours)
    for a, b in zip(res.contours, ref.contours):
        assert np.array_equal(a, b)
    for c in range(len(ref.contours)):
        ra, rb = res.results[c], ref.results[c]
        for name in ref.results.dtype.names:
            if name.startswith("reserved"):
                continue
            assert np.array_equal(ra[name], rb[name]), f"contour {c} field {name}: gpu {ra[name]} oracle {rb[name]}"
        assert res.directions[c].tobytes() == ref.directions[c].tobytes(), f"contour {c} directions"
        assert res.hits[c].tobytes() == ref.hits[c].tobytes(), f"contour {c} hit set"


@pytest.mark.parametrize("n,seed", [(32, 0), (64, 0), (64, 3)])
def test_prp_two_sheets(oracle, u26ctx, n, seed):
    m = synthetic.two_sheets(n, seed=seed)
    res, ref = _run_both(oracle, u26ctx, m)
    assert len(ref.contours) > 0
    assert any(r["hit_count"] > 0 for r in ref.results)
    _compare(res, ref)
    assert res.device_error_flags == 0


def test_prp_two_sheets_26_directions(oracle, u26ctx):
    m = synthetic.two_sheets(32, seed=1)
    res, ref = _run_both(oracle, u26ctx, m, direction_mode=1)
    assert all(r["num_dirs"] == 26 for r in ref.results if r["flags"] & 16)
    _compare(res, ref)


@pytest.mark.parametrize("ccr", [(1, 1, 1, 0), (1, 1, 0, 0), (1, 0, 1, 0), (0, 0, 0, 0), (1, 1, 1, 1)])
def test_prp_folded_sheet(oracle, u26ctx, ccr):
    """Contour-side restriction modes: rest AND current (default), rest only, current only,
    off, and the blended coordinate (weight 0.5)."""
    m = synthetic.folded_sheet(48, seed=2)
    res, ref = _run_both(oracle, u26ctx, m, use_ccr=ccr[0], ccr_use_rest=ccr[1], ccr_use_current=ccr[2], ccr_blend=ccr[3],
                         max_contours=64)
    assert len(ref.contours) > 1
    _compare(res, ref)


def test_prp_two_objects_rest_only_restriction(oracle, u26ctx):
    # rest-geodesic ownership only applies when both sides share an object and component;
    # across two sheets the candidates stay unrestricted
    m = synthetic.two_sheets(32, seed=2)
    res, ref = _run_both(oracle, u26ctx, m, ccr_use_current=0)
    _compare(res, ref)


def test_prp_no_intersections(oracle, u26ctx):
    m = synthetic.two_sheets(16, seed=0)
    m.x[m.num_verts // 2:, 2] += 3.0
    res, ref = _run_both(oracle, u26ctx, m)
    assert len(res.contours) == 0 and len(ref.contours) == 0


@pytest.mark.parametrize("iters", [1, 8])
def test_prp_direction_refinement(oracle, u26ctx, iters):
    """Projected Newton / Cauchy refinement of the selected direction on S^2: the steps,
    the trial evaluations from the initial k-ring level and the accept / reject decisions
    (trial and accepted counts) match the oracle bit for bit."""
    m = synthetic.folded_sheet(48, seed=2)
    res, ref = _run_both(oracle, u26ctx, m, opt_iterations=iters, max_contours=64)
    assert any(r["opt_accepted"] > 0 for r in ref.results)
    assert all(r["opt_attempted"] <= iters for r in ref.results)
    _compare(res, ref)
    assert res.device_error_flags == 0


def test_prp_direction_refinement_flat_supports(oracle, u26ctx):
    # two flat sheets: the supports' normals are parallel to the selected direction, the
    # tangent gradient vanishes and no trial is taken
    m = synthetic.two_sheets(32, seed=0)
    res, ref = _run_both(oracle, u26ctx, m, opt_iterations=4)
    assert all(r["opt_attempted"] == 0 for r in ref.results)
    _compare(res, ref)


@pytest.mark.parametrize("mesh_fn", [lambda: synthetic.folded_sheet(48, seed=2), lambda: synthetic.two_sheets(64, seed=3)])
def test_prp_plain_form_same_results(u26ctx, mesh_fn):
    """The plain form (one thread per request from the tree root, per-contour launches, no
    candidate-box clipping) decides the same pairs and returns the same results as the
    batched packet form."""
    m = mesh_fn()
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    chosen = sc.untangle_pass(prp_params(max_contours=64))
    plain = sc.untangle_pass(prp_params(max_contours=64, form=1))
    sc.close()
    assert plain.device_error_flags == 0 and chosen.device_error_flags == 0
    _compare(plain, chosen)


def test_prp_solid_interior_links(oracle, u26ctx):
    """Solid-interior hit links (rigid / tetrahedral meshes): with every mesh treated as solid,
    the rays through the folded sheet's two layers link entry and exit hits; the components,
    supports and metrics change and still match the oracle bit for bit."""
    m = synthetic.folded_sheet(48, seed=2)
    res, ref = _run_both(oracle, u26ctx, m, solid_all=1, max_contours=64)
    base = oracle.PrpRun(m, *oracle.detect_ef(m), oracle.prp_params(max_contours=64))
    assert any(a["hit_count"] != b["hit_count"] for a, b in zip(ref.results, base.results))
    _compare(res, ref)
