"""PRP parity on the benchmarked workloads at full size: the GPU pass (u26_prp_resolve through
the C ABI) against the oracle on the same inputs.

* the precision-form scene (one 256 x 256 sheet folded once, 130,050 triangles): the GPU
  evaluates the first 256 contours; the oracle evaluates every 8th of them (its cost), and
  each of those is compared field by field, direction by direction and hit by hit. With
  the 26 lattice directions and up to 8 S^2 refinement steps (the precision form's
  settings) every 16th contour is compared.
* the batching form (64 two-body scenes, 1.97 M triangles, one batched pass): four whole
  scenes (s % 16 == 4) against the oracle's pass of each scene alone.
A contour that cross-contour suppression removed in either pass is compared on its
pre-suppression fields: the sampled oracle pass sees only some of its suppression partners.
"""
import numpy as np
import pytest

from oracle.compare import compare_contours, compare_scene
from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import prp_params

pytestmark = pytest.mark.gpu

ALL = dict(max_contours=1 << 20, batch_size=1 << 20)


def _gpu_pass(ctx, mesh, **kw):
    sc = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0, max_ef_pairs=max(1 << 16, mesh.num_edges))
    sc.construct_lbvh()
    res = sc.untangle_pass(prp_params(**kw))
    sc.close()
    assert res.device_error_flags == 0
    return res


@pytest.fixture(scope="module")
def folded256():
    return synthetic.folded_sheet(256, seed=1)


@pytest.fixture(scope="module")
def folded256_ef(oracle, folded256):
    return oracle.detect_ef(folded256)


@pytest.mark.parametrize("stride,kw", [(8, {}), (16, dict(direction_mode=1, opt_iterations=8))],
                         ids=["seeds", "26dirs_8steps"])
def test_folded256_contours(oracle, u26ctx, folded256, folded256_ef, stride, kw):
    m = folded256
    res = _gpu_pass(u26ctx, m, max_contours=256, **kw)
    ref = oracle.PrpRun(m, *folded256_ef, oracle.prp_params(max_contours=256, contour_stride=stride, **kw))
    # the EF list, its loop-vertex pairs and the contours do not depend on the sampling
    assert res.pairs.tobytes() == ref.pairs.tobytes()
    assert len(res.contours) == len(ref.contours) > 256
    for a, b in zip(res.contours, ref.contours):
        assert np.array_equal(a, b)
    cs = list(range(0, 256, stride))
    assert all(ref.results[c]["flags"] & 16 for c in cs)
    nh = compare_contours(res, ref, cs)
    assert nh > 0
    if kw.get("opt_iterations"):
        # the 26 lattice directions; the refinement's outcome (steps tried and accepted, both zero on
        # these contours when their supports give no tangent descent) is among the compared fields
        assert all(r["num_dirs"] == 26 for r in ref.results[cs])


def test_batch64_scenes(oracle, u26ctx):
    b = synthetic.batch_scenes(64, seed=2)
    res = _gpu_pass(u26ctx, b, **ALL)
    ncont = 0
    for s in (4, 20, 36, 52):
        m = synthetic.scene_mesh(b, s)
        ef, idx = oracle.detect_ef(m)
        ref = oracle.PrpRun(m, ef, idx, oracle.prp_params(**ALL))
        c, h = compare_scene(res, b, s, ref)
        ncont += c
    assert ncont >= 4
