"""The scale form at full size: five stacked 512 x 512 sheets (2.6 M triangles, nested
contours through several neighbours), two passes of the repair loop.

* pass 1 (all 199 contours, up to 10^9 ray requests in one level): the GPU's EF list and
  every contour equal the oracle's; contours 1, 3 and 5 (the oracle needs 3-30 s per contour
  of this mesh, up to minutes for the largest regions) are compared field by field, direction
  by direction and hit by hit;
* the fixed step along the GPU's assembled response (u26_response_step) gives the positions
  the oracle's restatement of the step gives, bit for bit;
* pass 2 on the stepped positions: the GPU's EF list equals the oracle's again (the
  "remaining EF pairs" of the repair loop).
"""
import copy

import numpy as np
import pytest

from oracle.compare import compare_contours
from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import prp_params, response_params

pytestmark = pytest.mark.gpu

PARAMS = dict(max_contours=256, batch_size=32)
RESPONSE = (3e-3, 1e8)


def test_layered_repair_two_passes(oracle, u26ctx):
    m = synthetic.layered_sheets(512, layers=5, seed=4)
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0, max_ef_pairs=1 << 18)
    try:
        sc.construct_lbvh()
        res = sc.untangle_pass(prp_params(**PARAMS), response=response_params(*RESPONSE))
        assert res.device_error_flags == 0
        ef, idx = oracle.detect_ef(m)
        assert len(ef) > 10000
        nh = 0
        for off in (1, 3, 5):
            ref = oracle.PrpRun(m, ef, idx, oracle.prp_params(contour_stride=256, contour_offset=off, **PARAMS))
            if off == 1:
                assert res.pairs.tobytes() == ref.pairs.tobytes()
                assert len(res.contours) == len(ref.contours) > 100
                assert all(np.array_equal(a, b) for a, b in zip(res.contours, ref.contours))
            # a contour suppressed in the whole pass is compared on its pre-suppression fields
            nh += compare_contours(res, ref, [off])
        assert nh > 0
        # the step along the GPU's response, restated on the CPU
        want, moved = oracle.response_step(res.response.host_pairs(), m.x, 1.0)
        assert sc.response_step(res.response, 1.0) == moved > 0
        x1 = sc.x.cpu().numpy().reshape(-1, 3)
        assert x1.tobytes() == want.tobytes()
        # pass 2: the remaining EF pairs
        sc.detect_ef_fused()
        got, got_idx = sc.ef_pairs()
        stepped = copy.copy(m)
        stepped.x = x1
        ef2, idx2 = oracle.detect_ef(stepped)
        assert 0 < len(got) == len(ef2)
        assert np.array_equal(got_idx.reshape(-1, 2), np.asarray(idx2, np.uint32).reshape(-1, 2))
        assert got.tobytes() == ef2.tobytes()
    finally:
        sc.close()
