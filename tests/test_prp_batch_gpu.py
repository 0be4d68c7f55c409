"""Independent scenes evaluated in one batch (the batching form): the batched pass returns,
for every scene, exactly the per-contour results and supports S(r) of that scene's own pass
(per-scene launches), and matches the oracle on the batched mesh."""
import numpy as np
import pytest

from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import prp_params

pytestmark = pytest.mark.gpu

ALL = dict(max_contours=1 << 20, batch_size=1 << 20)


def _pass(ctx, mesh, **kw):
    sc = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    res = sc.untangle_pass(prp_params(**kw))
    sc.close()
    assert res.device_error_flags == 0
    return res


def _map_hits(h, v0, e0, f0):
    h = h.copy()
    vf, ee, fv = h["type"] == 0, h["type"] == 1, h["type"] == 2
    h["src_id"][vf] -= v0
    h["dst_id"][vf] -= f0
    h["src_id"][ee] -= e0
    h["dst_id"][ee] -= e0
    h["src_id"][fv] -= f0
    h["dst_id"][fv] -= v0
    for k in ("sv", "dv"):
        a = h[k]
        a[a != 0xFFFFFFFF] -= v0
    return h


def test_batched_scenes_match_per_scene_passes(u26ctx):
    b = synthetic.batch_scenes(num=4, seed=5, tris_lo=2000, tris_hi=6000)
    big = _pass(u26ctx, b, **ALL)
    assert len(big.contours) >= 4
    for s in range(4):
        info = b.meta["scenes"][s]
        v0, f0 = info["verts"][0], info["faces"][0]
        e0 = int(np.searchsorted(b.edges[:, 0], v0))
        small = _pass(u26ctx, synthetic.scene_mesh(b, s), **ALL)
        mine = [c for c in range(len(big.contours)) if big.results[c]["object_id0"] // 2 == s]
        assert len(mine) == len(small.contours)
        for cs, cb in enumerate(mine):
            ra, rb = small.results[cs], big.results[cb]
            for name in ra.dtype.names:
                if name in ("contour_idx", "object_id0", "object_id1", "opt_accepted"):
                    continue
                assert np.array_equal(ra[name], rb[name]), f"scene {s} contour {cs} field {name}"
            assert small.directions[cs].tobytes() == big.directions[cb].tobytes()
            assert small.hits[cs].tobytes() == _map_hits(big.hits[cb], v0, e0, f0).tobytes()


def test_batched_scenes_oracle_parity(oracle, u26ctx):
    from test_prp_gpu import _compare
    b = synthetic.batch_scenes(num=2, seed=7, tris_lo=2000, tris_hi=4000)
    res = _pass(u26ctx, b, **ALL)
    ef, idx = oracle.detect_ef(b)
    ref = oracle.PrpRun(b, ef, idx, oracle.prp_params(**ALL))
    _compare(res, ref)


def test_solid_shells_oracle_parity(oracle, u26ctx):
    """Closed shells declared solid (object_solid) in a batch with sheets."""
    from test_prp_gpu import _compare
    b = synthetic.batch_scenes(num=3, seed=13, tris_lo=2000, tris_hi=5000)
    kinds = [s["kind"] for s in b.meta["scenes"]]
    b.object_solid = np.array([1 if kinds[o // 2] == "shells" else 0 for o in range(b.num_objects)], np.uint32)
    res = _pass(u26ctx, b, **ALL)
    ef, idx = oracle.detect_ef(b)
    ref = oracle.PrpRun(b, ef, idx, oracle.prp_params(**ALL))
    _compare(res, ref)
