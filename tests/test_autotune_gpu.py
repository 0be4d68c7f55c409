"""Ray-casting configurations and the autotuner: every configuration (subtree parts x blocks per
SM x grid form, a warp per work item or a persistent work-queue grid) returns exactly the
oracle's results; the autotuning pass times all eighteen, picks the fastest and the scene's later
passes use it, with unchanged results."""
import pytest

from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import RAYCAST_CONFIGS, config_name, prp_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def folded_ref(oracle):
    m = synthetic.folded_sheet(48, seed=2)
    ef, idx = oracle.detect_ef(m)
    return m, oracle.PrpRun(m, ef, idx, oracle.prp_params(max_contours=64, fp64_recheck=1))


@pytest.mark.parametrize("k", range(1, len(RAYCAST_CONFIGS) + 1), ids=[config_name(c) for c in RAYCAST_CONFIGS])
def test_every_configuration_matches_oracle(u26ctx, folded_ref, k):
    from test_prp_gpu import _compare
    m, ref = folded_ref
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    res = sc.untangle_pass(prp_params(max_contours=64, raycast_config=k))
    sc.close()
    rc = res.raycast_config
    assert (rc["parts"], rc["blocks_per_sm"], rc["queue"]) == RAYCAST_CONFIGS[k - 1]
    _compare(res, ref)
    assert res.fp64["rechecks"] == ref.fp64["rechecks"] and res.fp64["flips"] == ref.fp64["flips"]


def test_autotune_picks_the_fastest_and_keeps_it(u26ctx, folded_ref):
    from test_prp_gpu import _compare
    m, ref = folded_ref
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    first = sc.untangle_pass(prp_params(max_contours=64, autotune=1))
    second = sc.untangle_pass(prp_params(max_contours=64, autotune=1))
    sc.close()
    assert first.raycast_config["tuned_this_pass"] and not second.raycast_config["tuned_this_pass"]
    times = first.raycast_config["tune_ms"]
    assert len(times) == len(RAYCAST_CONFIGS) and all(t > 0 for t in times.values())
    best = min(times, key=times.get)
    rc = second.raycast_config
    assert best == config_name((rc["parts"], rc["blocks_per_sm"], rc["queue"]))
    _compare(first, ref)
    _compare(second, ref)
