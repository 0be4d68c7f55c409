"""The reference's seven canonical self-intersection units (Resources/InputMesh/
SelfIntersectionUnit/unit_*.obj, named after Wicke et al.'s contour types), read as inputs
at test time from the reference checkout (U26_UNIT_MESH_DIR overrides the directory); the
tests skip where those files are absent. Nothing of them is copied into this repository.

The contour type is classify_contour_type's (intersection_resolver2.cpp:311-375). With
use_untangling_GIA off, the setting of the PRP path (cli.py:99), every EF pair whose edge
has an incident face closing on the intersected face adds its own loop-vertex pair
(find_loop_vertex, intersection_resolver.cpp:431-500, 986-1011), and a loop pair is
adjacent to its EF pair only. So the Eight unit, whose one loop vertex is reached from two
EF pairs, carries two loop pairs and classifies as LL, and the Cross unit falls apart at
its loop vertex into two BLI contours; the other five units classify as their names say.
"""
import os

import numpy as np
import pytest

from untangling26_b200 import mesh_io

CLOSED, EIGHT, LL, BLI, CROSS, BIBI, BBII = 1, 2, 3, 4, 5, 6, 7
EXPECTED = {  # unit -> contour types of its pass
    "Closed": [CLOSED], "LL": [LL], "BLI": [BLI], "BIBI": [BIBI], "BBII": [BBII],
    "Eight": [LL], "Cross": [BLI, BLI],
}


def _unit_dir():
    d = os.environ.get("U26_UNIT_MESH_DIR")
    if d:
        return d
    return os.path.join(os.sep, "root", "reference", "Resources", "InputMesh", "SelfIntersectionUnit")


def _unit_mesh(name):
    path = os.path.join(_unit_dir(), f"unit_{name}.obj")
    if not os.path.exists(path):
        pytest.skip(f"reference unit mesh not present: {path}")
    return mesh_io.mesh_from_bodies(mesh_io.load_bodies([path]))


@pytest.mark.parametrize("name", sorted(EXPECTED))
def test_unit_contour_types_oracle(oracle, name):
    m = _unit_mesh(name)
    ef, idx = oracle.detect_ef(m)
    run = oracle.PrpRun(m, ef, idx, oracle.prp_params())
    assert [int(r["contour_type"]) for r in run.results] == EXPECTED[name]
    # every contour gets a response: a direction whose support separates it
    assert all(r["combo_idx"] != 0xFFFFFFFF and r["hit_count"] > 0 for r in run.results)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(EXPECTED))
def test_unit_gpu_matches_oracle(oracle, u26ctx, name):
    from test_prp_gpu import _compare
    from untangling26_b200.intersection_resolver import CollisionScene
    from untangling26_b200.prp import prp_params
    m = _unit_mesh(name)
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    res = sc.untangle_pass(prp_params())
    sc.close()
    ef, idx = oracle.detect_ef(m)
    ref = oracle.PrpRun(m, ef, idx, oracle.prp_params())
    assert [int(r["contour_type"]) for r in res.results] == EXPECTED[name]
    _compare(res, ref)
    assert np.all(res.results["hit_count"] > 0)
