"""The untangling26 entry point on the GPU: a two-sheet interpenetration written as OBJ is
repaired by updates along the assembled responses; the report has the reference CLI's keys
(cli.py:194-215) and the written mesh is the state the last report describes; the response
step (u26_response_step) is deterministic."""
import json

import numpy as np
import pytest

from untangling26 import cli
from untangling26_b200 import mesh_io

pytestmark = pytest.mark.gpu


def test_repair_two_sheets(tmp_path, u26ctx):
    from test_cli import _write_sheets
    _write_sheets(tmp_path / "in.obj", n=16)
    rc = cli.main([str(tmp_path / "in.obj"), str(tmp_path / "out.obj"), "--max-iters", "40"])
    report = json.loads((tmp_path / "out.json").read_text())
    for k in ("inputs", "outputs", "bodies", "converged", "stop_reason", "initial_ef_pairs", "final_ef_pairs", "iterations",
              "solver_calls", "elapsed_seconds", "configuration", "normalization", "history"):
        assert k in report, k
    assert report["initial_ef_pairs"] > 0
    assert rc == (0 if report["converged"] else 1)
    assert report["final_ef_pairs"] < report["initial_ef_pairs"]
    out = mesh_io.load_bodies([tmp_path / "out.obj"])
    assert [len(b.vertices) for b in out] == [b["vertices"] for b in report["bodies"]]
    assert all(np.isfinite(b.vertices).all() for b in out)


def test_response_step_is_deterministic(u26ctx):
    from untangling26_b200 import synthetic
    from untangling26_b200.intersection_resolver import CollisionScene
    from untangling26_b200.prp import prp_params, response_params
    m = synthetic.two_sheets(32, seed=0)
    outs = []
    for _ in range(2):
        sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
        sc.construct_lbvh()
        res = sc.untangle_pass(prp_params(), response=response_params(3e-3, 1e8))
        assert sc.response_step(res.response, 1.0) > 0
        outs.append(sc.x.cpu().numpy().copy())
        sc.close()
    assert outs[0].tobytes() == outs[1].tobytes()
    assert not np.array_equal(outs[0], m.x)
    # every displacement is bounded by half the largest requested depth (3e-3 + 3e-3) per pair
    assert np.abs(outs[0] - m.x).max() <= 3.1e-3
