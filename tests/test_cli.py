"""The untangling26 entry point without a GPU: argument handling, OBJ input / output and
output protection (the reference tests its CLI the same way, PythonBindings/tests/test_cli.py,
with the native solver left out)."""
import numpy as np
import pytest

from untangling26 import cli
from untangling26_b200 import mesh_io, synthetic


def _write_sheets(path, n=8):
    m = synthetic.two_sheets(n, seed=0)
    nv = m.num_verts // 2
    bodies = [mesh_io.Body("a", m.x[:nv].astype(np.float64), m.faces[: len(m.faces) // 2].astype(np.int32), "gen"),
              mesh_io.Body("b", m.x[nv:].astype(np.float64), (m.faces[len(m.faces) // 2:] - nv).astype(np.int32), "gen")]
    mesh_io.write_mesh(path, bodies)
    return m, bodies


def test_obj_round_trip(tmp_path):
    m, bodies = _write_sheets(tmp_path / "in.obj")
    got = mesh_io.load_bodies([tmp_path / "in.obj"])
    assert [len(b.vertices) for b in got] == [len(b.vertices) for b in bodies]
    for g, b in zip(got, bodies):
        assert np.array_equal(g.faces, b.faces)
        assert np.array_equal(g.vertices.astype(np.float32), b.vertices.astype(np.float32))
    mesh = mesh_io.mesh_from_bodies(got)
    assert mesh.num_objects == 2 and np.array_equal(mesh.faces, m.faces)


def test_obj_polygons_negative_indices_and_split(tmp_path):
    p = tmp_path / "quad.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf -4 -3 -2 -1\nv 5 0 0\nv 6 0 0\nv 5 1 0\nf 5 6 7\n")
    (one,) = mesh_io.load_bodies([p])
    assert one.faces.tolist() == [[0, 1, 2], [0, 2, 3], [4, 5, 6]]
    parts = mesh_io.load_bodies([p], split=True)
    assert [len(b.vertices) for b in parts] == [4, 3]
    assert parts[1].faces.tolist() == [[0, 1, 2]]


def test_normalize_and_validate():
    b = mesh_io.Body("x", np.array([[0, 0, 0], [2, 0, 0], [0, 4, 0]], float), np.array([[0, 1, 2]]), "s")
    (n,), center, scale = mesh_io.normalize_bodies([b])
    assert scale == 4.0 and np.allclose(center, [1, 2, 0]) and np.ptp(n.vertices, axis=0).max() == 1.0
    with pytest.raises(ValueError):
        mesh_io.validate_mesh(np.array([[0, 0, np.nan]]), np.array([[0, 0, 0]]), "bad")
    with pytest.raises(ValueError):
        mesh_io.validate_mesh(np.zeros((3, 3)), np.array([[0, 1, 3]]), "bad")


def test_output_paths_and_protection(tmp_path):
    _, bodies = _write_sheets(tmp_path / "in.obj")
    meshes, report = mesh_io.output_paths(tmp_path / "out.obj", bodies)
    assert meshes == [(tmp_path / "out.obj").resolve()] and report.suffix == ".json"
    meshes, report = mesh_io.output_paths(tmp_path / "outdir", bodies)
    assert meshes[0].name == "resolved.obj" and len(meshes) == 3 and report.name == "summary.json"
    with pytest.raises(ValueError):
        mesh_io.check_outputs([tmp_path / "in.obj"], [tmp_path / "in.obj"], overwrite=True)
    (tmp_path / "out.obj").write_text("x")
    with pytest.raises(ValueError):
        mesh_io.check_outputs([tmp_path / "out.obj"], [tmp_path / "in.obj"])
    mesh_io.check_outputs([tmp_path / "out.obj"], [tmp_path / "in.obj"], overwrite=True)


def test_cli_errors_exit_2(tmp_path, capsys):
    assert cli.main([str(tmp_path / "missing.obj"), str(tmp_path / "out.obj")]) == 2
    assert "not found" in capsys.readouterr().err
    (tmp_path / "in.stl").write_text("solid x\nendsolid x\n")
    assert cli.main([str(tmp_path / "in.stl"), str(tmp_path / "out.obj")]) == 2
    with pytest.raises(SystemExit):
        cli.make_parser().parse_args(["a.obj", "b.obj", "--max-contours", "0"])
    args = cli.make_parser().parse_args(["a.obj", "b.obj", "--material", "rigid", "--direction-iters", "3"])
    params, resp = cli.configure(args)
    assert params.opt_iterations == 3 and params.ignore_near_zero_dist_pairs == 0 and resp.depth_threshold == 1.0
