"""bench.py's reference arm on the CPU: one JSON line with the contract's keys, the CPU
restatement timed on a small workload (no GPU needed)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2", "--warmup", "0",
                          "--workload", "batch8"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.strip().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "vs_baseline",
              "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert line["config"]["workload"] == "batch_8_small_scenes"
    # the two steps together are one pass over the timed scenes (each scene once)
    assert line["pass_seconds"] == pytest.approx(2 * line["ms_per_step"] / 1e3)
    assert line["leaf_tests_per_pass"] > 0


def test_reference_arm_config_matches_the_gpu_arm():
    """Both arms describe the workload with the same config dict (the GPU arm builds it
    from the same Workload)."""
    sys.path.insert(0, ROOT)
    import bench
    a, b = bench.Workload("batch8"), bench.Workload("batch8")
    assert a.config == b.config and a.timed_ids == [0, 2, 4, 6]
    assert a.timed_scene_ids(0, 2) + a.timed_scene_ids(1, 2) == [0, 4, 2, 6]
