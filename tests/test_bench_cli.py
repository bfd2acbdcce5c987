"""bench.py's reference arm (no GPU): one JSON line with the keys the bench contract names, timed
on the reference's own OpenMP build or on the oracle's serial restatement; under torchrun only
rank 0 prints."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BENCH = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
PORT_LIB = os.path.join(ROOT, "oracle", "_port", "liboracle.so")
KEYS = ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def run_arm(kind, env=None):
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--size", "32", "--steps", "3",
           "--warmup", "3", "--ref-cycles", "10", "--cpu-ref", kind]
    return subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300,
                          env=dict(os.environ, **(env or {})))


@pytest.mark.parametrize("kind,binary", [("reference", REF_BENCH), ("port", PORT_LIB)])
def test_reference_arm_line(kind, binary):
    if not os.path.exists(binary):
        pytest.skip(f"{binary} not built (make -C oracle ref port)")
    out = run_arm(kind)
    assert out.returncode == 0, out.stderr
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert all(k in d for k in KEYS), sorted(set(KEYS) - set(d))
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == kind and cb["value"] == d["value"] and cb["cores"] >= 1
    if kind == "port":
        assert cb["cores"] == 1
    # the reference's per-cycle sweep size: the solver's active window of the same problem
    sys.path.insert(0, ROOT)
    import bench
    import exaca_b200 as ex

    assert d["config"]["cells"] == ex.Problem.directional(32, 32, 32, **bench.WORKLOAD).geometry.active_size


def test_reference_arm_other_ranks_print_nothing():
    out = run_arm("auto", env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
