"""bench.py --impl reference on the host cores: the reference's own program
(oracle/_ref/nimbus_sim_ref, built from its sources) and the reference
objects on the workload's median run, reported as one JSON line in the
benchmark's metric; under torchrun only rank 0 runs and prints."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "oracle" / "_ref" / "nimbus_sim_ref"
HARNESS = ROOT / "oracle" / "_ref" / "libnimbus_ref_harness.so"

pytestmark = pytest.mark.skipif(not (CLI.exists() and HARNESS.exists()), reason="reference tools not built")


def _run(extra_env=None):
    env = dict(os.environ, **(extra_env or {}))
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        if not extra_env or k not in extra_env:
            env.pop(k, None)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_line_in_the_benchmark_metric():
    proc = _run()
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [l for l in proc.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, proc.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == line["unit"] == "cell-updates/s"
    assert line["higher_is_better"] is True
    assert line["value"] > 0
    assert line["config"]["workload"] == "ensemble_64"
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] >= 1 and cpu["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    proc = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert proc.returncode == 0, proc.stderr[-2000:]
    assert proc.stdout.strip() == ""
