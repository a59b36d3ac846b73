"""The reference's own program with the CUDA backend registered
(nimbus_b200/reference_backend/registration.patch, registered.mk): nimbus_sim
run as `--compute-backend=cuda` on the 1 km supercell preset (64x64x40,
Kessler, WENO5 transport, split-explicit acoustic loop on the flat C-grid).

The run is held to the reference's own accelerator qualification: with
NIMBUS_VALIDATE_PARITY=1 its runtime replays every sampled device dispatch on
its CPU path and compares the two with its parity tiers
(src/compute/parity_check.cpp, parity_comparison.cpp), printing
"[PARITY] RESULT: PASS" only when no record breached.  The log must show the
cuda backend active (not fallen back to the CPU backend); operators the
backend does not take run on the reference's CPU path, as the runtime's
default per-dispatch fallback allows.
"""
import os
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PROGRAM = ROOT / "nimbus_b200" / "reference_backend" / "_registered" / "nimbus_sim_cuda"
PRESET = ROOT / "oracle" / "configs" / "supercell_1km_64x64x40.yaml"

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not PROGRAM.exists(), reason="registered program not built")]


def _config(tmp_path, backend, strict=False):
    text = PRESET.read_text()
    extra = "\n    allow_fallback: false" if strict else ""
    text = re.sub(r"^(\s*backend:)\s*\S+", rf"\g<1> {backend}{extra}", text, count=1, flags=re.M)
    text = re.sub(r"^(\s*warmup_steps:)\s*\S+", r"\g<1> 2", text, count=1, flags=re.M)
    path = tmp_path / f"{backend}.yaml"
    path.write_text(text)
    return path


def _run(tmp_path, backend, parity, steps=10, strict=False):
    cfg = _config(tmp_path, backend, strict)
    out = tmp_path / f"out_{backend}_{int(parity)}"
    out.mkdir()
    env = dict(os.environ, NIMBUS_VALIDATE_PARITY="1" if parity else "0")
    cmd = [str(PROGRAM), "--config", str(cfg), "--headless", "--timing", "--threads", "8", "--write-every=0",
           f"--outdir={out}", "--guard-mode", "sanitize", "--duration", str(6 * steps),
           f"--compute-backend={backend}"]
    proc = subprocess.run(cmd, capture_output=True, text=True, cwd=tmp_path, env=env, timeout=900)
    log = proc.stdout + proc.stderr
    assert proc.returncode == 0, log[-3000:]
    return log


def test_reference_program_runs_on_the_cuda_backend_and_passes_its_parity_check(tmp_path):
    log = _run(tmp_path, "cuda", parity=True)
    assert re.search(r"\[COMPUTE\] backend=cuda, requested=cuda, .*fallback=off", log), log[-3000:]
    result = re.search(r"\[PARITY\] RESULT: (\w+) \((\d+) kernel-field-domain records, (\d+) samples", log)
    assert result, log[-3000:]
    kernels = set(re.findall(r"^\S*\s*\[PARITY\] (\w+)\s+\w+\s+(?:pointwise|stencil|microphys|mp-heating)", log,
                             flags=re.M))
    report = "\n".join(line for line in log.splitlines() if "[PARITY]" in line)
    print(report)
    assert result.group(1) == "PASS", report
    # The device dispatches the run took and the reference replayed.
    for k in ("acoustic_batched_cartesian_cgrid", "cartesian_cgrid_slow_tendencies"):
        assert k in kernels, report


def test_reference_program_cuda_backend_step_time(tmp_path):
    """The same program and workload on its CPU backend and on the CUDA
    backend (parity replay off): both complete; the step times are reported."""
    times = {}
    for backend in ("cpu", "cuda"):
        log = _run(tmp_path, backend, parity=False)
        m = re.search(r"\[PERF SUMMARY\].*?avg_step_ms=([0-9.eE+-]+)", log)
        assert m, log[-2000:]
        times[backend] = float(m.group(1))
    print(f"reference program, 64x64x40 supercell, avg_step_ms: {times}")
    assert all(t > 0 for t in times.values())


def test_reference_program_runs_on_the_cuda_backend_with_fallback_off(tmp_path):
    """allow_fallback: false -- every dispatch the runtime requires natively on
    an accelerator backend must be served (a declined one is an error): the
    run completes on the CUDA backend."""
    log = _run(tmp_path, "cuda", parity=False, steps=4, strict=True)
    assert re.search(r"\[COMPUTE\] backend=cuda, requested=cuda, .*fallback=off, fallback_allowed=off", log), \
        log[-3000:]
    assert re.search(r"\[PERF SUMMARY\].*avg_step_ms=", log), log[-2000:]
