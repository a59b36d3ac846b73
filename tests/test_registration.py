"""The registration of the CUDA backend in the reference's program, checked
without a GPU: the registered tree carries exactly the patch, and the registered
program parses `--compute-backend=cuda`, builds the backend through its
factory and -- with no sm_100 device here -- falls back to its CPU backend
when fallback is allowed, or stops with the backend's own error when it is
not.  (Runs on the CUDA backend are in test_registered_program_gpu.py.)
"""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from tests.test_registered_program_gpu import PROGRAM, _config

ROOT = Path(__file__).resolve().parents[1]
PATCH = ROOT / "nimbus_b200" / "reference_backend" / "registration.patch"
TREE = ROOT / "nimbus_b200" / "reference_backend" / "_registered" / "tree"


def test_registration_patch_is_the_registered_trees_change():
    """The patched copy registered.mk built the program from carries exactly
    this patch (it reverses cleanly)."""
    if not (TREE / ".patched").exists() or shutil.which("patch") is None:
        pytest.skip("registered tree or patch(1) not available")
    files = sorted({m.group(1) for m in re.finditer(r"^\+\+\+ b/(\S+)", PATCH.read_text(), flags=re.M)})
    assert "src/compute/compute_backend.cpp" in files and "include/compute/backend_types.hpp" in files
    proc = subprocess.run(["patch", "-p1", "-R", "--dry-run", "-d", str(TREE)], input=PATCH.read_text(), text=True,
                          capture_output=True)
    assert proc.returncode == 0, proc.stdout + proc.stderr


def _cpu_host_run(tmp_path, strict):
    if not PROGRAM.exists():
        pytest.skip("registered program not built")
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present: the GPU tests cover the cuda runs")
    except ImportError:
        pass
    cfg = _config(tmp_path, "cuda", strict)
    out = tmp_path / "out"
    out.mkdir()
    cmd = [str(PROGRAM), "--config", str(cfg), "--headless", "--threads", "2", "--write-every=0", f"--outdir={out}",
           "--guard-mode", "sanitize", "--duration", "6", "--compute-backend=cuda"]
    return subprocess.run(cmd, capture_output=True, text=True, cwd=tmp_path, timeout=600)


def test_registered_program_falls_back_to_cpu_without_a_device(tmp_path):
    proc = _cpu_host_run(tmp_path, strict=False)
    log = proc.stdout + proc.stderr
    assert proc.returncode == 0, log[-2000:]
    assert "Requested backend 'cuda' failed to initialize: no sm_100 CUDA device" in log, log[-2000:]
    assert re.search(r"\[COMPUTE\] backend=cpu, requested=cuda, .*fallback=active", log), log[-2000:]


def test_registered_program_fails_closed_without_a_device_when_fallback_is_off(tmp_path):
    proc = _cpu_host_run(tmp_path, strict=True)
    log = proc.stdout + proc.stderr
    assert proc.returncode != 0
    assert "no sm_100 CUDA device" in log, log[-2000:]
