"""Builds the in-tree CUDA backend library for sm_100a.

    python -m nimbus_b200.build

Produces nimbus_b200/lib/libnimbus_cuda.so from nimbus_b200/csrc with
`nvcc -gencode arch=compute_100a,code=sm_100a`, one object per translation
unit.  The reference-precision units are compiled with --fmad=false: the CPU
solver they match performs every multiply and add separately, and a
contracted FMA would change the rounding of stored values.  The FP32 form's
unit (fp32_*.cu) is compiled with --fmad=true.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "nimbus_cuda.h"]


def build(force: bool = False, verbose: bool = False) -> Path:
    LIB.mkdir(exist_ok=True)
    out = LIB / "libnimbus_cuda.so"
    newest = max(p.stat().st_mtime for p in sources())
    if out.exists() and not force and out.stat().st_mtime >= newest:
        return out
    obj_dir = LIB / "obj"
    obj_dir.mkdir(exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
    if verbose:
        common.append("-Xptxas=-v")
    jobs, objs = [], []
    for src in sorted(CSRC.glob("*.cu")):
        obj = obj_dir / (src.stem + ".o")
        # The FP32 form's unit contracts multiply-adds; every other unit keeps
        # the reference's uncontracted arithmetic.
        fmad = "--fmad=true" if src.name.startswith("fp32_") else "--fmad=false"
        cmd = [*common, fmad, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        jobs.append(subprocess.Popen(cmd))
        objs.append(obj)
    if any(j.wait() != 0 for j in jobs):
        raise subprocess.CalledProcessError(1, "nvcc")
    subprocess.run([nvcc(), *ARCH, "-shared", *[str(o) for o in objs], "-o", str(out)], check=True)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
