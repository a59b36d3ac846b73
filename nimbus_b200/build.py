"""Builds the in-tree CUDA backend library for sm_100a.

    python -m nimbus_b200.build

Produces nimbus_b200/lib/libnimbus_cuda.so from nimbus_b200/csrc with
`nvcc -gencode arch=compute_100a,code=sm_100a`, one object per translation
unit.  The reference-precision units are compiled with --fmad=false: the CPU
solver they match performs every multiply and add separately, and a
contracted FMA would change the rounding of stored values.  The FP32 form's
unit (fp32_*.cu) is compiled with --fmad=true.

Where the reference solver's headers are present it also builds
nimbus_b200/lib/libnimbus_reference_backend.so, the ComputeBackend adapter
(reference_backend/nimbus_compute_backend.cpp) that plugs this library into
the reference's own backend interface.
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


# The reference solver's source tree (its headers, for the ComputeBackend
# adapter): the directory NIMBUS_REFERENCE_DIR names; the adapter is skipped
# without it.
ADAPTER = PKG / "reference_backend" / "nimbus_compute_backend.cpp"


def reference_dir() -> Path | None:
    value = os.environ.get("NIMBUS_REFERENCE_DIR")
    return Path(value) if value else None


def build_reference_backend(force: bool = False) -> Path | None:
    """nimbus_b200/lib/libnimbus_reference_backend.so: the CUDA backend as a
    ComputeBackend of the reference solver, compiled against its headers and
    linked to libnimbus_cuda.so.  Skipped (None) without the reference tree
    (NIMBUS_REFERENCE_DIR)."""
    REFERENCE = reference_dir()
    if REFERENCE is None or not (REFERENCE / "include" / "compute" / "backend_interface.hpp").exists():
        return None
    out = LIB / "libnimbus_reference_backend.so"
    cuda_lib = LIB / "libnimbus_cuda.so"
    if out.exists() and not force and out.stat().st_mtime >= max(ADAPTER.stat().st_mtime, cuda_lib.stat().st_mtime):
        return out
    cxx = os.environ.get("CXX", "g++")
    subprocess.run([cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-w", "-I", str(REFERENCE / "include"),
                    "-I", str(REFERENCE / "src"), str(ADAPTER), "-o", str(out), "-L", str(LIB), "-lnimbus_cuda",
                    "-Wl,-rpath,$ORIGIN", "-Wl,--no-undefined"], check=True)
    return out


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
    build_reference_backend(force=True)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_reference_backend())
