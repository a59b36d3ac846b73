"""Benchmark of the Nimbus hot path on B200.

One step = one large step of every run in the workload: Heun slow step,
boundary refresh and KW78 seed, N acoustic substeps (retained mass flux,
continuity + EOS, momentum, boundary closure), conservative WENO5 transport
of theta, qv, qc, qr, the Kessler step and the EOS re-projection.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ensemble_64|supercell_250m_256x256x80|...]

Prints one JSON line (rank 0).  `value` is device-timed whole-job throughput
in cell-updates/s (one cell advanced one large step) of the batched FP32 form
(member engine, CUDA graph) with the state resident in HBM.  `config` carries
the plain per-operation path on the same runs, the reference-precision form,
the error of the FP32 form against the FP64 oracle, and the serving numbers
(p50/p99 completion latency beside throughput).  `e2e` is the same metric
through the library's host-buffer API (every step writes each run's state
from pinned host memory and reads it back).  Under torchrun each rank
advances its own ensemble (members share nothing), so scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s"
WORKLOAD = "ensemble_64"
SINGLE_RUNS = ("supercell_1km_64x64x40", "supercell_250m_256x256x80", "supercell_100m_512x512x128")
# Algorithmic (compulsory) bytes per cell (FP32 fields, each read once and
# written once per named pass): acoustic substep 68 (reads u,v,w,rho,p,theta
# and three retained fluxes; writes u,v,w,rho,p and the fluxes), WENO5
# transport 20 + 8 per scalar, slow Heun 112, Kessler 40, EOS 12.
SUBSTEP_BYTES = 68
STEP_FIXED_BYTES = (20 + 8 * 4) + 112 + 40 + 12


def step_bytes(n_substeps: int) -> int:
    return SUBSTEP_BYTES * n_substeps + STEP_FIXED_BYTES


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--lanes", type=int, default=4,
                    help="parallel member groups inside the engine's step graph")
    ap.add_argument("--e2e-groups", type=int, default=8,
                    help="engines (each on its own stream) the runs are split over for the end-to-end pass")
    ap.add_argument("--plain-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-single", action="store_true", help="skip the 250 m and 100 m single-run legs")
    ap.add_argument("--no-autotune", action="store_true", help="keep --lanes and the default kernel form")
    ap.add_argument("--pass-forms", default=None, metavar="CONTINUITY,MOMENTUM",
                    help="with --no-autotune: the acoustic passes' kernel forms, each one of "
                         "table, const, march, pair, bulk, cmarch")
    ap.add_argument("--scaling", choices=("weak", "strong"), default="weak",
                    help="weak: each rank its own ensemble; strong: one ensemble split over the ranks")
    ap.add_argument("--no-error", action="store_true")
    ap.add_argument("--no-relaxation", action="store_true")
    ap.add_argument("--no-output", action="store_true")
    ap.add_argument("--no-sgs", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=32)
    ap.add_argument("--error-seconds", type=float, default=600.0)
    ap.add_argument("--precision", choices=("fp32", "reference"), default="fp32",
                    help="fp32: FP32 stencils on the FP64 base state (the timed form); "
                         "reference: FP64 interior arithmetic, bit-exact to the CPU solver")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def workload_cases(name, rank=0, members=64, world=1, strong=False):
    """This rank's runs.  Weak scaling: every rank its own seeded ensemble.
    Strong scaling: one ensemble, its members split over the ranks by the
    greedy size-balanced placement (nimbus_b200.ensemble.shard)."""
    from nimbus_b200.ensemble import ensemble_cases, shard
    from nimbus_b200.initial import benchmark_case

    if name == "ensemble_64":
        if strong:
            cases = ensemble_cases(members, seed=2026)
            return [cases[i] for i in shard(cases, world, rank)]
        return ensemble_cases(members, seed=2026 + 1000 * rank)
    case = benchmark_case(name)
    case.member = rank
    case.seed = case.seed + 1000 * rank
    return [case]


# ---------------------------------------------------------------------------
# The reference CPU path: the reference solver's own objects (oracle/_ref,
# built from its sources) assembled into one large step, on a bounded sample.
# ---------------------------------------------------------------------------
def sample_case(case):
    from nimbus_b200.initial import Case

    nx, ny = min(case.nx, 96), min(case.ny, 96)
    return Case(nx, ny, case.nz, case.dx, case.dy, case.dz, case.dt, substeps=case.substeps,
                noise_amp=case.noise_amp, seed=case.seed, bubble_rh=case.bubble_rh, bubble_rz=case.bubble_rz,
                bubble_zc=case.bubble_zc, bubble_amp=case.bubble_amp, bc=case.bc, member=case.member)


def reference_step_runner(case, threads):
    """(step_fn, kind, cores, n_substeps): one large step of the reference CPU
    path on `case`'s grid (the restatement when the reference is not built)."""
    import oracle
    from nimbus_b200.initial import initial_state
    from nimbus_b200.run import substeps_for

    st, base = initial_state(case)
    n = substeps_for(case, st, base)
    grid = (case.dx, case.dy, case.dz)
    if oracle.reference_available():
        impl = oracle.ReferenceHarness(threads=threads)
        kind, cores = "reference", impl.threads
    else:
        impl = oracle.Restatement("f32")
        kind, cores = "port", 1

    def step():
        impl.large_step(st, base, grid, case.dt, n, case.bc)

    return step, kind, cores, n


REF_CLI = ROOT / "oracle" / "_ref" / "nimbus_sim_ref"
REF_CLI_TEMPLATE = ROOT / "oracle" / "configs" / "supercell_1km_64x64x40.yaml"


def reference_cli_run(case, steps, warmup, threads):
    """The reference solver's own command-line program (built from its sources
    into oracle/_ref) run headless on the host cores, the stock CPU path: the
    1 km supercell preset (oracle/configs/) with this run's grid, spacing, dt
    and requested substeps, `warmup` untimed then `steps` timed large steps;
    returns (avg_step_ms, acoustic substeps after the scheme's promotion, log
    lines).  Its [PERF SUMMARY] times whole model steps excluding file output."""
    import re

    text = REF_CLI_TEMPLATE.read_text()
    repl = {"nx": case.nx, "ny": case.ny, "nz": case.nz, "dx": case.dx, "dy": case.dy, "dz": case.dz,
            "ztop": case.dz * case.nz, "dt_large": case.dt, "acoustic_substeps": max(case.substeps, 1),
            "warmup_steps": warmup, "center_x_m": 0.5 * case.nx * case.dx, "center_y_m": 0.5 * case.ny * case.dy}
    for key, val in repl.items():
        text = re.sub(rf"^(\s*{key}:)\s*\S+", rf"\g<1> {val}", text, count=1, flags=re.M)
    with tempfile.TemporaryDirectory() as tmp:
        cfg = Path(tmp) / "run.yaml"
        cfg.write_text(text)
        out = Path(tmp) / "out"
        out.mkdir()
        cmd = [str(REF_CLI), "--config", str(cfg), "--headless", "--timing", "--threads", str(threads),
               "--write-every=0", f"--outdir={out}", "--guard-mode", "sanitize",
               "--duration", str(int(math.ceil(case.dt * (steps + warmup))))]
        proc = subprocess.run(cmd, capture_output=True, text=True, cwd=tmp, timeout=1800)
    log = proc.stdout + proc.stderr
    m = re.search(r"\[PERF SUMMARY\].*?avg_step_ms=([0-9.eE+-]+)", log)
    if proc.returncode != 0 or not m:
        raise RuntimeError("reference CLI run failed: " + log[-400:])
    promoted = re.search(r"promoting to (\d+)", log)
    n = int(promoted.group(1)) if promoted else max(case.substeps, 1)
    return float(m.group(1)), n, log


def cpu_baseline(cases, budget_s=12.0):
    """The reference's stock CPU path (its own program, all host threads) on
    the workload's median run; the reference objects through the harness when
    the program was not built."""
    mid = sorted(cases, key=lambda c: c.cells)[len(cases) // 2]
    threads = os.cpu_count()
    if REF_CLI.exists():
        steps = 20
        ms, n, _ = reference_cli_run(mid, steps, 5, threads)
        return {"value": mid.cells / (ms / 1e3), "unit": METRIC, "cores": threads, "kind": "reference",
                "sample": f"{steps} timed large steps (after 5 warm-up steps) of the workload's median run "
                          f"({mid.nx}x{mid.ny}x{mid.nz}, N={n}) in the reference's own program, headless, "
                          f"on {threads} host threads: {ms:.1f} ms per step"}
    sc = sample_case(mid)
    step, kind, cores, n = reference_step_runner(sc, threads)
    step()  # warm-up
    t0 = time.perf_counter()
    steps = 0
    while True:
        step()
        steps += 1
        if time.perf_counter() - t0 > budget_s or steps >= 50:
            break
    el = time.perf_counter() - t0
    return {"value": sc.cells * steps / el, "unit": METRIC, "cores": cores, "kind": kind,
            "sample": f"{steps} large steps of a {sc.nx}x{sc.ny}x{sc.nz} grid (the workload's median run, "
                      f"N={n} acoustic substeps, full step incl. slow Heun, transport, Kessler, EOS), "
                      f"{el:.1f} s on {cores} host threads"}


def run_reference_arm(args):
    """The reference's own CPU implementation of the path on the host cores:
    its stock command-line program (headless, --timing) on the workload's
    median run, every host thread, args.warmup untimed then args.steps timed
    large steps; beside it, the same grid through the reference objects the
    parity harness drives (the hot path alone, without the runtime around it).
    Without the built program the harness rate is the line's value."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    cases = workload_cases(args.workload, 0, args.members)
    mid = sorted(cases, key=lambda c: c.cells)[len(cases) // 2]
    threads = os.cpu_count()
    # the hot path alone, through the reference's objects (bounded sample)
    sc = sample_case(mid)
    step, kind, cores, n = reference_step_runner(sc, threads)
    for _ in range(min(args.warmup, 3)):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    harness_value = sc.cells * args.steps / (time.perf_counter() - t0)
    harness = {"value": harness_value, "grid": [sc.nx, sc.ny, sc.nz], "acoustic_substeps": n, "cores": cores,
               "path": "slow Heun, boundary refresh, acoustic loop, transport, Kessler, EOS from the reference "
                       "solver's objects (oracle/_ref harness)"}
    value, ms, grid, path, n_used = harness_value, 1e3 * sc.cells / harness_value, [sc.nx, sc.ny, sc.nz], \
        harness["path"], n
    sample = (f"each step: one large step of a {sc.nx}x{sc.ny}x{sc.nz} grid through the reference's objects "
              f"(the workload's median run, capped at 96x96 columns)")
    cli = None
    if REF_CLI.exists():
        ms, n_used, _ = reference_cli_run(mid, args.steps, max(args.warmup, 3), threads)
        value, grid = mid.cells / (ms / 1e3), list(mid.shape)
        path = ("the reference's stock CLI (nimbus_sim built from its sources), headless, --timing, "
                "--guard-mode sanitize; [PERF SUMMARY] avg_step_ms after its warm-up steps")
        sample = (f"{args.steps} timed large steps of the workload's median run ({mid.nx}x{mid.ny}x{mid.nz}, "
                  f"dx {mid.dx:g} m, dt {mid.dt:g} s, N={n_used}) in the reference's own program")
        cli = {"value": value, "avg_step_ms": ms, "grid": grid, "acoustic_substeps": n_used, "threads": threads}
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 arithmetic, f32 storage",
        "data": "synthetic (the reference's parametric supercell preset with this run's grid)" if cli else
                "synthetic (seeded WK82 supercell initial states)",
        "config": {"workload": args.workload, "sample_grid": grid, "acoustic_substeps": n_used, "scalars": 4,
                   "path": path, "per_cell_rate": "cell-updates/s of one run: the ensemble's runs are independent "
                   "and the reference advances one run per process", "reference_cli": cli,
                   "reference_objects": harness},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows)}


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


# ---------------------------------------------------------------------------
# Our arm.
# ---------------------------------------------------------------------------
def time_on_stream(torch, stream, fn, steps):
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        fn()
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end)


def error_study(ctx, seconds):
    """FP32 form and reference-precision form on the device against the FP64
    oracle, supercell_1km_64x64x40 (dt 6 s) for `seconds` of model time."""
    import numpy as np

    import oracle
    from nimbus_b200 import cuda
    from nimbus_b200.initial import benchmark_case, initial_state
    from nimbus_b200.run import EngineRun, substeps_for

    case = benchmark_case("supercell_1km_64x64x40")
    st, base = initial_state(case)
    n = substeps_for(case, st, base)
    steps = int(round(seconds / case.dt))
    o64 = oracle.Restatement("f64")
    ref = {k: v.astype(np.float64) for k, v in st.items()}
    t0 = time.perf_counter()
    for _ in range(steps):
        o64.large_step(ref, base, (case.dx, case.dy, case.dz), case.dt, n, case.bc)
    oracle_s = time.perf_counter() - t0
    theta0 = base["theta0"][None, None, :]
    out = {"workload": "supercell_1km_64x64x40", "model_seconds": steps * case.dt, "steps": steps,
           "acoustic_substeps": n, "oracle": "FP64 restatement (FP64 storage and arithmetic)",
           "oracle_seconds": oracle_s, "metric": "relative L2 (max abs) per field; theta' = theta - theta0(z)"}
    for name, prec in (("fp32", cuda.PRECISION_FP32), ("reference_precision", cuda.PRECISION_REFERENCE)):
        run = EngineRun(ctx, prec)
        mid = run.admit(case, st, base)
        run.step(steps)
        got = run.read(mid)
        run.close()
        fields = {}
        for k in ("u", "v", "w", "theta", "qv", "p", "rho"):
            a = got[k].astype(np.float64)
            b = ref[k]
            if k == "theta":
                a, b = a - theta0, b - theta0
            den = float(np.linalg.norm(b))
            fields["theta'" if k == "theta" else k] = {
                "rel_l2": float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b)),
                "max_abs": float(np.abs(a - b).max())}
        out[name] = fields
    return out


def relaxation_study(ctx, device):
    """The end-of-step sponge (nimbus_cuda_state_relaxation, the next row
    after the large step) on one 512x512x80 level (four fields of 84 MB, larger
    than L2) with the reference's default sponge: device-timed, against the
    HBM roofline.  Algorithmic bytes: 16 read + 16 written per cell the sponge
    touches (upper levels, lid levels, lateral band); untouched cells move
    nothing."""
    import numpy as np
    import torch

    from nimbus_b200 import cuda
    from nimbus_b200.initial import Case, initial_state
    from nimbus_b200.sponge import SpongeConfig, build_profiles

    case = Case(512, 512, 80, 500.0, 500.0, 20000.0 / 80, 3.0, seed=11)
    st, base = initial_state(case)
    P = build_profiles(SpongeConfig(wind=(0.0, 0.0, 5.0, 2.0, 15.0, 6.0)), case.nz, case.dz, base["theta0"])
    dev = {k: torch.from_numpy(np.ascontiguousarray(st[k])).to(f"cuda:{device}") for k in ("u", "v", "w", "theta")}
    args = cuda.state_relaxation_args(dev, P, case.dt, memory=cuda.MEMORY_DEVICE)
    on = (P.alpha > 0) | (P.upper_w_alpha > 0) | (P.w_only_alpha > 0)
    i = np.arange(case.nx)[:, None]
    j = np.arange(case.ny)[None, :]
    band = np.minimum(np.minimum(i, case.nx - 1 - i), np.minimum(j, case.ny - 1 - j)) < len(P.lateral_alpha)
    touched = int(on.sum()) * case.nx * case.ny + int(band.sum()) * int((~on).sum())
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{device}")
    for _ in range(3):
        ctx.check(ctx.state_relaxation(args))
    launches = 20
    ms = time_on_stream(torch, stream, lambda: ctx.check(ctx.state_relaxation(args)), launches) / launches
    ctx.synchronize()
    peak, kind = load_peaks()
    achieved = 32.0 * touched / (ms / 1e3) / 1e9
    return {"grid": list(case.shape), "cells": case.cells, "cells_touched": touched,
            "ms_per_call": ms, "achieved_gbs": achieved, "peak_gbs": peak, "frac": achieved / peak,
            "peak_kind": kind, "algorithmic_bytes_per_touched_cell": 32,
            "note": "includes the host forming the per-level factors and staging the tables each call"}


def output_study(ctx, device):
    """Device-side output of one 512x512x80 level (84 MB per field, larger
    than L2): the cell-centre kernel (nimbus_cuda_cell_centre_velocity)
    device-timed against the HBM roofline, 24 algorithmic bytes per cell
    (three face fields read once, three centre fields written); a whole
    history frame (nimbus_cuda_history_snapshot: the kernel and the copies of
    all nine fields into pinned host memory) device-timed against the host
    link; the nine npy files of one frame written by nimbus_history_write,
    wall-timed; and the reference's own interpolate_*_face_to_center and
    npy::write_3d on the same fields, on the host cores."""
    import shutil
    import tempfile

    import numpy as np
    import torch

    import oracle
    from nimbus_b200 import cuda
    from nimbus_b200.initial import Case, initial_state

    case = Case(512, 512, 80, 500.0, 500.0, 20000.0 / 80, 3.0, seed=13)
    st, _ = initial_state(case)
    dev = {k: torch.from_numpy(np.ascontiguousarray(st[k])).to(f"cuda:{device}") for k in cuda.HISTORY_FIELDS}
    centre = tuple(torch.empty_like(dev[k]) for k in "uvw")
    args = cuda.cell_centre_args(dev["u"], dev["v"], dev["w"], outputs=centre, memory=cuda.MEMORY_DEVICE)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{device}")
    for _ in range(3):
        ctx.check(ctx.cell_centre_velocity(args))
    launches = 20
    k_ms = time_on_stream(torch, stream, lambda: ctx.check(ctx.cell_centre_velocity(args)), launches) / launches
    peak, kind = load_peaks()
    achieved = 24.0 * case.cells / (k_ms / 1e3) / 1e9
    image = torch.empty(9 * case.cells, dtype=torch.float32).pin_memory().numpy()
    hargs = cuda.history_args(dev, cuda.HISTORY_CORE, image, case.shape)
    for _ in range(2):
        ctx.check(ctx.history_snapshot(hargs))
    frames = 5
    f_ms = time_on_stream(torch, stream, lambda: ctx.check(ctx.history_snapshot(hargs)), frames) / frames
    ctx.synchronize()
    frame_bytes = 36 * case.cells
    tmp = Path(tempfile.mkdtemp(prefix="nimbus_history_"))
    try:
        t0 = time.perf_counter()
        rc = cuda.history_write(image, cuda.HISTORY_CORE, case.shape, tmp, ctx.lib)
        write_s = time.perf_counter() - t0
        ref = None
        if oracle.reference_available():
            h = oracle.ReferenceHarness(os.cpu_count())
            host = {k: st[k] for k in "uvw"}
            h.cell_centre(host["u"], host["v"], host["w"])
            t0 = time.perf_counter()
            uc, vc, wc = h.cell_centre(host["u"], host["v"], host["w"])
            r_interp = time.perf_counter() - t0
            t0 = time.perf_counter()
            for k, a in zip(cuda.HISTORY_FIELDS, (uc, vc, wc, *[st[k] for k in cuda.HISTORY_FIELDS[3:]])):
                h.npy_write_3d(a, tmp / f"ref_{k}.npy")
            r_write = time.perf_counter() - t0
            ref = {"kind": "reference", "cores": h.threads, "interpolate_ms": 1e3 * r_interp,
                   "npy_write_s": r_write, "sample": "interpolate_u/v/w_face_to_center on the same three fields, "
                                                     "then npy::write_3d of the nine fields of one frame"}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return {"grid": list(case.shape), "cells": case.cells,
            "cell_centre": {"ms_per_call": k_ms, "achieved_gbs": achieved, "peak_gbs": peak,
                            "frac": achieved / peak, "peak_kind": kind, "algorithmic_bytes_per_cell": 24},
            "history_frame": {"fields": 9, "bytes": frame_bytes, "ms_per_frame": f_ms,
                              "d2h_gbs": frame_bytes / (f_ms / 1e3) / 1e9,
                              "path": "one centring launch + one device-to-host copy for the velocities and one per scalar, "
                                      "into pinned host memory"},
            "npy_write": {"status": cuda.STATUS_NAMES.get(rc, rc), "seconds": write_s,
                          "gbs": frame_bytes / write_s / 1e9, "target": "local temporary directory"},
            "reference_cpu": ref}


def sgs_study(ctx, device):
    """The Smagorinsky SGS path on one 512x512x80 level with rigid lateral
    walls (84 MB per field, larger than L2), reference precision: the fused
    closure (nimbus_cuda_smagorinsky_fused: eddy coefficients + stress and
    scalar diffusion tendencies, 92 algorithmic bytes per cell: u, v, w,
    theta, qv, rho read and nu_t, K_theta, K_q written by the coefficient
    pass, u, v, w, rho, nu_t, K_theta, K_q, theta, qv read and five rates
    written by the tendency pass), the stability limit
    (nimbus_cuda_sgs_stability, synchronous) and the SGS apply, each
    device-timed; the explicit SGS integration of a 3 s step with dt_sgs =
    1 s (three substeps: closure, stability, apply); and the reference's
    SmagorinskyScheme::compute on the same level on the host cores."""
    import numpy as np
    import torch

    import oracle
    from nimbus_b200 import cuda
    from nimbus_b200.initial import Case, cloudy_state
    from nimbus_b200.sgs import SgsConfig

    case = Case(512, 512, 80, 500.0, 500.0, 250.0, 3.0, seed=17, bc=(2, 2, 2, 2, 1, 0))
    st, base = cloudy_state(case, seed=17)
    rng = np.random.default_rng(17)
    for k in "uvw":
        st[k] = (st[k] + rng.standard_normal(case.shape).astype(np.float32)).astype(np.float32)
    cfg = SgsConfig.from_bc(case.bc, dt_sgs=1.0)
    dz = np.full(case.nz, case.dz)
    grid = (case.dx, case.dy, case.dz)
    dev = {k: torch.from_numpy(np.ascontiguousarray(st[k])).to(f"cuda:{device}")
           for k in ("u", "v", "w", "theta", "qv", "rho")}
    ctx.set_precision(cuda.PRECISION_REFERENCE)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{device}")
    closure = cuda.smagorinsky_args(dev, dz, grid, cfg, memory=cuda.MEMORY_DEVICE)
    for _ in range(3):
        ctx.check(ctx.smagorinsky_fused(closure))
    calls = 10
    c_ms = time_on_stream(torch, stream, lambda: ctx.check(ctx.smagorinsky_fused(closure)), calls) / calls
    ctx.synchronize()
    peak, kind = load_peaks()
    achieved = 92.0 * case.cells / (c_ms / 1e3) / 1e9
    # The FP32 form of the closure (same call on an FP32-precision context).
    ctx.set_precision(cuda.PRECISION_FP32)
    ctx.check(ctx.smagorinsky_fused(closure))
    f_ms = time_on_stream(torch, stream, lambda: ctx.check(ctx.smagorinsky_fused(closure)), calls) / calls
    ctx.synchronize()
    ctx.set_precision(cuda.PRECISION_REFERENCE)
    ctx.check(ctx.smagorinsky_fused(closure))
    ctx.synchronize()
    stab_args = cuda.smagorinsky_args(dev, dz, grid, cfg, rates={k: closure.outputs[k] for k in cuda.SGS_RATES},
                                      memory=cuda.MEMORY_DEVICE)
    ctx.sgs_stability(stab_args)
    t0 = time.perf_counter()
    for _ in range(3):
        limits = ctx.sgs_stability(stab_args)
    s_ms = 1e3 * (time.perf_counter() - t0) / 3
    state = {k: v.clone() for k, v in dev.items()}
    apply = cuda.sgs_apply_args(state, {k: closure.outputs[k] for k in cuda.SGS_RATES}, 1.0,
                                theta0=base["theta0"], memory=cuda.MEMORY_DEVICE)
    ctx.check(ctx.sgs_apply(apply))
    a_ms = time_on_stream(torch, stream, lambda: ctx.check(ctx.sgs_apply(apply)), calls) / calls
    step = cuda.sgs_step_args(state, dz, grid, cfg, case.dt, theta0=base["theta0"])
    ctx.sgs_step(step)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    substeps, _ = ctx.sgs_step(step)
    torch.cuda.synchronize()
    step_ms = 1e3 * (time.perf_counter() - t0)
    ref = None
    if oracle.reference_available():
        h = oracle.ReferenceHarness(os.cpu_count())
        t0 = time.perf_counter()
        h.smagorinsky(st, dz, grid, cfg)
        r_s = time.perf_counter() - t0
        ref = {"kind": "reference", "cores": h.threads, "closure_s": r_s,
               "sample": "SmagorinskyScheme::compute (coefficients + momentum, theta, qv tendencies) on the same "
                         "512x512x80 level, one call"}
    return {"grid": list(case.shape), "cells": case.cells, "precision": "reference (FP64 arithmetic, FP32 storage)",
            "closure": {"ms_per_call": c_ms, "achieved_gbs": achieved, "peak_gbs": peak, "frac": achieved / peak,
                        "peak_kind": kind, "algorithmic_bytes_per_cell": 92},
            "closure_fp32": {"ms_per_call": f_ms, "achieved_gbs": 92.0 * case.cells / (f_ms / 1e3) / 1e9,
                             "frac": 92.0 * case.cells / (f_ms / 1e3) / 1e9 / peak},
            "stability": {"ms_per_call": s_ms, "limit_s": limits["maximum"],
                          "note": "wall time incl. one host synchronisation; slab sums are serial per x-slab"},
            "apply": {"ms_per_call": a_ms, "algorithmic_bytes_per_cell": 60},
            "sgs_step": {"dt_s": case.dt, "dt_sgs_s": cfg.dt_sgs, "substeps": substeps, "ms": step_ms},
            "reference_cpu": ref}


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from nimbus_b200 import cuda
    from nimbus_b200.initial import initial_state
    from nimbus_b200.run import EngineRun, HostPipeline, ResidentRun, substeps_for

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    device = local if world > 1 else 0
    torch.cuda.set_device(device)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world > 1:
            t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    strong = args.scaling == "strong" and args.workload == "ensemble_64"
    cases = workload_cases(args.workload, rank, args.members, world, strong)
    prepared = [initial_state(c) for c in cases]
    subs = [substeps_for(c, *p) for c, p in zip(cases, prepared)]
    cells = sum(c.cells for c in cases)
    ctx = cuda.Context(device)
    precision = cuda.PRECISION_FP32 if args.precision == "fp32" else cuda.PRECISION_REFERENCE
    other = cuda.PRECISION_REFERENCE if precision == cuda.PRECISION_FP32 else cuda.PRECISION_FP32
    # ---- batched form: every run resident in one engine, CUDA graph ----
    run = EngineRun(ctx, precision, lanes=args.lanes)
    for c, (st, base), n in zip(cases, prepared, subs):
        run.admit(c, st, base)  # substep count re-derived before every step
    # The engine autotuner picks lanes and the acoustic kernel form on these
    # runs (their states are restored afterwards); --lanes fixes the lanes.
    tuned = None
    if not args.no_autotune:
        ctx.set_precision(precision)
        tuned = run.engine.autotune(steps=2)
    elif args.pass_forms:
        names = {"table": cuda.ACOUSTIC_TABLE, "const": cuda.ACOUSTIC_CONST, "march": cuda.ACOUSTIC_MARCH,
                 "pair": cuda.ACOUSTIC_PAIR, "bulk": cuda.ACOUSTIC_BULK, "cmarch": cuda.ACOUSTIC_CMARCH}
        cont, mom = (names[f.strip()] for f in args.pass_forms.split(","))
        run.engine.set_pass_forms(cont, mom)
    stream = torch.cuda.ExternalStream(run.engine.stream, device=f"cuda:{device}")
    for _ in range(max(args.warmup, 3)):
        run.step(1)
    ctx.synchronize()
    lanes_used = run.engine.lanes  # the lanes the built table uses
    forms_used = [cuda.ACOUSTIC_FORM_NAMES[f] for f in run.engine.pass_forms]
    barrier()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    with ClockSampler(device) as clocks:
        ms = time_on_stream(torch, stream, lambda: run.step(1), args.steps)
    run.engine.synchronize()
    launches = ctx.kernel_launches - launches0
    barrier()
    ms = max_over_ranks(ms)
    clock = clocks.summary()
    if strong:  # the whole ensemble, whichever rank holds a member
        from nimbus_b200.ensemble import ensemble_cases
        total_cells = sum(c.cells for c in ensemble_cases(args.members, seed=2026))
    else:
        total_cells = cells * world
    value = total_cells * args.steps / (ms / 1e3)
    bytes_per_step = sum(c.cells * step_bytes(n) for c, n in zip(cases, subs))

    # ---- per-kernel device time (eager launches bracketed by events), one
    # lane so that no two launches share the GPU ----
    run.engine.set_lanes(1)
    run.step(1)
    ctx.synchronize()
    ctx.set_kernel_timing(True)
    for _ in range(args.steps):
        run.step(1)
    timing = ctx.kernel_timing()
    ctx.set_kernel_timing(False)
    run.engine.set_lanes(lanes_used)
    total_kernel_ms = sum(v[1] for v in timing.values())
    shares = {k: round(v[1] / total_kernel_ms, 4) for k, v in timing.items()} if total_kernel_ms else {}
    sub_ms = timing["acoustic_substep"][1] + timing["acoustic_momentum"][1]
    sub_launches = timing["acoustic_substep"][0]
    sub_bytes = sum(c.cells * n for c, n in zip(cases, subs)) * SUBSTEP_BYTES * args.steps
    achieved = sub_bytes / (sub_ms / 1e3) / 1e9 if sub_ms else None
    peak, peak_kind = load_peaks()
    # Measured DRAM bytes per cell-substep of the continuity + momentum pair
    # (ncu, profiles/), scaled to this workload's average substep.
    per_cell = load_traffic().get(args.workload, {}).get("acoustic_substep_dram_bytes_per_cell")
    cells_per_substep = sum(c.cells * n for c, n in zip(cases, subs)) / max(subs)
    traffic = per_cell * cells_per_substep if per_cell else None
    step_gbs = bytes_per_step * args.steps / (ms / 1e3) / 1e9

    # ---- the other precision, same runs ----
    ctx.set_precision(other)
    run.precision = other
    for _ in range(2):
        run.step(1)
    alt_ms = time_on_stream(torch, stream, lambda: run.step(1), args.steps) / args.steps
    run.precision = precision
    ctx.set_precision(precision)

    # ---- end to end through the host-buffer API ----
    run.close()
    e2e = None
    if args.e2e_steps > 0:
        pipe = HostPipeline(ctx, cases, prepared, groups=args.e2e_groups, precision=precision)
        pipe.step()
        barrier()
        t0 = time.perf_counter()
        pipe.step(args.e2e_steps)
        el = max_over_ranks(time.perf_counter() - t0)
        pipe.close()
        e2e = {"value": total_cells * args.e2e_steps / el, "unit": METRIC, "h2d_bytes_per_step": total_cells * 4 * 9,
               "d2h_bytes_per_step": total_cells * 4 * 9, "steps": args.e2e_steps,
               "api": "nimbus_cuda_engine_upload_image_async + nimbus_cuda_engine_step + "
                      "nimbus_cuda_engine_download_image_async, the runs split over "
                      f"{args.e2e_groups} engines on their own streams (each engine's nine prognostic fields of "
                      "every run in one pinned host block, one copy each way per step, stream-ordered, so one "
                      "group's copies overlap another group's step)"}

    # ---- plain path: each run alone, one C-ABI call per operation ----
    plain = None
    if not args.no_plain:
        ctx.set_substep_form(cuda.SUBSTEP_SPLIT)
        runs = [ResidentRun(ctx, c, st, base, device=f"cuda:{device}", precision=precision, autotune=False)
                for c, (st, base) in zip(cases, prepared)]

        def plain_step():
            for r in runs:
                r.step()

        plain_step()
        ctx.synchronize()
        ctx_stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{device}")
        p_ms = max_over_ranks(time_on_stream(torch, ctx_stream, plain_step, args.plain_steps))
        plain = {"value": total_cells * args.plain_steps / (p_ms / 1e3), "ms_per_step": p_ms / args.plain_steps,
                 "steps": args.plain_steps,
                 "path": "each run alone through the per-operation entry points (slow_step, acoustic_boundaries, "
                         "acoustic_batched, scalar_transport, kessler_step, eos_projection), host-enqueued launches"}
        plain["batched_over_plain"] = value / plain["value"]
        del runs
        torch.cuda.empty_cache()
        ctx.set_substep_form(cuda.SUBSTEP_AUTO)

    serving = None
    single = None
    error = None
    cpu = None
    relaxation = None
    output = None
    sgs = None
    if rank == 0 and world == 1:
        if not args.no_relaxation:
            relaxation = relaxation_study(ctx, device)
        if not args.no_output:
            output = output_study(ctx, device)
        if not args.no_sgs:
            sgs = sgs_study(ctx, device)
            ctx.set_precision(precision)
        if not args.no_serving:
            serving = serving_study(ctx, args, precision)
        if not args.no_single:
            single = single_run_study(ctx, args, precision)
        if not args.no_error:
            error = error_study(ctx, args.error_seconds)
        if not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline(cases)
            except Exception as exc:  # the baseline is reported, never required
                cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "unavailable", "sample": str(exc)}

    if rank == 0:
        nsub = sorted(set(subs))
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if strong else "weak",
            "vs_baseline": None,
            "dtype": "f32 (f64 only in the per-level base-state data and out-of-range EOS fallbacks)"
            if precision == cuda.PRECISION_FP32 else "f64 arithmetic, f32 storage",
            "data": "synthetic (seeded WK82 supercells: analytic sounding, cos^2 bubble, theta noise)",
            "config": {
                "workload": args.workload, "runs_per_gpu": len(cases), "cells_per_gpu": cells,
                "grids": "ragged: %d distinct shapes %s..%s" % (len({c.shape for c in cases}),
                                                                min(c.shape for c in cases),
                                                                max(c.shape for c in cases)),
                "acoustic_substeps": nsub, "scalars": 4,
                "path": "full large step: slow Heun, boundary refresh + KW78 seed, N split substeps "
                        "(mass flux, continuity+EOS, momentum, boundaries), WENO5 transport, Kessler, EOS",
                "form": f"batched member engine: the runs in {lanes_used} size-balanced lanes (parallel branches of "
                        "one CUDA graph), one launch per phase per lane",
                "lanes": lanes_used,
                "pass_forms": {"continuity": forms_used[0], "momentum": forms_used[1]},
                "autotune": tuned,
                "precision": args.precision,
                "precision_modes": {
                    args.precision: {"value": value, "ms_per_step": ms / args.steps},
                    ("reference" if args.precision == "fp32" else "fp32"): {
                        "value": total_cells * 1e3 / alt_ms if world == 1 else None, "ms_per_step": alt_ms}},
                "plain": plain,
                "serving": serving,
                "single_runs": single,
                "error_vs_fp64": error,
                "state_relaxation": relaxation,
                "output": output,
                "smagorinsky_sgs": sgs,
                "parallelism": (f"{world} GPU(s) sharing one {args.members}-member ensemble, members placed by "
                                "size-balanced greedy partition (no data-path collective)") if strong else
                               f"{world} GPU(s), each with its own independent ensemble (no collective)",
                "l2": "inputs larger than L2 (%.1f GB resident per GPU)" % (cells * 4 * 40 / 1e9),
                "algorithmic_bytes_per_step": bytes_per_step,
                "effective_step_bandwidth_gbs": step_gbs},
            "roofline": {"bound": "hbm", "kernel": "acoustic substep (continuity+EOS and momentum kernels)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "peak_kind": peak_kind,
                         "traffic": traffic, "traffic_unit": "DRAM bytes per substep (both kernels, all members)",
                         "algorithmic_bytes_per_substep": SUBSTEP_BYTES * cells_per_substep,
                         "algorithmic_bytes_per_cell_substep": SUBSTEP_BYTES,
                         "launches": sub_launches, "substep_ms_total": sub_ms,
                         "whole_step_frac": step_gbs / peak, "kernel_shares": shares},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clock,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


# Algorithmic bytes per cell of each kernel family's pass (see SUBSTEP_BYTES);
# the acoustic pair's per substep.
FAMILY_BYTES = {"acoustic": SUBSTEP_BYTES, "transport": 20 + 8 * 4, "slow": 112, "microphysics": 40 + 12}


def single_run_study(ctx, args, precision):
    """The single-run configurations: the 250 m supercell (256x256x80, dt
    1.5 s, 8 substeps) and the 100 m supercell (512x512x128, dt 0.6 s, 10
    substeps), each as one member of the engine (graph, its kernel forms
    autotuned on the grid) and on the plain
    per-operation path, with every kernel family's event-timed duration and
    HBM rate (its algorithmic bytes over that duration, against the measured
    copy rate).  The reference CPU solver runs one large step of the 250 m
    grid on the host cores; the 100 m grid's CPU time is that rate scaled by
    cells and algorithmic bytes per cell (labelled as an extrapolation)."""
    import torch

    from nimbus_b200 import cuda
    from nimbus_b200.initial import benchmark_case, initial_state
    from nimbus_b200.run import EngineRun, ResidentRun

    peak, peak_kind = load_peaks()
    out = {}
    cpu_rate = None
    for name in ("supercell_250m_256x256x80", "supercell_100m_512x512x128"):
        case = benchmark_case(name)
        st, base = initial_state(case)
        run = EngineRun(ctx, precision)
        mid = run.admit(case, st, base)
        ctx.set_precision(precision)
        tuned = run.engine.autotune(steps=2)  # the kernel forms for this grid (states restored)
        stream = torch.cuda.ExternalStream(run.engine.stream)
        for _ in range(3):
            run.step(1)
        ctx.synchronize()
        steps = max(3, min(args.steps, 10))
        ms = time_on_stream(torch, stream, lambda: run.step(1), steps) / steps
        n = run.substeps(mid)
        ctx.set_kernel_timing(True)
        for _ in range(steps):
            run.step(1)
        timing = ctx.kernel_timing()
        ctx.set_kernel_timing(False)
        run.close()
        fam_ms = {k: v[1] / steps for k, v in timing.items() if v[1] > 0}
        groups = {"acoustic": ("acoustic_substep", "acoustic_momentum"),
                  "transport": ("transport_faces", "transport_limiter", "transport_update"),
                  "slow": ("slow",), "microphysics": ("microphysics",)}
        kernels = {}
        for g, fams in groups.items():
            t = sum(fam_ms.get(f, 0.0) for f in fams)
            nbytes = case.cells * FAMILY_BYTES[g] * (n if g == "acoustic" else 1)
            if t > 0:
                gbs = nbytes / (t / 1e3) / 1e9
                kernels[g] = {"ms_per_step": round(t, 4), "algorithmic_gb": round(nbytes / 1e9, 4),
                              "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
        kernels["acoustic_boundary"] = {"ms_per_step": round(fam_ms.get("acoustic_boundary", 0.0), 4)}
        # plain path: one C-ABI call per operation
        ctx.set_substep_form(cuda.SUBSTEP_SPLIT)
        plain = ResidentRun(ctx, case, {k: v.copy() for k, v in st.items()}, base, precision=precision,
                            autotune=False)
        plain.step()
        ctx.synchronize()
        cstream = torch.cuda.ExternalStream(ctx.stream)
        p_ms = time_on_stream(torch, cstream, plain.step, steps) / steps
        del plain
        torch.cuda.empty_cache()
        ctx.set_substep_form(cuda.SUBSTEP_AUTO)
        bytes_step = case.cells * step_bytes(n)
        entry = {"grid": list(case.shape), "dt_s": case.dt, "acoustic_substeps": n, "cells": case.cells,
                 "engine": {"ms_per_step": round(ms, 4), "value": case.cells / (ms / 1e3), "unit": METRIC,
                            "whole_step_gbs": round(bytes_step / (ms / 1e3) / 1e9, 1),
                            "whole_step_frac": round(bytes_step / (ms / 1e3) / 1e9 / peak, 4)},
                 "plain": {"ms_per_step": round(p_ms, 4), "value": case.cells / (p_ms / 1e3)},
                 "kernels": kernels, "peak_gbs": peak, "peak_kind": peak_kind,
                 "forms": {"continuity": tuned["continuity_form"], "momentum": tuned["momentum_form"]}}
        if not args.no_cpu_baseline:
            if cpu_rate is None:
                step, kind, cores, n_ref = reference_step_runner(case, os.cpu_count())
                t0 = time.perf_counter()
                step()
                el = time.perf_counter() - t0
                cpu_rate = (case.cells / el, kind, cores, el, case.cells * step_bytes(n_ref))
                entry["cpu_reference"] = {"value": cpu_rate[0], "unit": METRIC, "kind": kind, "cores": cores,
                                          "sample": f"one large step of this grid (N={n_ref}), {el:.1f} s"}
            else:
                rate, kind, cores, _, ref_bytes = cpu_rate
                per_byte = rate * step_bytes(8) / step_bytes(n)
                entry["cpu_reference"] = {"value": per_byte, "unit": METRIC, "kind": kind, "cores": cores,
                                          "sample": "extrapolated from the 250 m grid's measured step: that "
                                                    "rate scaled by algorithmic bytes per cell (N=8 there, "
                                                    f"N={n} here); not run on this grid"}
        out[name] = entry
    return out


def serving_study(ctx, args, precision):
    """Poisson streams of increasing rate (4, 16 and 64 requests per second,
    the last past saturation) and a burst of the same requests: continuous
    batching in the engine against running them one by one on the plain path.
    Initial states are prepared (and pinned) before each stream starts."""
    import torch

    from nimbus_b200.ensemble import request_stream
    from nimbus_b200.initial import initial_state
    from nimbus_b200.serve import Server, serve_one_by_one, summarize

    def pinned(st):
        return {k: torch.from_numpy(v).pin_memory().numpy() for k, v in st.items()}

    out = {}
    streams = [("poisson_%d_per_s" % rate, rate, False) for rate in (4, 16, 64)] + [("burst", 4, True)]
    for label, rate, burst in streams:
        reqs = request_stream(args.serving_requests, rate_per_s=float(rate), seed=7, burst=burst)
        prepared = {}
        for r in reqs:
            st, base = initial_state(r.case)
            prepared[r.rid] = (pinned(st), base)
        server = Server(ctx, precision)
        done, span = server.serve(reqs, prepared)
        builds = server.run.engine.graph_builds()
        server.close()
        plain, p_span = serve_one_by_one(ctx, reqs, precision, prepared)
        batched = summarize(done, span)
        batched["graph_instantiations"], batched["graph_updates"] = builds
        out[label] = {"batched": batched, "one_by_one_plain": summarize(plain, p_span)}
    out["requests"] = ("%d runs per stream, grids log-uniform 32x32x40..256x256x80, durations U(60,600) s at dt 3 s, "
                       "seeded" % args.serving_requests)
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
