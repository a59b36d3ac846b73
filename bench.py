"""Benchmark of the Nimbus hot path on B200: one large step = the
split-explicit acoustic loop (N substeps with boundary closure and retained
mass flux) + conservative WENO5 transport of theta, qv, qc, qr.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is device-timed whole-job throughput
in cell-updates/s (one cell advanced one large step) with the state resident
in HBM; `e2e` is the same metric through the reference-facing host-memory API
(every step stages its inputs from pinned host memory and reads its results
back).  Under torchrun each rank advances its own independent run (ensemble
members share nothing), so scaling is weak.
"""
from __future__ import annotations

import argparse
import json
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
WORKLOAD = "supercell_250m_256x256x80"
# Algorithmic (compulsory) bytes per cell: one acoustic substep reads
# u,v,w,rho,p,theta and the three retained mass fluxes and writes
# u,v,w,rho,p and the three mass fluxes (17 FP32 fields).
SUBSTEP_BYTES_PER_CELL = 68
TRANSPORT_BYTES_PER_CELL = lambda scalars: 20 + 8 * scalars  # noqa: E731


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--substep-form", choices=("auto", "fused", "split"), default="auto",
                    help="acoustic substep kernels: autotuned (default) or pinned (profiling runs pin the "
                         "form the plain run chose, since a profiler distorts the autotuner's timings)")
    ap.add_argument("--precision", choices=("fp32", "reference"), default="fp32",
                    help="fp32: FP32 stencils on the FP64 base state (the timed form); "
                         "reference: FP64 interior arithmetic, bit-exact to the CPU solver")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ---------------------------------------------------------------------------
# CPU baseline: the reference CPU solver (oracle/_ref, built from the
# reference's own sources) on a bounded sub-domain sample of the workload.
# ---------------------------------------------------------------------------
def sample_case(case):
    from nimbus_b200.initial import Case

    nx = min(case.nx, 128)
    ny = min(case.ny, 128)
    return Case(nx, ny, case.nz, case.dx, case.dy, case.dz, case.dt, substeps=case.substeps,
                noise_amp=case.noise_amp, seed=case.seed, bubble_rh=case.bubble_rh, bubble_rz=case.bubble_rz,
                bubble_zc=case.bubble_zc, bc=case.bc)


def reference_step_runner(case, threads):
    """Returns (step_fn, kind, cores, n_substeps): one large step of the
    reference CPU path on the sample grid."""
    import oracle
    from nimbus_b200.initial import initial_state, max_sound_speed, resolve_substep_count

    st, base = initial_state(case)
    n = resolve_substep_count(case.dt, max_sound_speed(st["p"], st["rho"], base), case.dx, case.dy, case.dz,
                              case.substeps)
    grid = (case.dx, case.dy, case.dz)
    if oracle.reference_available():
        ref = oracle.ReferenceHarness(threads=threads)
        kind, cores = "reference", ref.threads

        def step():
            out = ref.acoustic_loop(st, base["rho0"], base["p0"], case.dt, n, grid, case.bc)
            qs = [st[k] for k in ("theta", "qv", "qc", "qr")]
            ref.scalar_transport(qs, [0, 1, 1, 1], st["u"], st["v"], st["w"], st["rho"], out["rho_begin"],
                                 out["mfx"], out["mfy"], out["mfz"], case.dt, grid, top_open=case.bc[5] == 2)
    else:
        port = oracle.Restatement("f32")
        kind, cores = "port", 1

        def step():
            out = port.acoustic_loop(st, base["rho0"], base["p0"], case.dt, n, grid, case.bc)
            qs = [st[k] for k in ("theta", "qv", "qc", "qr")]
            port.scalar_transport(qs, [0, 1, 1, 1], st["rho"], out["rho_begin"], out["mfx"], out["mfy"], out["mfz"],
                                  case.dt, grid, top_open=case.bc[5] == 2)
    return step, kind, cores, n


def cpu_baseline(case, budget_s=12.0):
    sc = sample_case(case)
    step, kind, cores, n = reference_step_runner(sc, os.cpu_count())
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
            "sample": f"{steps} large steps of a {sc.nx}x{sc.ny}x{sc.nz} sub-domain of the workload "
                      f"(N={n} acoustic substeps + WENO5 transport of 4 scalars), {el:.1f} s on {cores} host threads"}


def run_reference_arm(args):
    rank, world, _ = dist_env()
    from nimbus_b200.initial import benchmark_case

    if rank != 0:
        return 0
    case = benchmark_case(args.workload)
    sc = sample_case(case)
    step, kind, cores, n = reference_step_runner(sc, os.cpu_count())
    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = sc.cells * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 arithmetic, f32 storage",
        "data": "synthetic (seeded WK82 supercell initial state)",
        "config": {"workload": args.workload, "sample_grid": [sc.nx, sc.ny, sc.nz], "acoustic_substeps": n,
                   "scalars": 4, "path": "acoustic loop + WENO5 transport (reference CPU solver)"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": kind,
                         "sample": f"each step: one large step of a {sc.nx}x{sc.ny}x{sc.nz} sub-domain"},
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


# ---------------------------------------------------------------------------
# Our arm.
# ---------------------------------------------------------------------------
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


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from nimbus_b200 import cuda
    from nimbus_b200.initial import benchmark_case
    from nimbus_b200.run import HostStepper, ResidentRun

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    device = local if world > 1 else 0
    torch.cuda.set_device(device)
    case = benchmark_case(args.workload)
    case.member = rank  # each rank advances its own ensemble member
    case.seed = case.seed + 1000 * rank
    ctx = cuda.Context(device)
    precision = cuda.PRECISION_FP32 if args.precision == "fp32" else cuda.PRECISION_REFERENCE
    other = cuda.PRECISION_REFERENCE if precision == cuda.PRECISION_FP32 else cuda.PRECISION_FP32
    form = {"auto": cuda.SUBSTEP_AUTO, "fused": cuda.SUBSTEP_FUSED, "split": cuda.SUBSTEP_SPLIT}[args.substep_form]
    ctx.set_substep_form(form)
    run = ResidentRun(ctx, case, device=f"cuda:{device}", precision=precision, autotune=form == cuda.SUBSTEP_AUTO)
    stream = run.torch_stream

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(max(args.warmup, 3)):
        run.step()
    stream.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            run.step()
        end.record(stream)
        end.synchronize()
    ctx.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches = ctx.kernel_launches - launches0
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    clock = clocks.summary()
    cells_total = case.cells * world
    value = cells_total * args.steps / (ms / 1e3)

    # Per-kernel device time over an identical pass with event bracketing.
    ctx.set_kernel_timing(True)
    for _ in range(args.steps):
        run.step()
    timing = ctx.kernel_timing()
    ctx.set_kernel_timing(False)
    n_sub = run.n_substeps
    launches_sub, total_sub = timing["acoustic_substep"]
    # One substep = the fused kernel, or the split form's two launches.
    substep_ms = (total_sub + timing["acoustic_momentum"][1]) / max(launches_sub, 1)
    achieved = SUBSTEP_BYTES_PER_CELL * case.cells / (substep_ms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    traffic = load_traffic().get(args.workload, {}).get("acoustic_substep_bytes_per_substep")
    total_ms = sum(v[1] for v in timing.values())
    shares = {k: round(v[1] / total_ms, 4) for k, v in timing.items()} if total_ms else {}

    # The other precision mode, same workload, device-timed (reported beside).
    alt = ResidentRun(ctx, case, device=f"cuda:{device}", precision=other, autotune=form == cuda.SUBSTEP_AUTO)
    for _ in range(3):
        alt.step()
    alt.torch_stream.synchronize()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(alt.torch_stream)
    for _ in range(args.steps):
        alt.step()
    a1.record(alt.torch_stream)
    a1.synchronize()
    alt_ms = a0.elapsed_time(a1) / args.steps
    del alt
    ctx.set_precision(precision)

    # End-to-end through the reference-facing host API (pinned host arrays).
    e2e = None
    if args.e2e_steps > 0:
        host = HostStepper(ctx, case, precision=precision)
        host.step()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            host.step()
        el = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([el], device=f"cuda:{device}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        h2d, d2h = host.bytes_per_step()
        e2e = {"value": cells_total * args.e2e_steps / el, "unit": METRIC, "h2d_bytes_per_step": h2d * world,
               "d2h_bytes_per_step": d2h * world, "steps": args.e2e_steps,
               "api": "nimbus_cuda_acoustic_batched + nimbus_cuda_scalar_transport, NIMBUS_MEMORY_HOST"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(case)
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "unavailable", "sample": str(exc)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (stencils), f64 (base state, EOS, mass-flux sums)" if precision == cuda.PRECISION_FP32
            else "f64 arithmetic, f32 storage",
            "data": "synthetic (seeded WK82 supercell: analytic sounding, cos^2 bubble, theta noise)",
            "config": {"workload": args.workload, "grid": list(case.shape), "dx_m": case.dx, "dz_m": case.dz,
                       "dt_s": case.dt, "acoustic_substeps": n_sub, "scalars": 4,
                       "path": "acoustic loop (mass flux, fused substep, KW78 boundaries) + WENO5 transport",
                       "precision": args.precision,
                       "precision_modes": {
                           args.precision: {"value": value, "ms_per_step": ms / args.steps},
                           ("reference" if args.precision == "fp32" else "fp32"): {
                               "value": cells_total * 1e3 / alt_ms if world == 1 else None, "ms_per_step": alt_ms}},
                       "substep_form": {"chosen": args.substep_form if form != cuda.SUBSTEP_AUTO else
                                        ("fused" if run.tuned and run.tuned[0] == 1 else "split"),
                                        "autotune_ms_per_substep": run.tuned[1] if run.tuned else None},
                       "parallelism": f"{world} independent member(s), one per GPU",
                       "l2": "inputs larger than L2 (resident state ~%d MB per GPU)" % (case.cells * 4 * 17 // 2**20)},
            "roofline": {"bound": "hbm",
                         "kernel": "acoustic substep (%s form)" % (args.substep_form if form != cuda.SUBSTEP_AUTO else
                                                                   ("fused" if run.tuned and run.tuned[0] == 1 else "split")),
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_cell": SUBSTEP_BYTES_PER_CELL,
                         "substep_ms": substep_ms, "kernel_shares": shares},
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


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
