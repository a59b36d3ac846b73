"""Device-resident runs of the hot path.

One large step (the order of step_dynamics_new, dynamics.cpp:5123-7317, for
the phases this backend owns):
  1. Heun slow step: k1, predictor, k2, the FP32 average applied with dt
     (prepare_slow_rk2_tendencies + apply_slow_tendencies);
  2. boundary refresh apply_acoustic(0) and the KW78 seed
     (seed_acoustic_radiation, dynamics.cpp:5384-5396);
  3. the acoustic loop: N substeps, each with the retained mass-flux
     accumulation, continuity + EOS, momentum and the boundary closure
     (split_explicit.cpp:174-260);
  4. conservative WENO5 transport of theta, qv, qc, qr against the retained
     fluxes and densities (advection_batch.cpp:565-760);
  5. the Kessler step over the C-grid cell domain (microphysics_step.cpp),
     then optionally the explicit Smagorinsky SGS integration
     (dynamics.cpp:7151-7250; ResidentRun only);
  6. the EOS pressure re-projection (eos_apply.cpp);
  7. optionally the end-of-step sponge (rayleigh_damping.cpp, called at
     dynamics.cpp:7323-7340) and the closing boundary refresh
     (apply_full_attributed, dynamics.cpp:7415).

Two drivers run it:
  ResidentRun   the plain path: one run, each operation enqueued through its
                own C-ABI entry point (the per-dispatch interface the
                reference's compute backends expose);
  EngineRun     the member engine: any number of runs, one batched launch per
                phase, the step replayed from a CUDA graph.
PyTorch only owns device memory for ResidentRun; every kernel is the
library's.
"""
from __future__ import annotations

import numpy as np
import torch

from . import cuda
from .initial import Case, initial_state, max_sound_speed, resolve_substep_count

SCALARS = ("theta", "qv", "qc", "qr")
POSITIVE = (0, 1, 1, 1)  # theta is the only non-positive-definite scalar (advection_batch.cpp:742-745)
PROGNOSTIC = ("u", "v", "w", "rho", "p") + SCALARS


def substeps_for(case: Case, state, base) -> int:
    return resolve_substep_count(case.dt, max_sound_speed(state["p"], state["rho"], base), case.dx, case.dy,
                                 case.dz, case.substeps)


class ResidentRun:
    def __init__(self, ctx: cuda.Context, case: Case, state=None, base=None, device="cuda",
                 precision: int = cuda.PRECISION_FP32, autotune: bool = True, coriolis_f: float = 0.0,
                 microphysics: bool = True, sponge=None, final_closure: bool = False, sgs=None,
                 resolve: bool = True):
        self.ctx = ctx
        self.precision = precision
        self.tuned = None
        if autotune:
            ctx.set_precision(precision)
            self.tuned = ctx.autotune_substep(case.nx, case.ny, case.nz)
        self.case = case
        if state is None:
            state, base = initial_state(case)
        self.base = base
        self.microphysics = microphysics
        self.n_substeps = substeps_for(case, state, base)
        dev = torch.device(device)
        self.fields = {k: torch.from_numpy(np.ascontiguousarray(state[k])).to(dev) for k in PROGNOSTIC}
        shape = case.shape
        self.mf = [torch.zeros(shape, dtype=torch.float32, device=dev) for _ in range(3)]
        self.rho_begin = torch.zeros(shape, dtype=torch.float32, device=dev)
        self.wave = torch.zeros(2 * (case.nx + case.ny) * case.nz, dtype=torch.float32, device=dev)
        self.prof = {k: torch.from_numpy(np.ascontiguousarray(base[k], dtype=np.float64)).to(dev)
                     for k in ("rho0", "p0", "qv0", "u0", "v0")}
        self.stream = ctx.stream
        grid = (case.dx, case.dy, case.dz)
        n = self.n_substeps
        f = self.fields
        self._slow = cuda.slow_args(f, self.prof, grid, dt_large=case.dt, coriolis_f=coriolis_f,
                                    memory=cuda.MEMORY_DEVICE)
        self._refresh = cuda.boundary_args(f, grid, case.bc, 0.0)
        # resolve: the substep count re-derived from the state before every
        # large step, as the reference does (one device scan of p and rho and
        # a host wait per step); otherwise the admission count throughout.
        self.resolve = resolve
        self.substep_counts = []
        self._loop = self._loop_args(n)
        qs = [f[k] for k in SCALARS]
        self._transport = cuda.transport_args(qs, qs, POSITIVE, f["rho"], self.rho_begin, *self.mf, case.dt,
                                              grid, weno=True, top_open=case.bc[5] == 2, memory=cuda.MEMORY_DEVICE)
        self._kessler = cuda.kessler_args(f, case.dz, case.dt, memory=cuda.MEMORY_DEVICE)
        self._eos = cuda.eos_args(f["p"], f["rho"], f["theta"], f["qv"], f["qc"], f["qr"], memory=cuda.MEMORY_DEVICE,
                                  p0=self.prof["p0"])
        # The end-of-step sponge (SpongeProfiles), after the EOS projection.
        self._sponge = (cuda.state_relaxation_args(f, sponge, case.dt, memory=cuda.MEMORY_DEVICE)
                        if sponge is not None else None)
        self.final_closure = final_closure
        # The explicit Smagorinsky SGS integration (nimbus_b200.sgs.SgsConfig).
        self.time_s = 0.0
        self.sgs_substeps = 0
        self._sgs = (cuda.sgs_step_args(f, np.full(case.nz, case.dz), grid, sgs, case.dt, theta0=base["theta0"])
                     if sgs is not None else None)
        self.torch_stream = torch.cuda.ExternalStream(self.stream, device=dev)

    def _loop_args(self, n: int):
        case = self.case
        grid = (case.dx, case.dy, case.dz)
        return cuda.batched_args(self.fields, self.prof["rho0"], self.prof["p0"], case.dt / n, n, grid, case.bc,
                                 *self.mf, (case.dt / n) / case.dt, None, self.wave, self.rho_begin,
                                 memory=cuda.MEMORY_DEVICE)

    @property
    def cells(self) -> int:
        return self.case.cells

    def resolve_substeps(self) -> int:
        """The substep count the reference would use for the next large step
        from the current device state (waits for enqueued work)."""
        case, c = self.case, self.ctx
        c_max = c.max_sound_speed(self.fields["p"], self.fields["rho"], case.shape, self.base)
        return c.resolve_substep_count(case.dt, c_max, min(case.dx, case.dy, case.dz), case.substeps)

    def step(self):
        """Enqueue one large step on the context stream (without resolve, no
        host synchronisation)."""
        c = self.ctx
        c.set_precision(self.precision)
        if self.resolve:
            n = self.resolve_substeps()
            if n != self.n_substeps:
                self.n_substeps = n
                self._loop = self._loop_args(n)
        self.substep_counts.append(self.n_substeps)
        c.check(c.slow_step(self._slow))
        c.check(c.acoustic_boundaries(self._refresh))
        with torch.cuda.stream(self.torch_stream):
            for m in self.mf:
                m.zero_()
        c.check(c.acoustic_batched(self._loop))
        c.check(c.scalar_transport(self._transport))
        if self.microphysics:
            c.check(c.kessler_step(self._kessler))
        if self._sgs is not None:  # synchronises once per SGS substep
            self._sgs.time_s = self.time_s
            count, _ = c.sgs_step(self._sgs)
            self.sgs_substeps += count
        c.check(c.eos_projection(self._eos))
        if self._sponge is not None:
            c.check(c.state_relaxation(self._sponge))
        if self.final_closure:  # apply_full_attributed = apply_acoustic(0)
            c.check(c.acoustic_boundaries(self._refresh))
        self.time_s += self.case.dt

    def download(self) -> dict:
        torch.cuda.current_stream().wait_stream(self.torch_stream)
        self.torch_stream.synchronize()
        return {k: v.cpu().numpy() for k, v in self.fields.items()}


class EngineRun:
    """Runs resident in one member engine, advanced together."""

    def __init__(self, ctx: cuda.Context, precision: int = cuda.PRECISION_FP32, graph: bool = True,
                 lanes: int | None = None):
        self.ctx = ctx
        self.precision = precision
        self.engine = cuda.Engine(ctx)
        self.engine.set_graph(graph)
        if lanes is not None:
            self.engine.set_lanes(lanes)
        self.members = {}

    def admit(self, case: Case, state=None, base=None, coriolis_f: float = 0.0, microphysics: bool = True,
              reserve_bytes: int = 0, n_substeps: int | None = None, sponge=None, final_closure: bool = False,
              resolve: bool | None = None):
        """Admit a run.  Without n_substeps (or with resolve=True) the engine
        re-derives its substep count before every large step from the live
        state, with case.substeps (or n_substeps) as the requested minimum,
        as the reference does; an explicit n_substeps alone fixes the count."""
        if state is None:
            state, base = initial_state(case)
        if resolve is None:
            resolve = n_substeps is None
        n = n_substeps if n_substeps is not None else (case.substeps if resolve else substeps_for(case, state, base))
        desc = cuda.member_desc(case.shape, (case.dx, case.dy, case.dz), case.dt, n, case.bc, base, coriolis_f,
                                microphysics=int(microphysics), sponge=sponge, final_closure=final_closure,
                                resolve_substeps=resolve)
        mid = self.engine.admit(desc, state, reserve_bytes)
        self.members[mid] = (case, self.engine.member_substeps(mid))
        return mid

    def substeps(self, member_id: int) -> int:
        """Substep count of the member's last enqueued (or first) large step."""
        return self.engine.member_substeps(member_id)

    def step(self, n: int = 1):
        self.ctx.set_precision(self.precision)
        self.engine.step(n)

    def read(self, member_id: int) -> dict:
        return self.engine.read(member_id)

    @property
    def cells(self) -> int:
        return sum(c.cells for c, _ in self.members.values())

    def close(self):
        self.engine.close()


class HostPipeline:
    """Large steps through the library's host-buffer API: every step uploads
    each run's state from pinned host memory, advances it and reads it back,
    so all host<->device copies are inside the step.

    The runs are split over `groups` engines, each on its own stream, and each
    engine's runs live in one pinned host block laid out as its state image
    (nimbus_cuda_engine_image_*): a step moves it with one copy each way, and
    one group's copies overlap another group's step."""

    def __init__(self, ctx: cuda.Context, cases, prepared=None, groups: int = 8,
                 precision: int = cuda.PRECISION_FP32, lanes: int | None = 1):
        self.ctx = ctx
        self.precision = precision
        prepared = prepared or [initial_state(c) for c in cases]
        order = sorted(range(len(cases)), key=lambda i: -cases[i].cells)
        groups = max(1, min(groups, len(cases)))
        self.runs = [EngineRun(ctx, precision, lanes=lanes) for _ in range(groups)]
        placed = []
        for r, idx in enumerate(order):
            run = self.runs[r % groups]
            st, base = prepared[idx]
            placed.append((run, run.admit(cases[idx], st, base), st))
        self.images = []
        views = {}
        for run in self.runs:
            img = torch.empty(max(run.engine.image_bytes(), 4), dtype=torch.uint8).pin_memory().numpy()
            self.images.append(img)
            views[id(run)] = run.engine.image_views(img)
        self.host = []  # (run, member id, {field: view into the group's pinned image})
        for run, mid, st in placed:
            arrays = views[id(run)][mid]
            for k in PROGNOSTIC:
                arrays[k][...] = st[k]
            self.host.append((run, mid, arrays))
        self.cells = sum(c.cells for c in cases)
        self._pool = None

    def bytes_per_step(self):
        """Host<->device bytes one step moves (the nine prognostic fields each way)."""
        n = self.cells * 4 * len(PROGNOSTIC)
        return n, n

    def step(self, n: int = 1):
        """n large steps, each uploading every state, advancing it and reading it
        back; each engine's stream orders step k's download before step k+1's
        upload of the same host block, so consecutive steps of different groups
        overlap.  Each group is driven from its own host thread: a step waits
        for its group's acoustic speed scan (the substep counts depend on the
        uploaded state), and the other groups keep enqueuing meanwhile (the
        library calls release the interpreter lock).  Waits for all of them
        before returning."""
        from concurrent.futures import ThreadPoolExecutor

        self.ctx.set_precision(self.precision)

        def drive(pair):
            run, image = pair
            for _ in range(n):
                run.engine.upload_image_async(image)
                run.engine.step(1)
                run.engine.download_image_async(image)
            run.engine.synchronize()

        if self._pool is None:
            self._pool = ThreadPoolExecutor(max_workers=len(self.runs))
        for f in [self._pool.submit(drive, pair) for pair in zip(self.runs, self.images)]:
            f.result()

    def close(self):
        if self._pool is not None:
            self._pool.shutdown()
            self._pool = None
        for run in self.runs:
            run.close()
