"""Device-resident single run: the state of one supercell stays in HBM and
each large step of the hot path is enqueued through the C-ABI.

One large step (the order of step_dynamics_new, dynamics.cpp:6590-6961, for
the hot path it owns):
  1. open the retained transport context: zero the face mass-flux sums
     (CartesianCGridTransportContext::begin);
  2. the acoustic loop: N substeps, each with mass-flux accumulation, the
     fused substep and the boundary closure; the KW78 radiation memory is
     re-seeded from the live faces at the start of every large step, as
     seed_acoustic_radiation does (split_explicit.cpp:174-205);
  3. conservative WENO5 transport of theta, qv, qc, qr against the retained
     fluxes and densities (advection_batch.cpp:565-760).

PyTorch is used only to own device memory; every kernel is the library's.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import cuda
from .initial import Case, initial_state, max_sound_speed, resolve_substep_count

SCALARS = ("theta", "qv", "qc", "qr")
POSITIVE = (0, 1, 1, 1)  # theta is the only non-positive-definite scalar (advection_batch.cpp:742-745)
PROGNOSTIC = ("u", "v", "w", "rho", "p") + SCALARS


class ResidentRun:
    def __init__(self, ctx: cuda.Context, case: Case, state=None, base=None, device="cuda",
                 precision: int = cuda.PRECISION_FP32, autotune: bool = True):
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
        self.n_substeps = resolve_substep_count(case.dt, max_sound_speed(state["p"], state["rho"], base), case.dx,
                                                case.dy, case.dz, case.substeps)
        dev = torch.device(device)
        self.fields = {k: torch.from_numpy(np.ascontiguousarray(state[k])).to(dev) for k in PROGNOSTIC}
        shape = case.shape
        self.mf = [torch.zeros(shape, dtype=torch.float32, device=dev) for _ in range(3)]
        self.rho_begin = torch.zeros(shape, dtype=torch.float32, device=dev)
        self.wave = torch.zeros(2 * (case.nx + case.ny) * case.nz, dtype=torch.float32, device=dev)
        self.rho0 = torch.from_numpy(base["rho0"]).to(dev)
        self.p0 = torch.from_numpy(base["p0"]).to(dev)
        self.stream = ctx.stream
        grid = (case.dx, case.dy, case.dz)
        n = self.n_substeps
        self._loop = cuda.batched_args(self.fields, self.rho0, self.p0, case.dt / n, n, grid, case.bc, *self.mf,
                                       (case.dt / n) / case.dt, None, self.wave, self.rho_begin,
                                       memory=cuda.MEMORY_DEVICE)
        qs = [self.fields[k] for k in SCALARS]
        self._transport = cuda.transport_args(qs, qs, POSITIVE, self.fields["rho"], self.rho_begin, *self.mf, case.dt,
                                              grid, weno=True, top_open=case.bc[5] == 2, memory=cuda.MEMORY_DEVICE)
        self.torch_stream = torch.cuda.ExternalStream(self.stream, device=dev)

    @property
    def cells(self) -> int:
        return self.case.cells

    def step(self):
        """Enqueue one large step on the context stream (no host synchronisation)."""
        self.ctx.set_precision(self.precision)
        with torch.cuda.stream(self.torch_stream):
            for m in self.mf:
                m.zero_()
        self.ctx.check(self.ctx.acoustic_batched(self._loop))
        self.ctx.check(self.ctx.scalar_transport(self._transport))

    def download(self) -> dict:
        torch.cuda.current_stream().wait_stream(self.torch_stream)
        self.torch_stream.synchronize()
        return {k: v.cpu().numpy() for k, v in self.fields.items()}


class HostStepper:
    """The same large step through the reference-facing host-memory API:
    every call uploads its inputs from (pinned) host arrays and returns the
    results to them, as the reference's fence-confirmed dispatches do."""

    def __init__(self, ctx: cuda.Context, case: Case, state=None, base=None, pin=True,
                 precision: int = cuda.PRECISION_FP32):
        self.ctx = ctx
        self.precision = precision
        self.case = case
        if state is None:
            state, base = initial_state(case)
        self.base = base
        self.n_substeps = resolve_substep_count(case.dt, max_sound_speed(state["p"], state["rho"], base), case.dx,
                                                case.dy, case.dz, case.substeps)

        def host(a):
            t = torch.from_numpy(np.ascontiguousarray(a))
            return (t.pin_memory() if pin else t.clone()).numpy()

        self.fields = {k: host(state[k]) for k in PROGNOSTIC}
        shape = case.shape
        self.mf = [host(np.zeros(shape, np.float32)) for _ in range(3)]
        self.rho_begin = host(np.zeros(shape, np.float32))
        self.wave = host(np.zeros(2 * (case.nx + case.ny) * case.nz, np.float32))
        grid = (case.dx, case.dy, case.dz)
        n = self.n_substeps
        self._loop = cuda.batched_args(self.fields, base["rho0"], base["p0"], case.dt / n, n, grid, case.bc, *self.mf,
                                       (case.dt / n) / case.dt, None, self.wave, self.rho_begin)
        qs = [self.fields[k] for k in SCALARS]
        self._transport = cuda.transport_args(qs, qs, POSITIVE, self.fields["rho"], self.rho_begin, *self.mf, case.dt,
                                              grid, weno=True, top_open=case.bc[5] == 2)

    def bytes_per_step(self):
        """Host<->device bytes one step moves through the host API (counted
        from the arrays each call stages)."""
        n = self.case.cells * 4
        w = self.wave.nbytes
        prof = self.base["rho0"].nbytes + self.base["p0"].nbytes
        # acoustic batch: in u,v,w,rho,p,theta + 3 mass fluxes + profiles (the KW78
        #                 memory is seeded on the device); out u,v,w,rho,p + 3 mass
        #                 fluxes + rho_begin + wave history
        # transport:      in rho_end, rho_begin, 3 mass fluxes, 4 scalars; out 4 scalars
        h2d = 9 * n + prof + 9 * n
        d2h = 9 * n + w + 4 * n
        return h2d, d2h

    def step(self):
        self.ctx.set_precision(self.precision)
        for m in self.mf:
            m[...] = 0.0
        self.ctx.check(self.ctx.acoustic_batched(self._loop))
        self.ctx.check(self.ctx.scalar_transport(self._transport))
