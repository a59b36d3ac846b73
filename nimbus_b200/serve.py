"""Serving loop: continuous batching of supercell runs on one GPU.

Requests arrive over time, each a run of its own grid and number of large
steps.  The server keeps every admitted run resident in HBM inside one
member engine and advances all of them together, one batched large step per
iteration; between iterations it retires the runs that finished (reading
their final state back) and admits queued runs in arrival order while their
footprint fits the free device memory (cudaMemGetInfo, less a reserve), the
admission rule of include/compute/compute_memory_admission.hpp.  A run's
result does not depend on which other runs shared its launches.

serve_one_by_one is the comparison: the same stream run sequentially, each
request alone on the plain per-operation path.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import cuda
from .initial import initial_state
from .run import EngineRun, ResidentRun


@dataclass
class Completion:
    rid: int
    arrival_s: float
    admitted_s: float
    done_s: float
    cells: int
    steps: int
    status: int = 0
    state: dict = field(default=None, repr=False)

    @property
    def latency_s(self) -> float:
        return self.done_s - self.arrival_s


def summarize(done: list, makespan_s: float) -> dict:
    lat = np.array([c.latency_s for c in done]) if done else np.zeros(1)
    work = sum(c.cells * c.steps for c in done)
    return {"requests": len(done), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "makespan_s": makespan_s,
            "cell_updates_per_s": work / makespan_s if makespan_s > 0 else None,
            "failed": sum(1 for c in done if c.status)}


class Server:
    def __init__(self, ctx: cuda.Context, precision: int = cuda.PRECISION_FP32, reserve_bytes: int = 4 << 30,
                 keep_results: bool = False, max_chunk: int = 8):
        self.ctx = ctx
        self.run = EngineRun(ctx, precision)
        self.reserve = reserve_bytes
        self.keep = keep_results
        self.max_chunk = max_chunk

    def close(self):
        self.run.close()

    def serve(self, requests: list, prepared=None) -> tuple:
        """Serve a request stream in real time; returns (completions, makespan_s).
        `prepared` maps rid -> (state, base) to keep host-side set-up out of the
        measured loop (pinned arrays upload without blocking the loop).

        Nothing here waits for the device except to learn a completion: the
        engine admits with stream-ordered allocation and copies, retires with
        a stream-ordered free, and rebuilds its step graphs in place; a
        finished run's final state (when kept) is read asynchronously behind
        its last step, and its completion is the moment the event recorded
        there fires.  The engine itself stays at most about one step ahead of
        the device (it reads each step's substep counts from the scan of the
        state that step starts from)."""
        import torch

        eng = self.run.engine
        stream = torch.cuda.ExternalStream(eng.stream)
        pending = sorted(requests, key=lambda r: (r.arrival_s, r.rid))
        queue = []
        active = {}     # member id -> [request, remaining steps, admitted_s]
        finishing = []  # (request, admitted_s, event, kept state, member id)
        done = []
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731

        def harvest(block=False):
            while finishing and (block or finishing[0][2].query()):
                r, admitted, ev, state, flags = finishing.pop(0)
                ev.synchronize()
                done.append(Completion(r.rid, r.arrival_s, admitted, now(), r.case.cells, r.steps, int(flags[0]),
                                       state))
                block = False

        while pending or queue or active or finishing:
            t = now()
            while pending and pending[0].arrival_s <= t:
                queue.append(pending.pop(0))
            while queue:  # FIFO admission while the head fits
                r = queue[0]
                state, base = prepared[r.rid] if prepared else initial_state(r.case)
                # the substep count is re-derived before every step, as the reference does
                desc = cuda.member_desc(r.case.shape, (r.case.dx, r.case.dy, r.case.dz), r.case.dt,
                                        r.case.substeps, r.case.bc, base, resolve_substeps=True)
                mid = eng.try_admit(desc, state, self.reserve)
                if mid is None:
                    if not active and not finishing:
                        raise RuntimeError(f"request {r.rid} does not fit an empty device")
                    break
                queue.pop(0)
                eng.shapes[mid] = r.case.shape
                active[mid] = [r, r.steps, now()]
            harvest()
            if not active:
                if finishing:
                    harvest(block=True)
                elif pending:
                    time.sleep(max(0.0, min(pending[0].arrival_s - now(), 0.05)))
                continue
            # Advance every resident run; several steps at once when no
            # arrival is due and no run finishes sooner.
            soonest = min(v[1] for v in active.values())
            due = queue or (pending and pending[0].arrival_s <= now() + 0.005)
            chunk = 1 if due else min(soonest, self.max_chunk)
            self.ctx.set_precision(self.run.precision)
            eng.step(chunk)
            for mid in list(active):
                rec = active[mid]
                rec[1] -= chunk
                if rec[1] <= 0:
                    r = rec[0]
                    state = None
                    if self.keep:
                        state = {k: np.empty(r.case.shape, np.float32) for k in cuda.MEMBER_FIELDS}
                        eng.read_async(mid, state)
                    # the run's status bits (refused EOS projection, non-finite
                    # flux) land in pinned memory behind its last step
                    flags = torch.zeros(1, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
                    eng.member_status_async(mid, flags)
                    ev = torch.cuda.Event()
                    ev.record(stream)
                    eng.retire(mid)
                    del active[mid]
                    finishing.append((r, rec[2], ev, state, flags))
        return done, now()


def serve_one_by_one(ctx: cuda.Context, requests: list, precision: int = cuda.PRECISION_FP32, prepared=None,
                     keep_results: bool = False) -> tuple:
    """The same stream, each request run alone on the plain path, in arrival order."""
    import torch

    done = []
    t0 = time.perf_counter()
    for r in sorted(requests, key=lambda q: (q.arrival_s, q.rid)):
        wait = r.arrival_s - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        start = time.perf_counter() - t0
        state, base = prepared[r.rid] if prepared else initial_state(r.case)
        run = ResidentRun(ctx, r.case, {k: v.copy() for k, v in state.items()}, base, precision=precision,
                          autotune=False)
        for _ in range(r.steps):
            run.step()
        run.torch_stream.synchronize()
        state_out = run.download() if keep_results else None
        done.append(Completion(r.rid, r.arrival_s, start, time.perf_counter() - t0, r.case.cells, r.steps, 0,
                               state_out))
        del run
        torch.cuda.empty_cache()
    return done, time.perf_counter() - t0
