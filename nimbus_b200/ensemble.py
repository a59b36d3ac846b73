"""Ensemble and request workloads, and their placement on GPUs.

* ensemble_cases: the ragged ensemble -- members whose grids are drawn from a
  seed, nx = ny = round(48 * 4**u), nz = round(40 * 1.6**u) with u ~ U(0, 1),
  dx = 500 m, uniform dz = 20 km / nz, dt = 3 s (3 * dx / 500 m), seeded theta'
  noise of +-0.2 K below 1 km and a bubble amplitude U(2, 4) K per member.
  The acoustic substep count follows the reference's CFL rule per member, so
  it differs between members.
* request_stream: served runs -- Poisson arrivals (mean 4 per second), grids
  log-uniform from 32x32x40 to 256x256x80, model durations U(60, 600) s.
* shard: greedy size-balanced partition of members across ranks (largest
  work first onto the least-loaded rank); members are independent, so no
  collective is needed on the data path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .initial import Case, initial_state
from .run import substeps_for


def ensemble_cases(members: int = 64, seed: int = 2026, dx: float = 500.0) -> list:
    rng = np.random.default_rng(seed)
    u = rng.uniform(0.0, 1.0, members)
    amp = rng.uniform(2.0, 4.0, members)
    cases = []
    for m in range(members):
        n = int(round(48 * 4.0 ** u[m]))
        nz = int(round(40 * 1.6 ** u[m]))
        cases.append(Case(n, n, nz, dx, dx, 20000.0 / nz, 3.0 * dx / 500.0, noise_amp=0.2, noise_depth=1000.0,
                          bubble_amp=float(amp[m]), seed=seed, member=m))
    return cases


@dataclass
class Request:
    rid: int
    case: Case
    steps: int
    arrival_s: float


def request_stream(count: int = 48, rate_per_s: float = 4.0, seed: int = 7, dx: float = 500.0,
                   burst: bool = False) -> list:
    """Seeded request stream; burst=True makes every request arrive at t=0."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, count)
    arrivals = np.zeros(count) if burst else np.cumsum(gaps) - gaps[0]
    u = rng.uniform(0.0, 1.0, count)
    duration = rng.uniform(60.0, 600.0, count)
    dt = 3.0 * dx / 500.0
    out = []
    for r in range(count):
        n = int(round(32 * 8.0 ** u[r]))
        nz = int(round(40 * 2.0 ** u[r]))
        case = Case(n, n, nz, dx, dx, 20000.0 / nz, dt, noise_amp=0.2, noise_depth=1000.0, seed=seed, member=r)
        out.append(Request(r, case, int(math.ceil(duration[r] / dt)), float(arrivals[r])))
    return out


def member_work(case: Case, n_substeps: int) -> float:
    """Relative cost of one large step: cells times (acoustic substeps + the
    rest of the step, about two substeps' worth of traffic)."""
    return float(case.cells) * (n_substeps + 2)


def shard(cases: list, world: int, rank: int, works=None) -> list:
    """Indices of the members rank `rank` owns under a greedy size-balanced
    split (deterministic: ties go to the lower rank)."""
    if works is None:
        works = []
        for c in cases:
            st, base = initial_state(Case(4, 4, c.nz, c.dx, c.dy, c.dz, c.dt, substeps=c.substeps))
            works.append(member_work(c, substeps_for(c, st, base)))
    order = sorted(range(len(cases)), key=lambda i: (-works[i], i))
    load = [0.0] * world
    owner = [0] * len(cases)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += works[i]
    return [i for i in range(len(cases)) if owner[i] == rank]
