"""Host logic of the ensemble and serving workloads: seeded member and request
generation, the greedy size-balanced placement of members on ranks, and the
placement exercised across two real ranks (gloo on CPU, 127.0.0.1)."""
import math
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from nimbus_b200.ensemble import ensemble_cases, member_work, request_stream, shard


def test_ensemble_is_seeded_ragged_and_in_range():
    a = ensemble_cases(64, seed=2026)
    b = ensemble_cases(64, seed=2026)
    assert [c.shape for c in a] == [c.shape for c in b]
    assert len(a) == 64
    for c in a:
        assert 48 <= c.nx <= 192 and c.nx == c.ny and 40 <= c.nz <= 64
        assert math.isclose(c.dz * c.nz, 20000.0) and c.dx == 500.0 and c.dt == 3.0
        assert 2.0 <= c.bubble_amp <= 4.0 and c.noise_amp == 0.2
    assert len({c.shape for c in a}) > 32
    total = sum(c.cells for c in a)
    assert 20e6 < total < 80e6
    assert [c.shape for c in ensemble_cases(64, seed=1)] != [c.shape for c in a]


def test_request_stream():
    reqs = request_stream(400, rate_per_s=4.0, seed=7)
    arr = np.array([r.arrival_s for r in reqs])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    assert 3.0 < len(reqs) / arr[-1] < 5.0  # mean rate 4/s
    for r in reqs:
        assert 32 <= r.case.nx <= 256 and 40 <= r.case.nz <= 80
        assert 20 <= r.steps <= 200
    burst = request_stream(10, burst=True)
    assert all(r.arrival_s == 0.0 for r in burst)


def _works(cases):
    return [member_work(c, 8 + (c.member % 3)) for c in cases]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_is_a_balanced_partition(world):
    cases = ensemble_cases(64)
    works = _works(cases)
    parts = [shard(cases, world, r, works) for r in range(world)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    loads = [sum(works[i] for i in p) for p in parts]
    # greedy LPT bound: no rank exceeds the ideal share by more than one member
    assert max(loads) - sum(loads) / world <= max(works) + 1e-9


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    cases = ensemble_cases(16, seed=5)
    works = _works(cases)
    mine = shard(cases, world, rank, works)
    sizes = [None] * world
    dist.all_gather_object(sizes, mine)
    # The bench times each rank on the device and reports the max over ranks.
    t = torch.tensor([float(sum(works[i] for i in mine))], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((sizes, float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_agree_on_the_placement():
    import socket
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    sizes, slowest = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(sizes[0] + sizes[1]) == list(range(16)) and not set(sizes[0]) & set(sizes[1])
    works = _works(ensemble_cases(16, seed=5))
    assert slowest == max(sum(works[i] for i in sizes[r]) for r in range(2))
