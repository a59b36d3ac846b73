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


def _small_ensemble():
    """Six small supercells of different grids (the ensemble's generator at
    a reduced size), for stepping on the CPU oracle."""
    from nimbus_b200.initial import Case
    rng = np.random.default_rng(12)
    out = []
    for m in range(6):
        n = int(rng.integers(10, 17))
        nz = int(rng.integers(8, 13))
        out.append(Case(n, n + m % 2, nz, 1000.0, 1000.0, 8000.0 / nz, 5.0, bubble_rh=4000.0, noise_amp=0.2,
                        seed=3, member=m, bubble_amp=float(rng.uniform(2, 4))))
    return out


def _advance(cases, indices, steps=2):
    """Advance the members `indices` with the oracle, substep counts
    re-derived before every step; returns {index: state}."""
    import oracle
    from nimbus_b200.initial import initial_state
    o = oracle.Restatement("f32")
    out = {}
    for i in indices:
        c = cases[i]
        st, base = initial_state(c)
        o.run(st, base, (c.dx, c.dy, c.dz), c.dt, steps, c.bc)
        out[i] = st
    return out


def _shard_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cases = _small_ensemble()
    works = [member_work(c, 6) for c in cases]
    mine = shard(cases, world, rank, works)
    states = _advance(cases, mine)
    gathered = [None] * world
    dist.all_gather_object(gathered, states)
    if rank == 0:
        merged = {}
        for part in gathered:
            merged.update(part)
        out.put(merged)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.skipif(not __import__("oracle").restatement_available(), reason="oracle restatement not built")
def test_sharded_ensemble_equals_single_rank_run():
    """Strong scaling's data path: each of two gloo ranks advances only the
    members the size-balanced placement gives it; the gathered states equal a
    single-rank run of the whole ensemble bit for bit (members share nothing,
    so no collective exists on the data path)."""
    import socket
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_shard_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    cases = _small_ensemble()
    assert sorted(merged) == list(range(len(cases)))
    alone = _advance(cases, range(len(cases)))
    for i in range(len(cases)):
        for k, a in alone[i].items():
            assert np.array_equal(a.view(np.uint32), merged[i][k].view(np.uint32)), (i, k)
